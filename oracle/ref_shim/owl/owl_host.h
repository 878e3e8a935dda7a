// TEST INFRASTRUCTURE ONLY.  Stand-in for OWL's host API header: the reference's
// renderer.h needs only the handle types, which owl/owl.h declares; renderer.cu's host
// code also names the buffer and acceleration-structure calls below.  They are declared
// so that renderer.cu compiles (oracle/ref_gpu_pins.cu); the pins launch renderer.cu's
// kernels themselves and never call them (the definitions there abort).
#pragma once

#include <cstddef>

#include "owl.h"

typedef int OWLDataType;
#define OWL_USER_TYPE(T) ((OWLDataType)(1000 + (int)sizeof(T)))
OWLBuffer owlDeviceBufferCreate(OWLContext context, OWLDataType type, size_t count, const void *init);
const void *owlBufferGetPointer(OWLBuffer buffer, int deviceID);
void owlGroupBuildAccel(OWLGroup group);
