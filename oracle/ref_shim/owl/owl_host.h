// TEST INFRASTRUCTURE ONLY.  Stand-in for OWL's host API header: the reference's
// renderer.h needs only the handle types, which owl/owl.h declares.
#pragma once

#include "owl.h"
