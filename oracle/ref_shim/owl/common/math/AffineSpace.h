// TEST INFRASTRUCTURE ONLY.  The reference's dda.h includes OWL's AffineSpace.h but uses
// no affine type; the box and vector stand-ins are all it needs.
#pragma once

#include "box.h"
