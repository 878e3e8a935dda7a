// TEST INFRASTRUCTURE ONLY.  Stand-in for the umesh library's mesh type (submodule
// empty): the reference's renderer.h holds shared pointers to it; the raw-volume path
// the pins run never touches a mesh.
#pragma once

#include <memory>

namespace umesh {
struct UMesh {
  typedef std::shared_ptr<UMesh> SP;
};
}  // namespace umesh
