// TEST INFRASTRUCTURE ONLY.  Stand-in for the umesh library's mesh type (submodule
// empty): the reference's renderer.h holds shared pointers to it and renderer.cu's
// unstructured-mesh path reads its element lists; the raw-volume path the pins run
// never touches a mesh.
#pragma once

#include <cstddef>
#include <memory>
#include <vector>

namespace umesh {
struct UMesh {
  typedef std::shared_ptr<UMesh> SP;
  struct Elem { int idx[8]; };
  struct Vertex { float x, y, z; };
  std::vector<Elem> tets, pyrs, wedges, hexes;
  std::vector<Vertex> vertices;
  size_t numVolumeElements() const { return tets.size() + pyrs.size() + wedges.size() + hexes.size(); }
};
}  // namespace umesh
