// Incremental marching cubes (placeholder: meshing not yet built).
#include "ff_mesh.h"

namespace ffb {

int mesh_update(MeshState &m, const MeshInputs &in, cudaStream_t s, std::string &err) {
  err = "meshing is not built yet";
  return 6;
}
int mesh_copy_out(MeshState &m, float *xyz, uint8_t *rgb, uint32_t *faces, cudaStream_t s, std::string &err) {
  return 0;
}
void mesh_free(MeshState &m) {}
void mesh_invalidate(MeshState &m) { m.valid = false; }
void mesh_note_frame(MeshState &m) {}

}  // namespace ffb
