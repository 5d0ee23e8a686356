// Incremental marching cubes over the dual cells of the brick octree
// (internal interface of the library).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "ff_common.cuh"
#include "ff_prof.h"

namespace ffb {

struct MeshInputs {
  const uint32_t *tree;
  uint32_t branches_used;
  const ushort4 *leaf;
  const uint32_t *parent;
  const float *sdf, *wgt;
  const __half *sdf16, *wgt16;
  const uint16_t *col;
  int storage;
  uint32_t leaves_used, leaves_max;
  const uint32_t *stamp;  // frame of the last update of each brick
  // per branch: the last frame that created a branch or leaf at or below it
  const uint32_t *bstamp;
  uint32_t grows = 0;   // volume growths so far (a growth moves every cell)
  int full_cells = 0;   // regenerate every cell instead of the changed ones
  bool top_changed = true;  // a frame since the last update created something near the root
  uint32_t spin_limit = SPIN_LIMIT;  // bound of the traversal's grid barriers (polls)
  uint32_t frame;
  uint32_t n;
  float offset[3];
  float scale;
  Counters *cnt;
  Counters *h_cnt;
  Prof *prof;
  // a part of a sharded map: the cells it meshes (ff_set_shard)
  uint32_t shard = 0, shards = 1;
  int32_t shift[3] = {0, 0, 0};
};

struct MeshState {
  // output of the last update
  float *d_xyz = nullptr;
  uint8_t *d_rgb = nullptr;
  uint32_t *d_faces = nullptr;
  uint64_t n_vertices = 0, n_faces = 0;
  uint64_t cap_vertices = 0, cap_faces = 0;
  uint64_t n_cells = 0, n_dirty = 0, n_generated = 0;
  bool top_kept = false;  // the last update started from the kept top-level traversal items
  uint32_t last_frame = 0;
  bool valid = false;
  void *impl = nullptr;  // buffers private to ff_mesh.cu
};

// returns 0 or an ff_status value
int mesh_update(MeshState &m, const MeshInputs &in, cudaStream_t s, std::string &err);
int mesh_copy_out(MeshState &m, float *xyz, uint8_t *rgb, uint32_t *faces, cudaStream_t s, std::string &err);
// cells of the last update: 14 int32 each (type, quirk, ox, oy, oz, size, L0..L7) and per cell
// (first vertex, vertex count, first face, face count)
int mesh_copy_cells(MeshState &m, int32_t *rows, int64_t *ranges, cudaStream_t s, std::string &err);
// The same through a fixed file-scope device buffer (no allocation), for at
// most 65536 cells.
int mesh_copy_cells_noalloc(MeshState &m, int32_t *rows, int64_t *ranges, cudaStream_t s, std::string &err);
void mesh_free(MeshState &m);
// The device buffers the next mesh_update writes its mesh into (the mesh of
// the update before last; null before two updates): a copy out of them must
// finish first.
void mesh_next_outputs(MeshState &m, const void **xyz, const void **rgb, const void **faces);
void mesh_invalidate(MeshState &m);
void mesh_note_frame(MeshState &m);

}  // namespace ffb
