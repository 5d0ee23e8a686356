// Host-side launchers of the fusion-path kernels (internal to the library).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "ff_common.cuh"

namespace ffb {

// A leaf claimed during the frame's traversal, before its index is assigned.
struct PendingLeaf {
  uint32_t slot;         // tree entry that will hold the leaf index
  uint32_t first_pixel;  // smallest processed pixel index that queried it
  ushort4 pos;           // x, y, z, scale
};

// First-frame integer bounding box (geometryfusion_mipmap_cpu.cpp:1270-1303).
void launch_first_bbox(const uint16_t *depth, int W, int H, const CamF &p, float scaling, float maxcam, int bw,
                       Counters *cnt, cudaStream_t s);

// Per-pixel voxel coordinates, validity and target brick scale (written to
// vox), then the row/column de-duplication of brick keys
// (traversal_wrapper_functions.cpp:613-639, 688-690).
// bnd: 4 buffers of boundary state; barrier: 8 zeroed uint32 words.
// int4 elements of the boundary buffer launch_dedupe needs for a W x H image.
size_t dedupe_boundary_elems(int W, int H);
cudaError_t launch_dedupe(const uint16_t *depth, const float *pxp, const float *pyp, const CamF &cam, float scaling,
                          float maxcam, int4 *vox, int W, int H, int4 *bnd, uint8_t *processed, Counters *cnt,
                          uint32_t *barrier, int device, cudaStream_t s);

// Octree descent / allocation of every processed pixel.
void launch_insert(const int4 *vox, const uint8_t *processed, int W, int H, uint32_t n, int bw, uint32_t *tree,
                   uint32_t leaves_max, uint32_t branches_max, uint32_t frame, uint32_t *stamp, uint32_t *queue,
                   PendingLeaf *pend, uint32_t pend_cap, Counters *cnt, cudaStream_t s);

// Sort scratch size for `n` pending leaves.
size_t pending_sort_bytes(int n);
// Order pending leaves by first pixel; out_rec receives record ids.
cudaError_t sort_pending(const PendingLeaf *pend, int npend, uint32_t *keys_in, uint32_t *vals_in, uint32_t *keys_out,
                         uint32_t *vals_out, void *tmp, size_t tmp_bytes, int end_bit, cudaStream_t s);

// Assign leaf indices in creation order, fill the leaf table, queue new leaves.
void launch_finalize(const PendingLeaf *pend, const uint32_t *order, int npend, uint32_t leaves_before,
                     uint32_t leaves_max, uint32_t *tree, ushort4 *leaf, uint32_t frame, uint32_t *stamp,
                     uint32_t *queue, Counters *cnt, cudaStream_t s);
// Parent leaf of each new leaf: finest ancestor leaf created before it.
void launch_parents(int npend, uint32_t leaves_before, uint32_t leaves_max, const uint32_t *tree, uint32_t n,
                    const ushort4 *leaf, uint32_t *parent, cudaStream_t s);

// Whether launch_finalize_small takes a W x H frame.
bool finalize_small_fits(uint32_t npix);

// Ranks (creation order), leaf table and parents of the frame's pending
// leaves in one launch, for images of up to about 1.6 million pixels; false
// (nothing launched) for larger ones.  npend < 0: the count is read on the
// device.  rank_scratch: W*H uint32.
bool launch_finalize_small(const PendingLeaf *pend, int npend, uint32_t npix, uint32_t *rank_scratch,
                           uint32_t leaves_before, uint32_t leaves_max, uint32_t *tree, ushort4 *leaf,
                           uint32_t frame, uint32_t *stamp, uint32_t *queue, Counters *cnt, uint32_t n,
                           uint32_t *parent, int device, cudaStream_t s);

// Load the kernels of each file ahead of their first launch.
cudaError_t prewarm_alloc_kernels();
cudaError_t prewarm_fuse_kernels();
cudaError_t prewarm_mesh_kernels();

// grow(): move child-branch pointers by `shift`, leaf positions by `add`.
void launch_shift_branches(uint32_t *tree, uint32_t used, uint32_t shift, cudaStream_t s);
void launch_shift_leaves(ushort4 *leaf, uint32_t n_leaves, ushort3 add, cudaStream_t s);
void launch_fill(uint32_t *p, size_t n, uint32_t v, cudaStream_t s);

// Device-side gate of a frame's voxel update whose brick count the host has
// not read yet (cnt == nullptr: no gate, the host passes the count).
struct FuseGate {
  const Counters *cnt;
  uint32_t n, leaves_before, leaves_max, branches_max;
};

// Voxel update of the queued bricks (update_functions.cpp:1187-1444).
void launch_fuse(const uint32_t *queue, int nq, const FuseGate &gate, const ushort4 *leaf, float *sdf, float *wgt,
                 __half *sdf16, __half *wgt16, uint16_t *col, int storage, const uint16_t *depth, const uint8_t *bgr,
                 int W, int H, const CamF &q, float scale, float thr, float scaling, float maxcam,
                 const uint32_t *rcp_tab, int rcp_shift, cudaStream_t s);

// Table of the host CPU's RCPPS over the mantissas of [1,2), indexed by the
// mantissa >> shift (the low bits the instruction ignores are dropped); false
// when the host is not x86-64 or the instruction does not follow the
// expected rules.
bool build_rcp_table(std::vector<uint32_t> &tab, int &shift);

}  // namespace ffb
