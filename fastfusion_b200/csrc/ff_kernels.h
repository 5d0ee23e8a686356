// Host-side launchers of the fusion-path kernels (internal to the library).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstddef>
#include <vector>

#include "ff_common.cuh"

namespace ffb {

// One map's frame as the per-frame kernels see it (device-resident, in a
// BatchDesc).  A batch holds the frames of several independent maps that
// the same launches process together; a single map is a batch of one.
struct PendingLeaf;
struct MapFrame {
  // the frame
  const uint16_t *depth;
  const uint8_t *bgr;
  const float *pxp, *pyp;  // per-column / per-row ray factors
  CamF p;                  // world -> voxel grid (traversal)
  CamF q;                  // voxel grid -> camera (update)
  float scaling, maxcam, scale, thr;
  int W, H, tilesX, tilesY;
  uint32_t npix, frame;
  // the map
  uint32_t n, bw, leaves_max, branches_max, leaves_before, pend_cap, nq_host;
  uint32_t *tree;
  ushort4 *leaf;
  uint32_t *parent;
  float *sdf, *wgt;
  __half *sdf16, *wgt16;
  uint16_t *col;
  uint32_t *stamp, *queue, *rank;
  // per branch (index = branch base / 16): the last frame that created a
  // branch or a leaf in the branch or below it (the mesher's test for
  // octree subtrees unchanged since its previous update)
  uint32_t *bstamp;
  PendingLeaf *pend;
  int4 *vox;
  uint8_t *proc;
  int4 *bnd;
  Counters *cnt;
  const uint32_t *rcp_tab;
  int rcp_shift;
  const float *conf;  // learned per-pixel confidence of the frame, or null (the reference's weight)
  // brick ownership: a map that is one of `shards` parts of a larger map
  // keeps only the bricks whose key hashes to `shard`; shift = the voxels
  // grow() has moved the grid by, so that keys do not change with growth
  uint32_t shard, shards;
  int32_t shift[3];
  // the frame's counters are set up by the de-duplication launch: zero, the
  // octree's branch count, and the in-volume box [0, n - 1]
  uint32_t branches_init;
  // iterations after which a device-side wait of this frame gives up
  uint32_t spin_limit;
  // the insert sums the octree levels it probes (the stage profile's bytes)
  uint32_t count_levels;
  // Deferred voxel update (upd_mask non-null): the leaf finalisation marks the
  // frame's queued bricks with bit upd_slot in upd_mask and appends bricks
  // not yet marked to upd_list (count in *upd_count); one k_fuse_multi pass
  // later updates every listed brick with all its marked frames in order.
  uint32_t *upd_mask, *upd_list, *upd_count;
  int32_t upd_slot;
  // A frame of a sequence of one map (ff_add_map_sequence_u16_device): all
  // its frames are de-duplicated in one launch, then inserted and finalised
  // frame after frame on the device.  chain: the frame's branch count and
  // leaf base come from the previous frame's finalisation (cnt->branches_used,
  // cnt->leaves_base) rather than from the host; next_cnt: the next frame's
  // counters, which this frame's finalisation sets up (or halts).
  uint32_t chain;
  Counters *next_cnt;
};

// Whether a frame's voxel update must not run with the others: an allocation
// error or a failed confidence network (the frame is not fused), or the
// volume must grow first (the host grows it and updates the frame itself).
// Mirrors the host's test after the traversal.
__device__ __forceinline__ bool fuse_deferred(const MapFrame &F) {
  const Counters *c = F.cnt;
  if ((c->error & ERR_FRAME_FAILED) || c->cnn_error) return true;
  const uint32_t leaves = (F.chain ? c->leaves_base : F.leaves_before) + c->pending;
  const uint32_t branches = min(c->branches_used, F.branches_max);
  const int n = (int)F.n;
  const bool outside = c->box_min[0] < 0 || c->box_min[1] < 0 || c->box_min[2] < 0 || c->box_max[0] >= n ||
                       c->box_max[1] >= n || c->box_max[2] >= n;
  return leaves < F.leaves_max && branches < F.branches_max && outside;
}

// Whether this part updates the brick at leaf position p (x, y, z, scale).
__device__ __forceinline__ bool owns_brick(const MapFrame &F, ushort4 p) {
  if (F.shards <= 1) return true;
  return shard_hash(p.x, p.y, p.z, (uint32_t)p.w * 8u, 0u, F.shift) % F.shards == F.shard;
}

// One frame of a deferred update: what the voxel update of that frame reads.
struct FuseSlot {
  CamF q;                // voxel grid -> camera, as of the frame
  const uint16_t *depth;
  const uint8_t *bgr;
  const float *conf;     // learned confidence, or null
  int W, H;
  float scaling, maxcam;
};

constexpr int FUSE_SLOTS_MAX = 32;      // frames one deferred pass takes (bits of upd_mask)
constexpr int FUSE_SLOTS_DEFAULT = 16;

// A deferred update pass over one map: every brick of list[0, *count) with
// the frames of its mask bits, in order (a kernel parameter).
struct FuseBatch {
  const ushort4 *leaf;
  float *sdf, *wgt;
  __half *sdf16, *wgt16;
  uint16_t *col;
  uint32_t *mask;
  const uint32_t *list, *count;
  unsigned long long *total;  // bricks of all passes so far (device counter)
  const uint32_t *rcp_tab;
  int rcp_shift;
  float scale, thr;
  int nslots;
  FuseSlot s[FUSE_SLOTS_MAX];
};

// Launch the deferred update pass (grid: blocks of 512 threads).
void launch_fuse_multi(const FuseBatch &fb, int storage, bool rcp_host, int grid, cudaStream_t s);

// Loop closure: one fused frame removed into the loop arrays
// (update8AddLoopSSESingleDeleteloop, loopclosure.cpp:15-228).
struct LoopFrame {
  CamF q;                      // voxel grid -> camera of the frame
  const float *depth;          // metres, NaN = no depth
  const uint8_t *red, *green, *blue;
  int W, H;
  const uint32_t *queue;       // the frame's queued leaves
  const uint32_t *slots;       // their loop slots
  const uint32_t *taken;       // entries of the queue that have a slot
  const ushort4 *leaf;
  float *sdf, *wgt;            // loop arrays [slot][512]
  uint16_t *col;               // [slot][3][512]
  const uint32_t *rcp_tab;
  int rcp_shift;
  float scale, thr;
};
// st[0]: slots in use; st[1] (out): queue entries that got a slot.
void launch_loop_slots(const uint32_t *queue, uint32_t nq, uint32_t *map, uint32_t capacity, uint32_t *slots,
                       uint32_t *st, cudaStream_t s);
void launch_loop_delete(const LoopFrame &L, bool rcp_host, int grid, cudaStream_t s);

// Halo exchange of a sharded map (records: uint32 leaf index, 12 bytes of
// padding, SDF, weight and colour planes as the pool stores them).
size_t halo_record_bytes(bool fp16);
// list[0, *count) += the leaves [0, nleaves) whose stamp is after `since` and
// that this part owns (every leaf when shards <= 1)
void launch_halo_select(const ushort4 *leaf, const uint32_t *stamp, uint32_t nleaves, uint32_t since,
                        uint32_t shard, uint32_t shards, const int32_t shift[3], uint32_t *list, uint32_t *count,
                        cudaStream_t s);
void launch_halo_pack(const uint32_t *list, uint32_t n, const float *sdf, const float *wgt, const __half *sdf16,
                      const __half *wgt16, const uint16_t *col, void *out, bool fp16, int grid, cudaStream_t s);
void launch_halo_unpack(const void *in, uint64_t n, uint32_t leaves_max, float *sdf, float *wgt, __half *sdf16,
                        __half *wgt16, uint16_t *col, bool fp16, int grid, cudaStream_t s);

constexpr int BATCH_MAX = 32;

struct BatchDesc {
  int n;                          // maps in the batch
  int max_rounds;                 // de-duplication round limit (largest image)
  uint32_t tile_end[BATCH_MAX];   // inclusive prefix of each map's de-duplication tiles
  uint32_t pix_end[BATCH_MAX];    // inclusive prefix of each map's pixels, each padded to 32
  MapFrame f[BATCH_MAX];
};

// Bytes of a BatchDesc holding n maps (the tail past f[n-1] is not uploaded).
inline size_t batch_desc_bytes(int n) { return offsetof(BatchDesc, f) + sizeof(MapFrame) * (size_t)n; }

// The descriptor of one map's frame, passed by value to its de-duplication
// launch (which stores it for the frame's later kernels): the first
// batch_desc_bytes(1) bytes of a BatchDesc.
struct BatchDesc1 {
  int n;
  int max_rounds;
  uint32_t tile_end[BATCH_MAX];
  uint32_t pix_end[BATCH_MAX];
  MapFrame f[1];
};
static_assert(offsetof(BatchDesc1, f) == offsetof(BatchDesc, f) && sizeof(BatchDesc1) == offsetof(BatchDesc, f) +
                                                                                          sizeof(MapFrame),
              "one-map descriptor layout");
static_assert(sizeof(BatchDesc1) % 8 == 0 && alignof(BatchDesc1) >= 8, "copied in 8-byte words");

// A leaf claimed during the frame's traversal, before its index is assigned.
struct PendingLeaf {
  uint32_t slot;         // tree entry that will hold the leaf index
  uint32_t first_pixel;  // smallest processed pixel index that queried it
  ushort4 pos;           // x, y, z, scale
};

// First-frame integer bounding box (geometryfusion_mipmap_cpu.cpp:1270-1303).
void launch_first_bbox(const uint16_t *depth, int W, int H, const CamF &p, float scaling, float maxcam, int bw,
                       Counters *cnt, cudaStream_t s);

// Tiles of the de-duplication for a W x H image with tiles `rows` high (and
// the tile grid); 16-row tiles unless the batch has more of them than warps
// can be resident, then 32-row tiles (dedupe_tile_rows).
int dedupe_tiles(int W, int H, int *tilesX, int *tilesY, int rows);
// Tiles one cooperative de-duplication launch holds (all warps resident).
cudaError_t dedupe_capacity(int device, int rows, uint32_t &tiles);
// int4 elements of the boundary buffer launch_dedupe needs for a W x H image.
size_t dedupe_boundary_elems(int W, int H);
// Per-pixel voxel coordinates, validity and target brick scale (written to
// each frame's vox), then the row/column de-duplication of brick keys
// (traversal_wrapper_functions.cpp:613-639, 688-690), for every frame of the
// batch in one cooperative launch per group of maps [m0, m1) whose `tiles`
// fit the launch.  barrier: 8 zeroed uint32 words per launch.
cudaError_t launch_dedupe(const BatchDesc *d_batch, int m0, int m1, uint32_t tiles, int rows, uint32_t *barrier,
                          int device, cudaStream_t s);
// The same for a one-map descriptor h_desc in host memory: passed as the
// launch's parameter (no upload of its own) and stored to d_batch by the
// launch for the frame's later kernels.
cudaError_t launch_dedupe_one(const BatchDesc *h_desc, BatchDesc *d_batch, uint32_t tiles, int rows,
                              uint32_t *barrier, int device, cudaStream_t s);

// Octree descent / allocation of every processed pixel of the batch's maps
// [m0, m1) (pixels [pix_end[m0 - 1], pix_end[m1 - 1]), pix = their count).
// pdl: launched as a programmatic dependent of the stream's previous kernel
// (which must be a kernel), as in the chained frames of a sequence.
void launch_insert(const BatchDesc *d_batch, uint32_t pix, cudaStream_t s, int block = 256, int m0 = 0,
                   int m1 = BATCH_MAX, bool pdl = false);

// Sort scratch size for `n` pending leaves.
size_t pending_sort_bytes(int n);
// Order pending leaves by first pixel: order[k] = record of the k-th (keys
// and keys_sorted: npend 64-bit words each of scratch).
cudaError_t sort_pending(const PendingLeaf *pend, int npend, uint64_t *keys, uint64_t *keys_sorted, uint32_t *order,
                         void *tmp, size_t tmp_bytes, int end_bit, cudaStream_t s);

// Assign leaf indices in creation order, fill the leaf table, queue new leaves.
void launch_finalize(const PendingLeaf *pend, const uint32_t *order, int npend, uint32_t leaves_before,
                     uint32_t leaves_max, uint32_t *tree, ushort4 *leaf, uint32_t frame, uint32_t *stamp,
                     uint32_t *queue, Counters *cnt, cudaStream_t s);
// Parents of the leaves placed by the one-block finalisation of frames
// [m0, m0 + nframes) of the descriptor (after it on the stream).
void launch_parents_frames(const BatchDesc *d_batch, int nframes, cudaStream_t s, int m0 = 0, bool pdl = false);
// Parent leaf of each new leaf: finest ancestor leaf created before it.
void launch_parents(int npend, uint32_t leaves_before, uint32_t leaves_max, const uint32_t *tree, uint32_t n,
                    const ushort4 *leaf, uint32_t *parent, cudaStream_t s);

// Whether launch_finalize_small takes a W x H frame.
bool finalize_small_fits(uint32_t npix);

// Ranks (creation order), leaf table and parents of each map's pending
// leaves, one block per map, counts read on the device; for images of up to
// about 1.6 million pixels (false, nothing launched, for larger ones).
bool launch_finalize_small(const BatchDesc *d_batch, int nmaps, uint32_t max_npix, int device, cudaStream_t s,
                           int m0 = 0, bool pdl = false);
// Set the finalisation kernel's shared-memory limit on this device (once).
bool finalize_small_prepare(int device);

// Load the kernels of each file ahead of their first launch.
cudaError_t prewarm_alloc_kernels();
cudaError_t prewarm_fuse_kernels();
cudaError_t prewarm_mesh_kernels();

// grow(): move child-branch pointers by `shift`, leaf positions by `add`.
void launch_shift_branches(uint32_t *tree, uint32_t used, uint32_t shift, cudaStream_t s);
void launch_shift_leaves(ushort4 *leaf, uint32_t n_leaves, ushort3 add, cudaStream_t s);
void launch_fill(uint32_t *p, size_t n, uint32_t v, cudaStream_t s);

// Voxel update of the queued bricks of every frame of the batch
// (update_functions.cpp:1187-1444).  gated: each map's brick count is read
// on the device (its queue after the new leaves) and a map whose volume must
// grow first is left for the host; otherwise MapFrame::nq_host is used.
// shape: block shape of the update, 0..FUSE_SHAPE_COUNT-1 (bricks per block
// and the blocks per SM its registers are budgeted for; 0 = 1 brick, 4).
constexpr int FUSE_SHAPE_COUNT = 4;
void launch_fuse(const BatchDesc *d_batch, int nmaps, bool gated, int storage, bool rcp_host, int grid,
                 cudaStream_t s, int shape = 0);
int fuse_shape_bricks(int shape);

// Table of the host CPU's RCPPS over the mantissas of [1,2), indexed by the
// mantissa >> shift (the low bits the instruction ignores are dropped); false
// when the host is not x86-64 or the instruction does not follow the
// expected rules.
bool build_rcp_table(std::vector<uint32_t> &tab, int &shift);

// ---- learned confidence weight (ff_cnn.cu) ----

constexpr int CNN_PARAMS = 8833;   // W1[16][5][25] b1[16] W2[16][16][25] b2[16] W3[1][16][25] b3[1]
constexpr int CNN_FEAT_CH = 8;     // channels per pixel of the feature map (5 used)
constexpr int CNN_HIDDEN = 16;

// The fused volume as the raycaster reads it.
struct RaycastMap {
  const uint32_t *tree;
  const ushort4 *leaf;
  const float *sdf, *wgt;
  const __half *sdf16, *wgt16;
  uint32_t n, leaves_max;
  int fp16;
  float thr;  // truncation distance (m) of scale-1 bricks
};

cudaError_t cnn_features(const uint16_t *depth, int n, int W, int H, float scaling, const float K[4],
                         __nv_bfloat16 *feat, cudaStream_t s);
// tau_cm > 0: out = the confidence weight; else out = the network's output.
// packed: CNN_PACKED_BYTES of device memory for the tensor-core operands of
// the weights, filled from params first unless packed_ready.
// err (may be null): ERR_SPIN_TIMEOUT if a tensor-core wait gave up (the
// layer's output is then NaN).
constexpr int CNN_PACKED_BYTES = 65 * 512;
cudaError_t cnn_forward(const __nv_bfloat16 *params, uint8_t *packed, bool packed_ready, const __nv_bfloat16 *feat,
                        int n, int W, int H, __nv_bfloat16 *a1, __nv_bfloat16 *a2, float *out, float tau_cm,
                        uint32_t *err, cudaStream_t s);
cudaError_t cnn_backward(const __nv_bfloat16 *params, const __nv_bfloat16 *feat, const __nv_bfloat16 *a1,
                         const __nv_bfloat16 *a2, const float *dpred, int n, int W, int H, float *g1, float *g2,
                         float *grads, cudaStream_t s);
cudaError_t cnn_mse(const float *pred, const float *target, int64_t count, float inv_count, float *dpred,
                    double *loss, cudaStream_t s);
cudaError_t cnn_adam(float *master, __nv_bfloat16 *params, float *grads, float *m, float *v, int n, float lr,
                     float b1, float b2, float eps, int step, cudaStream_t s);
cudaError_t launch_raycast(const RaycastMap &m, const CamF &p, int W, int H, const uint16_t *depth, float scaling,
                           float window, float step, float *out, cudaStream_t s);

}  // namespace ffb
