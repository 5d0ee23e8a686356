// C ABI of the B200 fusion path (include/fastfusion_b200.h): host-side
// orchestration of one map (the reference's FusionMipMapCPU).
//
// Per frame (ff_add_map_u16): camera parameters in FP64 rounded once to FP32
// like the reference's camPamsFloat; on the first frame the integer bounding
// box sizes the volume; then project -> de-duplicate -> insert on the device,
// one read-back of the counters, leaf-index assignment, grow() when the
// frame's points left the volume, and the voxel update of every queued brick.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fastfusion_b200.h"
#include "ff_kernels.h"
#include "ff_mesh.h"
#include "ff_prof.h"

namespace ffb {
std::atomic<unsigned long long> g_own_launches{0}, g_lib_calls{0};
}

using namespace ffb;

// grid-barrier words: 8 per de-duplication launch of a batch
constexpr int BARRIER_WORDS = 8 * BATCH_MAX;

struct ff_handle {
  ff_config cfg;
  std::string err;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // host-input frames: the colour image is copied on a second stream while
  // the allocation kernels run (it is first read by the voxel update)
  cudaStream_t copy_stream = nullptr;
  // ff_get_mesh_async: the mesh's device-to-host copies, after ev_mesh_ready;
  // the last two copies and the device buffers they read (the mesher writes
  // its two output buffers in turn, so an update waits only for the copy of
  // the mesh two updates back)
  cudaStream_t mesh_stream = nullptr;
  cudaEvent_t ev_mesh_ready = nullptr;
  struct MeshCopy {
    const void *src[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev = nullptr;
    bool pending = false;
  } mesh_copy[2];
  int mesh_copy_next = 0;
  // ff_add_map_sequence_u16: the frames' images staged on the device (up to
  // BATCH_MAX frames), and the colour copies the next update pass waits for
  uint16_t *d_hseq_depth = nullptr;
  uint8_t *d_hseq_bgr = nullptr;
  size_t hseq_frames = 0, hseq_pix = 0;
  cudaEvent_t ev_host_depth = nullptr, ev_host_images = nullptr;
  bool host_images_pending = false;
  cudaEvent_t ev_bgr_free = nullptr, ev_bgr_ready = nullptr;
  // recorded once a frame's counters have reached the host: a single-map
  // frame returns then, while its voxel update still runs
  cudaEvent_t ev_counters = nullptr;
  // A single-map frame's voxel update runs on fuse_stream, overlapping the
  // next frame's allocation kernels on the map's stream.  The buffers the
  // update reads (descriptor, counters, queue, host-input images, confidence
  // map) come in two sets used by alternate frames; a set is reused only
  // after the update that read it (ev_fuse[set]) has finished.
  // The leaf finalisation runs there too, ahead of the update, so that the
  // next frame's de-duplication (which reads no octree) overlaps it; the
  // next frame's insert waits for it (ev_fin, fin_pending).
  cudaStream_t fuse_stream = nullptr;
  cudaEvent_t ev_alloc = nullptr;  // the frame's insert done (map stream)
  cudaEvent_t ev_cnn_in = nullptr, ev_cnn_done = nullptr;  // the confidence network on fuse_stream
  bool cnn_on_side = false;  // a sequence's frames: their networks on fuse_stream, beside the allocation chain
  bool cnn_pending = false;
  cudaEvent_t ev_fin = nullptr;    // the frame's finalisation done (fuse_stream)
  bool fin_pending = false;
  cudaEvent_t ev_fuse[2] = {nullptr, nullptr};
  int last_fuse = -1;  // set of the last update launched on fuse_stream
  int set = 0;
  BatchDesc *d_batch_set[2] = {nullptr, nullptr}, *h_batch_set[2] = {nullptr, nullptr};
  Counters *d_cnt_set[2] = {nullptr, nullptr}, *h_cnt_set[2] = {nullptr, nullptr};
  uint32_t *d_queue_set[2] = {nullptr, nullptr};
  uint16_t *d_depth_set[2] = {nullptr, nullptr};
  uint8_t *d_bgr_set[2] = {nullptr, nullptr};
  float *d_conf_set[2] = {nullptr, nullptr};
  // the frame descriptor(s) the per-frame kernels read: this map's own, or a
  // whole batch when this handle leads ff_add_maps_u16_device
  BatchDesc *d_batch = nullptr, *h_batch = nullptr;

  // map state on the device
  uint32_t *d_tree = nullptr;
  ushort4 *d_leaf = nullptr;
  uint32_t *d_parent = nullptr;
  float *d_sdf = nullptr, *d_wgt = nullptr;
  __half *d_sdf16 = nullptr, *d_wgt16 = nullptr;
  uint16_t *d_col = nullptr;
  uint32_t *d_stamp = nullptr;
  uint32_t *d_bstamp = nullptr;  // per branch: last frame that created something at or below it
  uint32_t *d_queue = nullptr;
  uint32_t *d_queue_last = nullptr;  // the queue the last finished frame wrote (ff_get_queue)
  Counters *d_cnt = nullptr;
  Counters *h_cnt = nullptr;  // pinned
  uint32_t *d_barrier = nullptr;
  // the de-duplication barrier words need clearing before the next launch
  // (fresh memory, or a launch that ended without convergence)
  bool barrier_dirty = true;
  uint32_t *d_rcp_tab = nullptr;  // FF_RCP_HOST: the host CPU's RCPPS per mantissa >> rcp_shift
  int rcp_shift = 0;

  // per-image scratch
  int img_w = 0, img_h = 0, cap_pix = 0;
  uint16_t *d_depth = nullptr;
  uint8_t *d_bgr = nullptr;
  float *d_pxp = nullptr, *d_pyp = nullptr;
  int4 *d_vox = nullptr;
  uint8_t *d_proc = nullptr;
  int4 *d_bnd = nullptr;
  size_t bnd_elems = 0;
  PendingLeaf *d_pend = nullptr;
  // 6 x cap_pix words: pending-leaf sort keys (u64), sorted keys (u64), order; finalisation ranks
  uint32_t *d_keys = nullptr;
  void *d_sort_tmp = nullptr;
  size_t sort_tmp_bytes = 0;

  // host mirror of the scalar state
  uint32_t n = 0;
  float offset[3] = {0, 0, 0};
  uint32_t leaves_used = 0, branches_used = 16;
  uint32_t frames = 0, queued = 0, grows = 0, processed = 0, new_leaves = 0, dedupe_rounds = 0;
  bool meshing_ok = true;
  uint16_t bandwidth = 0;

  // learned confidence weight (ff_set_confidence): BF16 parameters, and the
  // per-frame features, activations and confidence map
  __nv_bfloat16 *d_cnn_params = nullptr;
  uint8_t *d_cnn_packed = nullptr;  // the weights as tensor-core operands
  bool cnn_packed_ready = false;
  float conf_tau_cm = 0.0f;  // > 0: the learned weight is on
  __nv_bfloat16 *d_feat = nullptr, *d_a1 = nullptr, *d_a2 = nullptr;
  float *d_conf = nullptr;
  size_t conf_cap = 0;  // pixels the buffers hold
  int conf_w = 0, conf_h = 0;  // size of the last confidence map

  // iterations after which a device-side wait gives up (ff_set_spin_limit),
  // and a failure the next frame reports as if a device wait had given up
  // (ff_inject_error)
  uint32_t spin_limit = SPIN_LIMIT;
  int full_cells = 0;  // 1: regenerate every mesh cell at every update (ff_set_cell_generation)
  bool top_changed = true;  // a frame since the last mesh update created a branch or leaf near the root
  int inject = 0;
  // loop closure (ff_loop_begin): the loop arrays, each leaf's slot in them,
  // per queue entry its slot, [slots in use, entries taken]
  uint32_t loop_cap = 0;
  uint32_t *d_loop_map = nullptr, *d_loop_slots = nullptr, *d_loop_st = nullptr, *h_loop_st = nullptr;
  size_t loop_slots_cap = 0;
  float *d_loop_sdf = nullptr, *d_loop_wgt = nullptr;
  uint16_t *d_loop_col = nullptr;
  uint32_t halo_since = 0;           // frames whose changes the last halo export covered
  uint32_t *h_halo_count = nullptr;  // pinned: the export's record count

  // Deferred voxel update: a single-map frame's update waits for one pass
  // (k_fuse_multi) over the union of the bricks of up to upd_batch frames,
  // run when the batch is full, before a growth of the volume, and before
  // anything reads or replaces voxel state (updateMeshes, accessors, ff_sync).
  // The waiting frames' images and confidence maps are kept in a ring of
  // slots; a slot is written again only after the pass that read it.
  int upd_batch = FUSE_SLOTS_DEFAULT;  // frames a pass takes (ff_set_update_batch)
  int upd_pending = 0;                 // frames waiting for the pass
  int cur_slot = -1;                   // the slot of the frame being added (-1: not deferred)
  FuseSlot upd_slot[FUSE_SLOTS_MAX];
  double pass_frame_bricks = 0;        // queued bricks of the waiting frames
  uint32_t *d_upd_mask = nullptr, *d_upd_list = nullptr, *d_upd_count = nullptr;
  unsigned long long *d_upd_total = nullptr, *h_upd_total = nullptr;  // bricks of all passes
  uint64_t fused_frame_bricks = 0, direct_bricks = 0;
  uint16_t *d_ring_depth = nullptr;
  uint8_t *d_ring_bgr = nullptr;
  float *d_ring_conf = nullptr;
  size_t ring_pix = 0, ring_conf_pix = 0;
  int ring_slots = 0;
  cudaEvent_t ev_ring_free = nullptr;  // the last pass has read the ring
  bool ring_read = false;              // a pass was launched since the ring was allocated
  cudaEvent_t ev_copy = nullptr;       // a device frame's images copied into its slot
  bool copy_pending = false;
  bool seq_images = false;             // the frames being finished are a sequence's (caller images)

  // a sequence of one map's frames (ff_add_map_sequence_u16_device): per
  // frame its voxel keys, processed flags, de-duplication boundaries and
  // counters (device, and a pinned mirror)
  int seq_frames = 0;
  size_t seq_pix = 0, seq_bnd = 0;
  int4 *d_seq_vox = nullptr;
  uint8_t *d_seq_proc = nullptr;
  int4 *d_seq_bnd = nullptr;
  Counters *d_seq_cnt = nullptr, *h_seq_cnt = nullptr;
  int pi_insert = -1;  // profile record of the last insert launch this map led

  // brick ownership (ff_set_shard) and the voxels grow() has moved the grid by
  uint32_t shard = 0, shards = 1;
  int32_t shift[3] = {0, 0, 0};

  // launch shapes (ff_set_tuning) and the device's SM count
  ff_tuning tune = {0, 0, 0, 0, 0};
  int sm_count = 148;
  // batched calls led by this map: their launches as a CUDA graph, replayed
  // while the signature (maps, image sizes, shapes) stays the same
  cudaGraphExec_t graph_exec = nullptr;
  std::vector<uint64_t> graph_key;
  uint64_t graph_launches = 0;  // own kernel launches inside the graph
  uint32_t graph_replays = 0;
  bool graph_failed = false;

  MeshState mesh;
  Prof prof;
};

static thread_local std::string g_create_error;

#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      h->err = std::string(#call) + ": " + cudaGetErrorString(e_);                    \
      return FF_ERR_CUDA;                                                             \
    }                                                                                 \
  } while (0)

// Return a failed ff_status (its message already set).
#define FCK(call)                  \
  do {                             \
    const ff_status s_ = (call);   \
    if (s_ != FF_OK) return s_;    \
  } while (0)

static ff_status set_err(ff_handle *h, ff_status s, const std::string &m) {
  if (h) h->err = m;
  return s;
}

// Make the per-frame buffers of set k current.
static void select_set(ff_handle *h, int k) {
  h->set = k;
  h->d_batch = h->d_batch_set[k];
  h->h_batch = h->h_batch_set[k];
  h->d_cnt = h->d_cnt_set[k];
  h->h_cnt = h->h_cnt_set[k];
  h->d_queue = h->d_queue_set[k];
  h->d_depth = h->d_depth_set[k];
  h->d_bgr = h->d_bgr_set[k];
  h->d_conf = h->d_conf_set[k];
}

// Wait for an event the next few microseconds will bring (a frame's counter
// copy): poll it first, which wakes sooner than a blocking wait, then block.
static cudaError_t wait_event_polling(cudaEvent_t ev) {
  for (int k = 0; k < 20000; k++) {
    const cudaError_t e = cudaEventQuery(ev);
    if (e != cudaErrorNotReady) return e;
  }
  return cudaEventSynchronize(ev);
}

// Order the map's stream after every voxel update launched on fuse_stream.
static cudaError_t join_fuse(ff_handle *h) {
  return h->last_fuse >= 0 ? cudaStreamWaitEvent(h->stream, h->ev_fuse[h->last_fuse], 0) : cudaSuccess;
}

// Run the deferred update of the waiting frames: one pass over the union of
// their bricks on fuse_stream (ordered after their finalisations there);
// the map's later work and every accessor order after it through ev_fuse.
static ff_status flush_updates(ff_handle *h) {
  if (!h->upd_pending) return FF_OK;
  FuseBatch fb;
  memset(&fb, 0, sizeof(fb));
  fb.leaf = h->d_leaf;
  fb.sdf = h->d_sdf;
  fb.wgt = h->d_wgt;
  fb.sdf16 = h->d_sdf16;
  fb.wgt16 = h->d_wgt16;
  fb.col = h->d_col;
  fb.mask = h->d_upd_mask;
  fb.list = h->d_upd_list;
  fb.count = h->d_upd_count;
  fb.total = h->d_upd_total;
  fb.rcp_tab = h->d_rcp_tab;
  fb.rcp_shift = h->rcp_shift;
  fb.scale = h->cfg.scale;
  fb.thr = h->cfg.threshold;
  fb.nslots = h->upd_pending;
  for (int j = 0; j < h->upd_pending; j++) fb.s[j] = h->upd_slot[j];
  cudaStream_t fs = h->fuse_stream;
  if (h->host_images_pending) {
    // the colour images of a host-image sequence, copied on the copy stream
    CK(cudaStreamWaitEvent(fs, h->ev_host_images, 0));
    h->host_images_pending = false;
  }
  const int pi = h->prof.begin(ST_FUSE, fs);
  launch_fuse_multi(fb, h->cfg.storage, h->d_rcp_tab != nullptr, h->sm_count * 2, fs);
  // every queued brick of every frame read and written once per frame in
  // the reference: the pass's algorithmic bytes
  const double brick_bytes = 512.0 * 2 * ((h->cfg.storage == FF_STORAGE_FP16 ? 4 : 8) + 6);
  h->prof.end(pi, h->pass_frame_bricks * brick_bytes, fs);
  CK(cudaGetLastError());
  CK(cudaMemsetAsync(h->d_upd_count, 0, sizeof(uint32_t), fs));
  CK(cudaMemcpyAsync(h->h_upd_total, h->d_upd_total, sizeof(unsigned long long), cudaMemcpyDeviceToHost, fs));
  CK(cudaEventRecord(h->ev_ring_free, fs));
  const int k = h->last_fuse >= 0 ? h->last_fuse : h->set;
  CK(cudaEventRecord(h->ev_fuse[k], fs));
  h->last_fuse = k;
  h->upd_pending = 0;
  h->pass_frame_bricks = 0;
  h->ring_read = true;
  return FF_OK;
}

// The waiting frames updated, and the map's stream ordered after every
// update: before anything reads or replaces voxel state.
static ff_status settle(ff_handle *h) {
  ff_status st = flush_updates(h);
  if (st != FF_OK) return st;
  CK(join_fuse(h));
  return FF_OK;
}

// ----------------------------------------------------------- camera math --

// p: world -> voxel grid (reference geometryfusion_mipmap_cpu.cpp:1617-1625)
static CamF cam_world_to_grid(const ff_handle *h, const double *K, const double *R, const double *t) {
  CamF p;
  for (int i = 0; i < 9; i++) p.r[i] = (float)(R[i] / (double)h->cfg.scale);
  for (int i = 0; i < 3; i++) p.t[i] = (float)((t[i] - (double)h->offset[i]) / (double)h->cfg.scale);
  p.fx = (float)K[0];
  p.fy = (float)K[1];
  p.cx = (float)K[2];
  p.cy = (float)K[3];
  return p;
}

// pInv: voxel grid (offset folded in) -> camera, from the extrinsic inverse
// [R^T | -R^T t] (geometryfusion_mipmap_cpu.cpp:1771-1793, camerautils.cpp:153-161);
// FP64 throughout, one rounding to FP32 per parameter.
static CamF cam_grid_to_camera(const ff_handle *h, const double *K, const double *R, const double *t) {
  CamF q;
  double r2[9], t2[3];
  for (int r = 0; r < 3; r++) {
    for (int c = 0; c < 3; c++) r2[r * 3 + c] = R[c * 3 + r];
    double s = R[0 * 3 + r] * t[0] + R[1 * 3 + r] * t[1];
    s = s + R[2 * 3 + r] * t[2];
    t2[r] = -s;
  }
  for (int i = 0; i < 9; i++) q.r[i] = (float)r2[i];
  for (int r = 0; r < 3; r++) {
    double v = r2[r * 3 + 0] * (double)h->offset[0] + r2[r * 3 + 1] * (double)h->offset[1];
    v = v + r2[r * 3 + 2] * (double)h->offset[2];
    v = v + t2[r];
    q.t[r] = (float)v;
  }
  q.fx = (float)K[0];
  q.fy = (float)K[1];
  q.cx = (float)K[2];
  q.cy = (float)K[3];
  return q;
}

// setInitialVolume (geometryfusion_mipmap_cpu.cpp:1186-1233)
static bool set_initial_volume(ff_handle *h, const int *mn, const int *mx) {
  if (mn[0] >= mx[0] || mn[1] >= mx[1] || mn[2] >= mx[2]) return false;
  uint16_t hi[3];
  for (int r = 0; r < 3; r++) hi[r] = (uint16_t)(mx[r] - mn[r]);
  uint16_t high = std::max(std::max(hi[0], hi[1]), hi[2]);
  uint16_t n;
  for (n = 2 * BL; n <= high; n = (uint16_t)(n * 2)) {
  }
  h->n = n;
  for (int r = 0; r < 3; r++) h->offset[r] = (float)(mn[r] - ((int)n - (int)hi[r]) / 2) * h->cfg.scale;
  return true;
}

static uint16_t highest_pow2(uint16_t in) {
  uint16_t r = 1;
  while (r * 2 <= in) r = (uint16_t)(r * 2);
  return r;
}

// grow() (geometryfusion_mipmap_cpu.cpp:3071-3319): add levels above the
// root so that the frame's bounding box fits; the old tree becomes a child.
static ff_status grow(ff_handle *h, const int *box_min, const int *box_max) {
  int n = h->n;
  uint16_t pl_[3], mi_[3];
  for (int r = 0; r < 3; r++) {
    pl_[r] = (uint16_t)((box_max[r] >= n) * ((box_max[r] - n) / n + 1));
    mi_[r] = (uint16_t)((box_min[r] < 0) * ((-box_min[r]) / n + 1));
  }
  for (int r = 0; r < 3; r++) {
    uint16_t cut = pl_[r] & mi_[r];
    if (cut) {
      if (mi_[r] > pl_[r])
        mi_[r] = (uint16_t)(2 * highest_pow2(mi_[r]) + (mi_[r] & (uint16_t)~cut));
      else
        pl_[r] = (uint16_t)(2 * highest_pow2(pl_[r]) + (pl_[r] & (uint16_t)~cut));
    }
  }
  uint16_t levels = highest_pow2(mi_[0]);
  for (int r = 0; r < 3; r++) {
    levels = std::max(levels, highest_pow2(pl_[r]));
    levels = std::max(levels, highest_pow2(mi_[r]));
  }
  uint32_t shift = (uint32_t)levels * 16;
  if (shift > h->cfg.branches_max - h->branches_used) return FF_OK;  // the reference's split() is a stub
  cudaStream_t s = h->stream;
  launch_shift_branches(h->d_tree, h->branches_used, shift, s);
  // move the tree up by `shift` entries (through the free tail of the array)
  uint32_t used = h->branches_used;
  if (used + shift + used <= h->cfg.branches_max) {
    CK(cudaMemcpyAsync(h->d_tree + used + shift, h->d_tree, sizeof(uint32_t) * used, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(h->d_tree + shift, h->d_tree + used + shift, sizeof(uint32_t) * used,
                       cudaMemcpyDeviceToDevice, s));
    launch_fill(h->d_tree + used + shift, used, BRANCHINIT, s);
  } else {
    uint32_t *tmp = nullptr;
    CK(cudaMallocAsync((void **)&tmp, sizeof(uint32_t) * used, s));
    CK(cudaMemcpyAsync(tmp, h->d_tree, sizeof(uint32_t) * used, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(h->d_tree + shift, tmp, sizeof(uint32_t) * used, cudaMemcpyDeviceToDevice, s));
    CK(cudaFreeAsync(tmp, s));
  }
  launch_fill(h->d_tree, shift, BRANCHINIT, s);
  h->branches_used += shift;
  uint16_t add[3] = {0, 0, 0};
  std::vector<std::pair<uint32_t, uint32_t>> links;
  uint32_t index = (uint32_t)(levels - 1) * 16;
  for (uint16_t level = 0; level < levels; level++) {
    unsigned dec = 1u << level;
    uint32_t co = 0;
    for (int r = 0; r < 3; r++) {
      if ((mi_[r] & dec) || (!(pl_[r] & dec) && (pl_[r] > mi_[r]))) {
        add[r] = (uint16_t)(add[r] + h->n);
        co += 1u << r;
      }
    }
    links.push_back({index + co + 8, index + 16});
    h->n = (uint16_t)(h->n * 2);
    index -= 16;
  }
  for (auto &l : links) CK(cudaMemcpyAsync(h->d_tree + l.first, &l.second, 4, cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));  // `links` lives on this stack frame
  for (int r = 0; r < 3; r++) {
    h->offset[r] -= (float)add[r] * h->cfg.scale;
    h->shift[r] += (int32_t)add[r];
  }
  uint32_t nl = std::min(h->leaves_used, h->cfg.leaves_max);
  launch_shift_leaves(h->d_leaf, nl, make_ushort3(add[0], add[1], add[2]), s);
  h->grows++;
  return FF_OK;
}

// ------------------------------------------------------------- buffers ----

template <typename T>
static cudaError_t alloc(T **p, size_t count) {
  return cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(count, 1));
}

static ff_status ensure_image(ff_handle *h, int W, int H) {
  int npix = W * H;
  if (npix > h->cap_pix) {
    for (int k = 0; k < 2; k++) {
      cudaFree(h->d_depth_set[k]);
      cudaFree(h->d_bgr_set[k]);
      h->d_depth_set[k] = nullptr;
      h->d_bgr_set[k] = nullptr;
    }
    cudaFree(h->d_vox);
    cudaFree(h->d_proc);
    cudaFree(h->d_pend);
    cudaFree(h->d_keys);
    cudaFree(h->d_sort_tmp);
    for (int k = 0; k < 2; k++) {
      CK(alloc(&h->d_depth_set[k], npix));
      CK(alloc(&h->d_bgr_set[k], (size_t)npix * 3));
    }
    select_set(h, h->set);
    CK(alloc(&h->d_vox, npix));
    CK(alloc(&h->d_proc, npix));
    CK(alloc(&h->d_pend, npix));
    CK(alloc(&h->d_keys, (size_t)npix * 6));
    h->sort_tmp_bytes = pending_sort_bytes(npix);
    CK(cudaMalloc(&h->d_sort_tmp, std::max<size_t>(h->sort_tmp_bytes, 16)));
    h->cap_pix = npix;
  }
  const size_t bnd_need = dedupe_boundary_elems(W, H);
  if (bnd_need > h->bnd_elems) {
    cudaFree(h->d_bnd);
    h->bnd_elems = bnd_need;
    CK(alloc(&h->d_bnd, h->bnd_elems));
  }
  return FF_OK;
}

// The ring of image slots for `slots` waiting frames of W x H pixels (and
// their confidence maps when the learned weight is on); a reallocation first
// runs the waiting frames' pass.
static ff_status ensure_ring(ff_handle *h, int W, int H) {
  const size_t npix = (size_t)W * H;
  const bool need_conf = h->conf_tau_cm > 0.0f;
  if (npix <= h->ring_pix && h->ring_slots >= h->upd_batch && (!need_conf || npix <= h->ring_conf_pix))
    return FF_OK;
  ff_status st = settle(h);
  if (st != FF_OK) return st;
  CK(cudaStreamSynchronize(h->fuse_stream));
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaStreamSynchronize(h->copy_stream));
  const int slots = std::max(h->upd_batch, h->ring_slots);
  const size_t pix = std::max(npix, h->ring_pix);
  if (pix > h->ring_pix || slots > h->ring_slots) {
    cudaFree(h->d_ring_depth);
    cudaFree(h->d_ring_bgr);
    h->d_ring_depth = nullptr;
    h->d_ring_bgr = nullptr;
    h->ring_pix = 0;
    CK(alloc(&h->d_ring_depth, pix * slots));
    CK(alloc(&h->d_ring_bgr, pix * 3 * slots));
    if (h->d_ring_conf) {
      cudaFree(h->d_ring_conf);
      h->d_ring_conf = nullptr;
      h->ring_conf_pix = 0;
    }
    h->ring_pix = pix;
    h->ring_slots = slots;
  }
  if (need_conf && h->ring_conf_pix < h->ring_pix) {
    cudaFree(h->d_ring_conf);
    h->d_ring_conf = nullptr;
    CK(alloc(&h->d_ring_conf, h->ring_pix * h->ring_slots));
    h->ring_conf_pix = h->ring_pix;
  }
  h->ring_read = false;
  return FF_OK;
}

// ------------------------------------------------------------------ API ---

extern "C" {

const char *ff_version(void) { return "fastfusion_b200 0.1 (sm_100a)"; }

const char *ff_last_error(const ff_handle *h) { return h ? h->err.c_str() : g_create_error.c_str(); }

ff_status ff_create(const ff_config *cfg, ff_handle **out) {
  if (!cfg || !out) {
    g_create_error = "ff_create: NULL argument";
    return FF_ERR_BAD_ARG;
  }
  *out = nullptr;
  if (!(cfg->scale > 0.0f) || !(cfg->threshold > 0.0f)) {
    g_create_error = "ff_create: scale and threshold must be > 0";
    return FF_ERR_BAD_ARG;
  }
  if (cfg->rcp_mode != FF_RCP_HOST && cfg->rcp_mode != FF_RCP_EXACT) {
    g_create_error = "ff_create: unknown rcp_mode";
    return FF_ERR_BAD_ARG;
  }
  if (cfg->storage != FF_STORAGE_FP32 && cfg->storage != FF_STORAGE_FP16) {
    g_create_error = "ff_create: unknown storage";
    return FF_ERR_BAD_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    cudaGetLastError();
    g_create_error = "ff_create: no CUDA device";
    return FF_ERR_NO_DEVICE;
  }
  if (cfg->device < 0 || cfg->device >= ndev) {
    g_create_error = "ff_create: bad device ordinal";
    return FF_ERR_BAD_ARG;
  }
  ff_handle *h = new ff_handle();
  h->cfg = *cfg;
  if (cudaSetDevice(cfg->device) != cudaSuccess) {
    g_create_error = "ff_create: cudaSetDevice failed";
    delete h;
    return FF_ERR_CUDA;
  }
  size_t brick_bytes = 512 * (cfg->storage == FF_STORAGE_FP16 ? 4 : 8) + 512 * 6;
  if (h->cfg.leaves_max == 0) {
    uint64_t pool = cfg->pool_bytes ? cfg->pool_bytes : 2000000000ull;
    h->cfg.leaves_max = (uint32_t)std::min<uint64_t>(pool / (brick_bytes + 24), 0x3FFFFFFFull);
  }
  if (h->cfg.branches_max == 0)
    h->cfg.branches_max = (uint32_t)std::min<uint64_t>((uint64_t)h->cfg.leaves_max * 4 + (1u << 20), 0xBFFFFFF0ull);
  h->cfg.branches_max &= ~15u;
  // _bandwidth(_distanceThreshold / _scale * BANDWIDTHFACTOR)
  h->bandwidth = (uint16_t)(double)(cfg->threshold / cfg->scale * 1.0);
  ff_status st = FF_OK;
  auto fail = [&](ff_status s, const char *m) {
    g_create_error = std::string("ff_create: ") + m + ": " + cudaGetErrorString(cudaGetLastError());
    st = s;
  };
  do {
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) { fail(FF_ERR_CUDA, "stream"); break; }
    if (cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, h->cfg.device) != cudaSuccess ||
        h->sm_count < 1)
      h->sm_count = 148;
    h->own_stream = true;
    if (cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_bgr_free, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_bgr_ready, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_counters, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->mesh_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_mesh_ready, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->mesh_copy[0].ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->mesh_copy[1].ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_host_images, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_host_depth, cudaEventDisableTiming) != cudaSuccess) {
      fail(FF_ERR_CUDA, "copy stream");
      break;
    }
    size_t L = h->cfg.leaves_max;
    if (alloc(&h->d_tree, h->cfg.branches_max) != cudaSuccess) { fail(FF_ERR_OOM_POOL, "tree"); break; }
    if (alloc(&h->d_leaf, L) != cudaSuccess || alloc(&h->d_parent, L) != cudaSuccess ||
        alloc(&h->d_stamp, L) != cudaSuccess || alloc(&h->d_queue_set[0], L) != cudaSuccess ||
        alloc(&h->d_queue_set[1], L) != cudaSuccess ||
        alloc(&h->d_bstamp, (size_t)h->cfg.branches_max / 16 + 1) != cudaSuccess) {
      fail(FF_ERR_OOM_POOL, "leaf table");
      break;
    }
    if (cfg->storage == FF_STORAGE_FP16) {
      if (alloc(&h->d_sdf16, L * 512) != cudaSuccess || alloc(&h->d_wgt16, L * 512) != cudaSuccess) {
        fail(FF_ERR_OOM_POOL, "brick pool");
        break;
      }
    } else {
      if (alloc(&h->d_sdf, L * 512) != cudaSuccess || alloc(&h->d_wgt, L * 512) != cudaSuccess) {
        fail(FF_ERR_OOM_POOL, "brick pool");
        break;
      }
    }
    if (alloc(&h->d_col, L * 1536) != cudaSuccess) { fail(FF_ERR_OOM_POOL, "colour pool"); break; }
    if (alloc(&h->d_cnt_set[0], 1) != cudaSuccess || alloc(&h->d_cnt_set[1], 1) != cudaSuccess ||
        alloc(&h->d_barrier, BARRIER_WORDS) != cudaSuccess) { fail(FF_ERR_CUDA, "counters"); break; }
    // (frames set their counters up on the device; the network's error word is kept)
    if (cudaMemset(h->d_cnt_set[0], 0, sizeof(Counters)) != cudaSuccess ||
        cudaMemset(h->d_cnt_set[1], 0, sizeof(Counters)) != cudaSuccess) { fail(FF_ERR_CUDA, "counters"); break; }
    if (cudaMallocHost((void **)&h->h_cnt_set[0], sizeof(Counters)) != cudaSuccess ||
        cudaMallocHost((void **)&h->h_cnt_set[1], sizeof(Counters)) != cudaSuccess) { fail(FF_ERR_CUDA, "pinned"); break; }
    if (cudaMalloc((void **)&h->d_batch_set[0], sizeof(BatchDesc)) != cudaSuccess ||
        cudaMalloc((void **)&h->d_batch_set[1], sizeof(BatchDesc)) != cudaSuccess ||
        cudaMallocHost((void **)&h->h_batch_set[0], sizeof(BatchDesc)) != cudaSuccess ||
        cudaMallocHost((void **)&h->h_batch_set[1], sizeof(BatchDesc)) != cudaSuccess) {
      fail(FF_ERR_CUDA, "frame descriptors");
      break;
    }
    if (cudaStreamCreateWithFlags(&h->fuse_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_fin, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_alloc, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_cnn_in, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_cnn_done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_fuse[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_fuse[1], cudaEventDisableTiming) != cudaSuccess) {
      fail(FF_ERR_CUDA, "update stream");
      break;
    }
    if (alloc(&h->d_upd_mask, L) != cudaSuccess || alloc(&h->d_upd_list, L) != cudaSuccess ||
        alloc(&h->d_upd_count, 1) != cudaSuccess || alloc(&h->d_upd_total, 1) != cudaSuccess ||
        cudaMallocHost((void **)&h->h_upd_total, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMallocHost((void **)&h->h_halo_count, sizeof(uint32_t)) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_ring_free, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_copy, cudaEventDisableTiming) != cudaSuccess) {
      fail(FF_ERR_OOM_POOL, "deferred update");
      break;
    }
    *h->h_upd_total = 0;
    select_set(h, 0);
    if (cfg->rcp_mode == FF_RCP_HOST) {
      std::vector<uint32_t> tab;
      if (!build_rcp_table(tab, h->rcp_shift)) {
        g_create_error = "ff_create: FF_RCP_HOST needs an x86-64 host whose RCPPS follows the mantissa-table rules";
        st = FF_ERR_BAD_ARG;
        break;
      }
      if (alloc(&h->d_rcp_tab, tab.size()) != cudaSuccess) { fail(FF_ERR_OOM_POOL, "rcp table"); break; }
      if (cudaMemcpy(h->d_rcp_tab, tab.data(), 4 * tab.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        fail(FF_ERR_CUDA, "rcp table upload");
        break;
      }
    }
    if (prewarm_alloc_kernels() != cudaSuccess || prewarm_fuse_kernels() != cudaSuccess ||
        prewarm_mesh_kernels() != cudaSuccess) {
      fail(FF_ERR_CUDA, "kernel load");
      break;
    }
    launch_fill(h->d_tree, h->cfg.branches_max, BRANCHINIT, h->stream);
    cudaMemsetAsync(h->d_stamp, 0, sizeof(uint32_t) * L, h->stream);
    cudaMemsetAsync(h->d_bstamp, 0, sizeof(uint32_t) * (h->cfg.branches_max / 16 + 1), h->stream);
    cudaMemsetAsync(h->d_parent, 0xFF, sizeof(uint32_t) * L, h->stream);
    cudaMemsetAsync(h->d_leaf, 0, sizeof(ushort4) * L, h->stream);
    if (h->d_sdf) {
      cudaMemsetAsync(h->d_sdf, 0, sizeof(float) * L * 512, h->stream);
      cudaMemsetAsync(h->d_wgt, 0, sizeof(float) * L * 512, h->stream);
    } else {
      cudaMemsetAsync(h->d_sdf16, 0, sizeof(__half) * L * 512, h->stream);
      cudaMemsetAsync(h->d_wgt16, 0, sizeof(__half) * L * 512, h->stream);
    }
    cudaMemsetAsync(h->d_col, 0, sizeof(uint16_t) * L * 1536, h->stream);
    cudaMemsetAsync(h->d_upd_mask, 0, sizeof(uint32_t) * L, h->stream);
    cudaMemsetAsync(h->d_upd_count, 0, sizeof(uint32_t), h->stream);
    cudaMemsetAsync(h->d_upd_total, 0, sizeof(unsigned long long), h->stream);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) { fail(FF_ERR_CUDA, "init"); break; }
  } while (0);
  if (st != FF_OK) {
    ff_destroy(h);
    return st;
  }
  *out = h;
  return FF_OK;
}

ff_status ff_destroy(ff_handle *h) {
  if (!h) return FF_ERR_BAD_ARG;
  cudaSetDevice(h->cfg.device);
  if (h->fuse_stream) cudaStreamSynchronize(h->fuse_stream);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->mesh_stream) cudaStreamSynchronize(h->mesh_stream);  // (copies out of the mesh buffers)
  mesh_free(h->mesh);
  h->prof.destroy();
  void *ptrs[] = {h->d_tree, h->d_leaf, h->d_parent, h->d_sdf, h->d_wgt, h->d_sdf16, h->d_wgt16, h->d_col,
                  h->d_stamp, h->d_bstamp, h->d_queue_set[0], h->d_queue_set[1], h->d_cnt_set[0], h->d_cnt_set[1],
                  h->d_barrier, h->d_depth_set[0], h->d_depth_set[1], h->d_bgr_set[0], h->d_bgr_set[1], h->d_pxp,
                  h->d_pyp, h->d_vox, h->d_proc, h->d_bnd, h->d_pend, h->d_keys, h->d_sort_tmp, h->d_rcp_tab,
                  h->d_cnn_params, h->d_cnn_packed, h->d_feat, h->d_a1, h->d_a2, h->d_conf_set[0], h->d_conf_set[1],
                  h->d_batch_set[0], h->d_batch_set[1], h->d_upd_mask, h->d_upd_list, h->d_upd_count,
                  h->d_upd_total, h->d_ring_depth, h->d_ring_bgr, h->d_ring_conf, h->d_seq_vox, h->d_seq_proc,
                  h->d_seq_bnd, h->d_seq_cnt, h->d_loop_map, h->d_loop_slots, h->d_loop_st, h->d_loop_sdf,
                  h->d_loop_wgt, h->d_loop_col};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  for (int k = 0; k < 2; k++) {
    if (h->h_cnt_set[k]) cudaFreeHost(h->h_cnt_set[k]);
    if (h->h_batch_set[k]) cudaFreeHost(h->h_batch_set[k]);
    if (h->ev_fuse[k]) cudaEventDestroy(h->ev_fuse[k]);
  }
  if (h->h_upd_total) cudaFreeHost(h->h_upd_total);
  if (h->h_halo_count) cudaFreeHost(h->h_halo_count);
  if (h->h_seq_cnt) cudaFreeHost(h->h_seq_cnt);
  if (h->h_loop_st) cudaFreeHost(h->h_loop_st);
  if (h->ev_ring_free) cudaEventDestroy(h->ev_ring_free);
  if (h->ev_copy) cudaEventDestroy(h->ev_copy);
  if (h->ev_fin) cudaEventDestroy(h->ev_fin);
  if (h->ev_alloc) cudaEventDestroy(h->ev_alloc);
  if (h->ev_cnn_in) cudaEventDestroy(h->ev_cnn_in);
  if (h->ev_cnn_done) cudaEventDestroy(h->ev_cnn_done);
  if (h->fuse_stream) cudaStreamDestroy(h->fuse_stream);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  if (h->copy_stream) {
    cudaStreamSynchronize(h->copy_stream);
    cudaStreamDestroy(h->copy_stream);
  }
  if (h->ev_bgr_free) cudaEventDestroy(h->ev_bgr_free);
  if (h->ev_bgr_ready) cudaEventDestroy(h->ev_bgr_ready);
  if (h->ev_counters) cudaEventDestroy(h->ev_counters);
  if (h->mesh_stream) cudaStreamDestroy(h->mesh_stream);
  if (h->ev_mesh_ready) cudaEventDestroy(h->ev_mesh_ready);
  for (auto &c : h->mesh_copy)
    if (c.ev) cudaEventDestroy(c.ev);
  if (h->ev_host_images) cudaEventDestroy(h->ev_host_images);
  if (h->ev_host_depth) cudaEventDestroy(h->ev_host_depth);
  if (h->d_hseq_depth) cudaFree(h->d_hseq_depth);
  if (h->d_hseq_bgr) cudaFree(h->d_hseq_bgr);
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  delete h;
  return FF_OK;
}

ff_status ff_set_shard(ff_handle *h, int shard, int shards) {
  if (!h) return FF_ERR_BAD_ARG;
  if (shards < 1 || shard < 0 || shard >= shards)
    return set_err(h, FF_ERR_BAD_ARG, "ff_set_shard: need 0 <= shard < shards");
  if (h->frames || h->n) return set_err(h, FF_ERR_BAD_ARG, "ff_set_shard: set before the first frame");
  h->shard = (uint32_t)shard;
  h->shards = (uint32_t)shards;
  return FF_OK;
}

ff_status ff_halo_export(ff_handle *h, void *d_records, uint64_t capacity, uint64_t *n_records,
                         uint64_t *record_bytes) {
  if (!h || !n_records) return FF_ERR_BAD_ARG;
  CK(cudaSetDevice(h->cfg.device));
  const bool fp16 = h->cfg.storage == FF_STORAGE_FP16;
  if (record_bytes) *record_bytes = halo_record_bytes(fp16);
  // the changes include the waiting frames' updates; the pass's brick list is
  // free once it has run
  FCK(settle(h));
  cudaStream_t s = h->stream;
  const uint32_t nl = std::min(h->leaves_used, h->cfg.leaves_max);
  CK(cudaMemsetAsync(h->d_upd_count, 0, sizeof(uint32_t), s));
  launch_halo_select(h->d_leaf, h->d_stamp, nl, h->halo_since, h->shard, h->shards, h->shift, h->d_upd_list,
                     h->d_upd_count, s);
  CK(cudaMemcpyAsync(h->h_halo_count, h->d_upd_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  const uint32_t n = *h->h_halo_count;
  *n_records = n;
  if (d_records) {
    if (n > capacity) {
      CK(cudaMemsetAsync(h->d_upd_count, 0, sizeof(uint32_t), s));
      CK(cudaStreamSynchronize(s));
      return set_err(h, FF_ERR_BAD_ARG, "ff_halo_export: " + std::to_string(n) + " records, room for " +
                                            std::to_string(capacity));
    }
    launch_halo_pack(h->d_upd_list, n, h->d_sdf, h->d_wgt, h->d_sdf16, h->d_wgt16, h->d_col, d_records, fp16,
                     h->sm_count * 4, s);
    CK(cudaGetLastError());
    h->halo_since = h->frames;
  }
  // the list belongs to the deferred update again
  CK(cudaMemsetAsync(h->d_upd_count, 0, sizeof(uint32_t), s));
  CK(cudaStreamSynchronize(s));
  return FF_OK;
}

ff_status ff_halo_import(ff_handle *h, const void *d_records, uint64_t n_records) {
  if (!h || (n_records && !d_records)) return FF_ERR_BAD_ARG;
  CK(cudaSetDevice(h->cfg.device));
  FCK(settle(h));
  launch_halo_unpack(d_records, n_records, h->cfg.leaves_max, h->d_sdf, h->d_wgt, h->d_sdf16, h->d_wgt16, h->d_col,
                     h->cfg.storage == FF_STORAGE_FP16, h->sm_count * 4, h->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  return FF_OK;
}

ff_status ff_loop_begin(ff_handle *h, uint32_t capacity) {
  if (!h) return FF_ERR_BAD_ARG;
  if (capacity < 1 || capacity > h->cfg.leaves_max)
    return set_err(h, FF_ERR_BAD_ARG, "ff_loop_begin: capacity must be 1..leaves_max");
  CK(cudaSetDevice(h->cfg.device));
  FCK(settle(h));
  cudaStream_t s = h->stream;
  CK(cudaStreamSynchronize(s));
  if (capacity != h->loop_cap) {
    cudaFree(h->d_loop_sdf);
    cudaFree(h->d_loop_wgt);
    cudaFree(h->d_loop_col);
    h->d_loop_sdf = h->d_loop_wgt = nullptr;
    h->d_loop_col = nullptr;
    h->loop_cap = 0;
    CK(alloc(&h->d_loop_sdf, (size_t)capacity * 512));
    CK(alloc(&h->d_loop_wgt, (size_t)capacity * 512));
    CK(alloc(&h->d_loop_col, (size_t)capacity * 1536));
    h->loop_cap = capacity;
  }
  if (!h->d_loop_map) {
    CK(alloc(&h->d_loop_map, (size_t)h->cfg.leaves_max));
    CK(alloc(&h->d_loop_st, (size_t)4));
    CK(cudaMallocHost((void **)&h->h_loop_st, 4 * sizeof(uint32_t)));
  }
  launch_fill(h->d_loop_map, h->cfg.leaves_max, BRANCHINIT, s);
  CK(cudaMemsetAsync(h->d_loop_st, 0, 4 * sizeof(uint32_t), s));
  CK(cudaMemsetAsync(h->d_loop_sdf, 0, sizeof(float) * capacity * 512, s));
  CK(cudaMemsetAsync(h->d_loop_wgt, 0, sizeof(float) * capacity * 512, s));
  CK(cudaMemsetAsync(h->d_loop_col, 0, sizeof(uint16_t) * capacity * 1536, s));
  CK(cudaStreamSynchronize(s));
  return FF_OK;
}

ff_status ff_loop_delete_frame(ff_handle *h, const float *d_depth, const uint8_t *d_red, const uint8_t *d_green,
                               const uint8_t *d_blue, int width, int height, const double K[4], const double R[9],
                               const double t[3], const uint32_t *d_queue, uint32_t n_queue, int *complete) {
  if (!h) return FF_ERR_BAD_ARG;
  if (!h->loop_cap) return set_err(h, FF_ERR_STATE, "ff_loop_delete_frame: call ff_loop_begin first");
  if (!d_depth || !d_red || !d_green || !d_blue || !K || !R || !t || width <= 0 || height <= 0 ||
      (n_queue && !d_queue))
    return set_err(h, FF_ERR_BAD_ARG, "ff_loop_delete_frame: NULL pointer or empty image");
  CK(cudaSetDevice(h->cfg.device));
  FCK(settle(h));
  cudaStream_t s = h->stream;
  if (n_queue > h->loop_slots_cap) {
    cudaFree(h->d_loop_slots);
    h->d_loop_slots = nullptr;
    h->loop_slots_cap = 0;
    CK(alloc(&h->d_loop_slots, (size_t)n_queue));
    h->loop_slots_cap = n_queue;
  }
  if (n_queue) {
    launch_loop_slots(d_queue, n_queue, h->d_loop_map, h->loop_cap, h->d_loop_slots, h->d_loop_st, s);
    LoopFrame L;
    L.q = cam_grid_to_camera(h, K, R, t);  // as deleteOldLoopPoses builds pInv (geometryfusion_mipmap_cpu.cpp:3990-4005)
    L.depth = d_depth;
    L.red = d_red;
    L.green = d_green;
    L.blue = d_blue;
    L.W = width;
    L.H = height;
    L.queue = d_queue;
    L.slots = h->d_loop_slots;
    L.taken = h->d_loop_st + 1;
    L.leaf = h->d_leaf;
    L.sdf = h->d_loop_sdf;
    L.wgt = h->d_loop_wgt;
    L.col = h->d_loop_col;
    L.rcp_tab = h->d_rcp_tab;
    L.rcp_shift = h->rcp_shift;
    L.scale = h->cfg.scale;
    L.thr = h->cfg.threshold;
    launch_loop_delete(L, h->d_rcp_tab != nullptr, h->sm_count * 4, s);
    CK(cudaGetLastError());
  }
  CK(cudaMemcpyAsync(h->h_loop_st, h->d_loop_st, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (complete) *complete = (!n_queue || h->h_loop_st[1] >= n_queue) ? 1 : 0;
  return FF_OK;
}

ff_status ff_loop_get(ff_handle *h, uint32_t *n_mapped, uint32_t *leaf_slot, float *sdf, float *weight,
                      uint16_t *rgb) {
  if (!h || !n_mapped) return FF_ERR_BAD_ARG;
  if (!h->loop_cap) return set_err(h, FF_ERR_STATE, "ff_loop_get: call ff_loop_begin first");
  CK(cudaSetDevice(h->cfg.device));
  cudaStream_t s = h->stream;
  CK(cudaMemcpyAsync(h->h_loop_st, h->d_loop_st, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  const uint32_t n = h->h_loop_st[0];
  *n_mapped = n;
  const uint32_t nl = std::min(h->leaves_used, h->cfg.leaves_max);
  if (leaf_slot && nl) CK(cudaMemcpyAsync(leaf_slot, h->d_loop_map, sizeof(uint32_t) * nl, cudaMemcpyDeviceToHost, s));
  if (sdf && n) CK(cudaMemcpyAsync(sdf, h->d_loop_sdf, sizeof(float) * n * 512, cudaMemcpyDeviceToHost, s));
  if (weight && n) CK(cudaMemcpyAsync(weight, h->d_loop_wgt, sizeof(float) * n * 512, cudaMemcpyDeviceToHost, s));
  if (rgb && n) {
    std::vector<uint16_t> planes((size_t)n * 1536);
    CK(cudaMemcpyAsync(planes.data(), h->d_loop_col, sizeof(uint16_t) * n * 1536, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (size_t b = 0; b < n; b++)
      for (int c = 0; c < 3; c++)
        for (int v = 0; v < 512; v++) rgb[(b * 512 + v) * 3 + c] = planes[b * 1536 + c * 512 + v];
  }
  CK(cudaStreamSynchronize(s));
  return FF_OK;
}

ff_status ff_set_update_batch(ff_handle *h, int frames) {
  if (!h) return FF_ERR_BAD_ARG;
  if (frames < 1 || frames > FUSE_SLOTS_MAX)
    return set_err(h, FF_ERR_BAD_ARG, "ff_set_update_batch: frames must be 1.." + std::to_string(FUSE_SLOTS_MAX));
  CK(cudaSetDevice(h->cfg.device));
  FCK(settle(h));
  h->upd_batch = frames;
  return FF_OK;
}

ff_status ff_set_spin_limit(ff_handle *h, uint32_t iterations) {
  if (!h) return FF_ERR_BAD_ARG;
  h->spin_limit = iterations;
  return FF_OK;
}

ff_status ff_set_cell_generation(ff_handle *h, int mode) {
  if (!h) return FF_ERR_BAD_ARG;
  if (mode != FF_CELLS_INCREMENTAL && mode != FF_CELLS_FULL)
    return set_err(h, FF_ERR_BAD_ARG, "ff_set_cell_generation: mode is FF_CELLS_INCREMENTAL or FF_CELLS_FULL");
  h->full_cells = mode == FF_CELLS_FULL ? 1 : 0;
  return FF_OK;
}

ff_status ff_inject_error(ff_handle *h, int what) {
  if (!h) return FF_ERR_BAD_ARG;
  if (what != 0 && what != FF_INJECT_CONFIDENCE_TIMEOUT)
    return set_err(h, FF_ERR_BAD_ARG, "ff_inject_error: unknown failure");
  h->inject = what;
  return FF_OK;
}

ff_status ff_set_tuning(ff_handle *h, const ff_tuning *t) {
  if (!h || !t) return FF_ERR_BAD_ARG;
  if ((t->dedupe_rows && t->dedupe_rows != 8 && t->dedupe_rows != 16 && t->dedupe_rows != 32) || t->fuse_shape < 0 ||
      t->fuse_shape >= FUSE_SHAPE_COUNT || t->fuse_blocks_per_sm < 0 || t->fuse_blocks_per_sm > 64 ||
      (t->insert_block && (t->insert_block < 64 || t->insert_block > 1024 || t->insert_block % 32)))
    return set_err(h, FF_ERR_BAD_ARG, "ff_set_tuning: dedupe_rows 0/8/16/32, fuse_shape 0..3, "
                                      "fuse_blocks_per_sm 0..64, insert_block 0 or 64..1024 in steps of 32");
  h->tune = *t;
  h->graph_key.clear();  // launches change: record again
  return FF_OK;
}

ff_status ff_sync(ff_handle *h) {
  if (!h) return FF_ERR_BAD_ARG;
  CK(cudaSetDevice(h->cfg.device));
  FCK(settle(h));
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaStreamSynchronize(h->fuse_stream));
  return ff_mesh_wait(h);
}

ff_status ff_set_stream(ff_handle *h, void *cuda_stream) {
  if (!h) return FF_ERR_BAD_ARG;
  cudaSetDevice(h->cfg.device);
  settle(h);
  cudaStreamSynchronize(h->stream);
  if (h->own_stream) cudaStreamDestroy(h->stream);
  if (cuda_stream) {
    h->stream = (cudaStream_t)cuda_stream;
    h->own_stream = false;
  } else {
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
  }
  return FF_OK;
}

// ---------------------------------------------------------------- frames ----
//
// A frame runs in three phases, shared by the single-map entry points and
// the batched one:
//   prepare  -- host side: first-frame volume, ray factors, counter reset,
//               the frame's descriptor (camera parameters in FP64 -> FP32);
//   launch   -- de-duplication, insert, leaf finalisation and the gated voxel
//               update of every frame of the batch, one launch each;
//   finish   -- after the one synchronisation: errors, bookkeeping, and the
//               volume growth (with its update launched again) where needed.

struct FramePlan {
  const uint16_t *d_depth;
  const uint8_t *d_bgr;
  int W, H;
  float scaling, maxcam;
  uint32_t frame, leaves_before;
  bool one_sync;
  // the counters reach the host before the leaf finalisation: their queued
  // count does not yet hold the frame's new leaves
  bool counters_early = false;
};

static uint32_t pad32(uint32_t v) { return (v + 31u) & ~31u; }

// Host part before the launches; fills the frame's descriptor.
// side: a single-map frame whose update runs on fuse_stream; its confidence
// network (learned weight) runs there too, overlapping the de-duplication and
// the insert, and the counter copy waits for it (it reports into them).
static ff_status frame_prepare(ff_handle *h, const uint16_t *d_depth, const uint8_t *d_bgr, int W, int H,
                               const double *K, const double *R, const double *t, float scaling, float maxcam,
                               MapFrame &mf, FramePlan &plan, bool side = false) {
  cudaStream_t s = h->stream;
  CamF p = cam_world_to_grid(h, K, R, t);
  Counters &hc = *h->h_cnt;
  if (!h->n) {
    // first frame: integer bounding box of the valid points (computeBoundingboxIntCPU)
    memset(&hc, 0, sizeof(Counters));
    for (int r = 0; r < 3; r++) {
      hc.box_min[r] = 1000000;
      hc.box_max[r] = -1000000;
    }
    CK(cudaMemcpyAsync(h->d_cnt, &hc, sizeof(Counters), cudaMemcpyHostToDevice, s));
    launch_first_bbox(d_depth, W, H, p, scaling, maxcam, h->bandwidth, h->d_cnt, s);
    CK(cudaMemcpyAsync(&hc, h->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    set_initial_volume(h, hc.box_min, hc.box_max);
    p = cam_world_to_grid(h, K, R, t);
  }
  if (h->img_w != W || h->img_h != H) {
    // _pxp/_pyp, recomputed on a size change only (geometryfusion_mipmap_cpu.cpp:1745-1764)
    std::vector<float> px(W), py(H);
    for (int x = 0; x < W; x++) px[x] = ((float)x - p.cx) / p.fx;
    for (int y = 0; y < H; y++) py[y] = ((float)y - p.cy) / p.fy;
    cudaFree(h->d_pxp);
    cudaFree(h->d_pyp);
    h->d_pxp = h->d_pyp = nullptr;
    CK(alloc(&h->d_pxp, W));
    CK(alloc(&h->d_pyp, H));
    CK(cudaMemcpyAsync(h->d_pxp, px.data(), sizeof(float) * W, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h->d_pyp, py.data(), sizeof(float) * H, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    h->img_w = W;
    h->img_h = H;
  }
  plan.d_depth = d_depth;
  plan.d_bgr = d_bgr;
  plan.W = W;
  plan.H = H;
  plan.scaling = scaling;
  plan.maxcam = maxcam;
  plan.frame = h->frames + 1;
  plan.leaves_before = h->leaves_used;
  plan.one_sync = finalize_small_fits((uint32_t)(W * H));
  memset(&mf, 0, sizeof(MapFrame));
  mf.depth = d_depth;
  mf.bgr = d_bgr;
  mf.pxp = h->d_pxp;
  mf.pyp = h->d_pyp;
  mf.p = p;
  // voxel -> camera parameters are taken before any grow() of this frame,
  // as in the reference (pInv is built before the traversal)
  mf.q = cam_grid_to_camera(h, K, R, t);
  mf.scaling = scaling;
  mf.maxcam = maxcam;
  mf.scale = h->cfg.scale;
  mf.thr = h->cfg.threshold;
  mf.W = W;
  mf.H = H;
  dedupe_tiles(W, H, &mf.tilesX, &mf.tilesY, 16);  // frame_launch may choose taller tiles
  mf.npix = (uint32_t)(W * H);
  mf.frame = plan.frame;
  mf.n = h->n;
  mf.bw = (uint32_t)h->bandwidth;
  mf.leaves_max = h->cfg.leaves_max;
  mf.branches_max = h->cfg.branches_max;
  mf.leaves_before = plan.leaves_before;
  mf.pend_cap = (uint32_t)(W * H);
  mf.nq_host = 0;
  mf.tree = h->d_tree;
  mf.leaf = h->d_leaf;
  mf.parent = h->d_parent;
  mf.sdf = h->d_sdf;
  mf.wgt = h->d_wgt;
  mf.sdf16 = h->d_sdf16;
  mf.wgt16 = h->d_wgt16;
  mf.col = h->d_col;
  mf.stamp = h->d_stamp;
  mf.bstamp = h->d_bstamp;
  mf.queue = h->d_queue;
  mf.rank = h->d_keys + 5 * h->cap_pix;
  mf.pend = h->d_pend;
  mf.vox = h->d_vox;
  mf.proc = h->d_proc;
  mf.bnd = h->d_bnd;
  mf.cnt = h->d_cnt;
  mf.branches_init = h->branches_used;  // (the counters are set up on the device)
  mf.rcp_tab = h->d_rcp_tab;
  mf.rcp_shift = h->rcp_shift;
  mf.conf = nullptr;
  mf.shard = h->shard;
  mf.shards = h->shards;
  mf.spin_limit = h->spin_limit;
  mf.count_levels = h->prof.on ? 1u : 0u;
  for (int r = 0; r < 3; r++) mf.shift[r] = h->shift[r];
  if (h->cur_slot >= 0) {
    mf.upd_mask = h->d_upd_mask;
    mf.upd_list = h->d_upd_list;
    mf.upd_count = h->d_upd_count;
    mf.upd_slot = h->cur_slot;
  }
  if (h->conf_tau_cm > 0.0f) {
    // the frame's confidence map, ahead of the launches that read it on this stream
    const size_t npx = (size_t)W * H;
    if (npx > h->conf_cap) {
      cudaFree(h->d_feat);
      cudaFree(h->d_a1);
      cudaFree(h->d_a2);
      h->d_feat = h->d_a1 = h->d_a2 = nullptr;
      for (int k = 0; k < 2; k++) {
        cudaFree(h->d_conf_set[k]);
        h->d_conf_set[k] = nullptr;
      }
      h->conf_cap = 0;
      CK(alloc(&h->d_feat, npx * CNN_FEAT_CH));
      CK(alloc(&h->d_a1, npx * CNN_HIDDEN));
      CK(alloc(&h->d_a2, npx * CNN_HIDDEN));
      CK(alloc(&h->d_conf_set[0], npx));
      CK(alloc(&h->d_conf_set[1], npx));
      h->d_conf = h->d_conf_set[h->set];
      h->conf_cap = npx;
    }
    // a waiting frame's confidence map lives in its ring slot until the pass
    if (h->cur_slot >= 0) h->d_conf = h->d_ring_conf + (size_t)h->cur_slot * h->ring_pix;
    const float kf[4] = {(float)K[0], (float)K[1], (float)K[2], (float)K[3]};
    cudaStream_t cs = s;
    if ((side && plan.one_sync) || h->cnn_on_side) {
      // after the depth image is ready on the map's stream; the network
      // feeds only the voxel update, so the frame's allocation need not wait
      cs = h->fuse_stream;
      CK(cudaEventRecord(h->ev_cnn_in, s));
      CK(cudaStreamWaitEvent(cs, h->ev_cnn_in, 0));
    }
    const int pc = h->prof.begin(ST_CONFIDENCE, cs);
    CK(cnn_features(d_depth, 1, W, H, scaling, kf, h->d_feat, cs));
    CK(cnn_forward(h->d_cnn_params, h->d_cnn_packed, h->cnn_packed_ready, h->d_feat, 1, W, H, h->d_a1, h->d_a2,
                   h->d_conf, h->conf_tau_cm, &h->d_cnt->cnn_error, cs));
    h->cnn_packed_ready = true;
    if (h->inject == FF_INJECT_CONFIDENCE_TIMEOUT) {
      // the word the network sets when one of its waits gives up
      CK(cudaMemsetAsync(&h->d_cnt->cnn_error, 0xFF, sizeof(uint32_t), cs));
      h->inject = 0;
    }
    // depth -> features -> a1 -> a2 -> confidence, each written once and read once
    h->prof.end(pc, (double)npx * ((2 + 16) + (16 + 32) + (32 + 32) + (32 + 4)), cs);
    if (cs != s) {
      CK(cudaEventRecord(h->ev_cnn_done, cs));
      h->cnn_pending = true;
    }
    h->conf_w = W;
    h->conf_h = H;
    mf.conf = h->d_conf;
  }
  if (h->inject == FF_INJECT_CONFIDENCE_TIMEOUT) {
    // no network this frame: the word is set all the same (the frame's
    // counter set-up keeps it; the update and the host read it)
    CK(cudaMemsetAsync(&h->d_cnt->cnn_error, 0xFF, sizeof(uint32_t), s));
    h->inject = 0;
  }
  return FF_OK;
}

// The launch plan of a batch: tile height, the groups of whole maps that
// share one cooperative de-duplication launch, padded pixel total.
struct LaunchPlan {
  int rows = 16;
  uint32_t pix = 0;
  double npix = 0;
  std::vector<std::array<uint32_t, 3>> groups;  // first map, end map, tiles
};

// Host part: tiles, prefixes and rounds of the batch in lead->h_batch (n
// frames), and its launch plan.
static ff_status frame_plan(ff_handle *lead, int n, LaunchPlan &lp) {
  ff_handle *h = lead;  // (error reporting)
  BatchDesc &B = *lead->h_batch;
  B.n = n;
  // 16-row tiles when they fit one cooperative launch, else 32-row tiles in
  // as many launches (groups of whole maps) as needed
  uint32_t tiles16 = 0, cap16 = 0, cap32 = 0;
  for (int i = 0; i < n; i++) tiles16 += (uint32_t)dedupe_tiles(B.f[i].W, B.f[i].H, nullptr, nullptr, 16);
  CK(dedupe_capacity(lead->cfg.device, 16, cap16));
  CK(dedupe_capacity(lead->cfg.device, 32, cap32));
  int rows = tiles16 <= cap16 ? 16 : 32;
  if (lead->tune.dedupe_rows == 32 || (lead->tune.dedupe_rows == 16 && tiles16 <= cap16)) rows = lead->tune.dedupe_rows;
  uint32_t cap = rows == 16 ? cap16 : cap32;
  if (lead->tune.dedupe_rows == 8) {
    uint32_t tiles8 = 0, cap8 = 0;
    for (int i = 0; i < n; i++) tiles8 += (uint32_t)dedupe_tiles(B.f[i].W, B.f[i].H, nullptr, nullptr, 8);
    CK(dedupe_capacity(lead->cfg.device, 8, cap8));
    if (tiles8 <= cap8) rows = 8, cap = cap8;
  }
  for (int i = 0; i < n; i++) {
    const uint32_t nt = (uint32_t)dedupe_tiles(B.f[i].W, B.f[i].H, &B.f[i].tilesX, &B.f[i].tilesY, rows);
    if (nt > cap) return set_err(lead, FF_ERR_BAD_ARG, "image too large for the de-duplication launch");
  }
  int rounds = 1;
  uint32_t tiles = 0, pix = 0;
  for (int i = 0; i < n; i++) {
    rounds = std::max(rounds, B.f[i].tilesX + B.f[i].tilesY + 1);
    tiles += (uint32_t)(B.f[i].tilesX * B.f[i].tilesY);
    pix += pad32(B.f[i].npix);
    B.tile_end[i] = tiles;
    B.pix_end[i] = pix;
  }
  B.max_rounds = rounds;
  lp.rows = rows;
  lp.pix = pix;
  lp.npix = 0;
  for (int i = 0; i < n; i++) lp.npix += (double)B.f[i].npix;
  lp.groups.clear();
  for (int m0 = 0; m0 < n;) {
    int m1 = m0;
    uint32_t group = 0;
    while (m1 < n && group + (uint32_t)(B.f[m1].tilesX * B.f[m1].tilesY) <= cap)
      group += (uint32_t)(B.f[m1].tilesX * B.f[m1].tilesY), m1++;
    if (lp.groups.size() >= (size_t)(BARRIER_WORDS / 8))
      return set_err(lead, FF_ERR_BAD_ARG, "batch too large for the de-duplication");
    lp.groups.push_back({(uint32_t)m0, (uint32_t)m1, group});
    m0 = m1;
  }
  return FF_OK;
}

// Device part: upload the descriptor and launch the de-duplication and (with
// insert) the insert on the lead's stream.
static ff_status frame_issue(ff_handle *lead, int n, const LaunchPlan &lp, bool insert = true) {
  ff_handle *h = lead;  // (error reporting)
  cudaStream_t s = lead->stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(s, &cap));
  // one map: the descriptor travels as the de-duplication launch's parameter,
  // which stores it for the later kernels; otherwise it is uploaded (a
  // recorded graph re-reads it from pinned memory at each replay)
  const bool by_param = n == 1 && lp.groups.size() == 1 && cap == cudaStreamCaptureStatusNone;
  if (!by_param)
    CK(cudaMemcpyAsync(lead->d_batch, lead->h_batch, batch_desc_bytes(n), cudaMemcpyHostToDevice, s));
  // (a recorded graph always clears them: its replays cannot look)
  if (lead->barrier_dirty || cap != cudaStreamCaptureStatusNone) {
    CK(cudaMemsetAsync(lead->d_barrier, 0, BARRIER_WORDS * sizeof(uint32_t), s));
    lead->barrier_dirty = false;
  }
  int pi = lead->prof.begin(ST_DEDUPE, s);
  if (by_param)
    CK(launch_dedupe_one(lead->h_batch, lead->d_batch, lp.groups[0][2], lp.rows, lead->d_barrier, lead->cfg.device,
                         s));
  else
    for (size_t g = 0; g < lp.groups.size(); g++)
      CK(launch_dedupe(lead->d_batch, (int)lp.groups[g][0], (int)lp.groups[g][1], lp.groups[g][2], lp.rows,
                       lead->d_barrier + 8 * g, lead->cfg.device, s));
  lead->prof.end(pi, lp.npix * 2, s);  // the depth image read (the keys and flags it writes stay in L2)
  if (!insert) {
    CK(cudaGetLastError());
    return FF_OK;
  }
  if (lead->fin_pending) {
    // the previous frame's finalisation (on fuse_stream) completes the octree
    CK(cudaStreamWaitEvent(s, lead->ev_fin, 0));
    lead->fin_pending = false;
  }
  pi = lead->prof.begin(ST_INSERT, s);
  launch_insert(lead->d_batch, lp.pix, s, lead->tune.insert_block > 0 ? lead->tune.insert_block : 256);
  // 16 B per octree level probed, counted on the device (set after the frame)
  lead->prof.end(pi, 0.0, s);
  lead->pi_insert = pi;
  CK(cudaGetLastError());
  return FF_OK;
}

static ff_status frame_launch(ff_handle *lead, int n) {
  LaunchPlan lp;
  ff_status st = frame_plan(lead, n, lp);
  return st != FF_OK ? st : frame_issue(lead, n, lp);
}

// counters: a single map's counters are copied to the host before the
// finalisation (which only places the new leaves and queues them: the host
// adds their number itself), and this event recorded after the copy, so the
// finalisation and the update overlap the host's return and its next frame.
static ff_status frame_launch_update(ff_handle *lead, int n, uint32_t max_npix, int &pi_fin, int &pi_fuse,
                                     cudaEvent_t counters = nullptr, bool side = false, bool deferred = false) {
  ff_handle *h = lead;  // (error reporting)
  cudaStream_t s = lead->stream;
  if (counters) {
    if (lead->cnn_pending) {
      // the frame's confidence network reports into these counters
      CK(cudaStreamWaitEvent(s, lead->ev_cnn_done, 0));
      lead->cnn_pending = false;
    }
    if (lead->copy_pending) {
      // a device frame's images are in its ring slot before the call returns
      CK(cudaStreamWaitEvent(s, lead->ev_copy, 0));
      lead->copy_pending = false;
    }
    CK(cudaMemcpyAsync(lead->h_cnt, lead->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, s));
    CK(cudaEventRecord(counters, s));
  }
  // side: the finalisation and the update run on fuse_stream after the insert
  cudaStream_t fs = s;
  if (side) {
    fs = lead->fuse_stream;
    CK(cudaEventRecord(lead->ev_alloc, s));
    CK(cudaStreamWaitEvent(fs, lead->ev_alloc, 0));
  }
  pi_fin = lead->prof.begin(ST_FINALIZE, fs);
  if (!launch_finalize_small(lead->d_batch, n, max_npix, lead->cfg.device, fs))
    return set_err(lead, FF_ERR_CUDA, "leaf finalisation could not be launched");
  if (side) {
    CK(cudaEventRecord(lead->ev_fin, fs));
    lead->fin_pending = true;
  }
  // the new leaves' parents: after the event the next frame's insert waits for
  launch_parents_frames(lead->d_batch, n, fs);
  lead->prof.end(pi_fin, 0.0, fs);
  if (!deferred) {
    pi_fuse = lead->prof.begin(ST_FUSE, fs);
    // enough blocks for a frame's bricks in one pass; blocks loop over larger batches
    const int shape = lead->tune.fuse_shape;
    const int per_sm =
        lead->tune.fuse_blocks_per_sm > 0 ? lead->tune.fuse_blocks_per_sm : 8 / fuse_shape_bricks(shape);
    launch_fuse(lead->d_batch, n, true, lead->cfg.storage, lead->d_rcp_tab != nullptr, lead->sm_count * per_sm, fs,
                shape);
    lead->prof.end(pi_fuse, 0.0, fs);
  }
  if (side) {
    CK(cudaEventRecord(lead->ev_fuse[lead->set], fs));
    lead->last_fuse = lead->set;
  }
  CK(cudaGetLastError());
  return FF_OK;
}

// After the synchronisation: one map's frame.  mf is its descriptor (for the
// update that runs now when the frame took the sort path or had to grow).
static ff_status frame_finish(ff_handle *h, const FramePlan &plan, MapFrame &mf, int pi_fin, int pi_fuse,
                              int32_t *queued) {
  cudaStream_t s = h->stream;
  const Counters &hc = *h->h_cnt;
  if (hc.top_created) h->top_changed = true;
  if (hc.error & ERR_DEDUPE_FAILED) {
    // the insert, the finalisation and the update left the frame out: the
    // map is as it was before the call
    h->barrier_dirty = true;
    if (hc.cnn_error) {
      CK(join_fuse(h));
      CK(cudaStreamSynchronize(s));
      CK(cudaMemsetAsync(&h->d_cnt->cnn_error, 0, sizeof(uint32_t), s));
      CK(cudaStreamSynchronize(s));
    }
    return set_err(h, FF_ERR_TIMEOUT,
                   (hc.error & ERR_DEDUPE_TIMEOUT)
                       ? "a bounded device-side wait gave up in the de-duplication; the frame was not fused"
                       : "the de-duplication did not settle within its round limit; the frame was not fused");
  }
  if (hc.error & ERR_PENDING_OVERFLOW) return set_err(h, FF_ERR_STATE, "pending-leaf buffer overflow");
  if (hc.error & ERR_BRANCH_OVERFLOW) h->meshing_ok = false;
  // A wait of the octree insert or of the confidence network that gave up:
  // the frame's new bricks are placed (the octree stays consistent) and the
  // bookkeeping below is done, but its voxel update is skipped (on the device
  // as well); the call then reports FF_ERR_TIMEOUT.
  const bool insert_timeout = (hc.error & ERR_SPIN_TIMEOUT) != 0;
  const bool cnn_failed = hc.cnn_error != 0;
  const bool skip_update = insert_timeout || cnn_failed;
  const uint32_t leaves_before = plan.leaves_before;
  const int W = plan.W, H = plan.H;
  h->branches_used = std::min(hc.branches_used, h->cfg.branches_max);
  h->processed = hc.processed;
  h->dedupe_rounds = hc.dedupe_iters;
  const uint32_t npend = hc.pending;
  uint32_t new_queued = 0;
  if (leaves_before < h->cfg.leaves_max) new_queued = std::min(npend, h->cfg.leaves_max - leaves_before);
  // counters read after the finalisation already include the new leaves
  const uint32_t nq = plan.one_sync && !plan.counters_early ? hc.queued : hc.queued + new_queued;
  if (!plan.one_sync && npend) {
    pi_fin = h->prof.begin(ST_FINALIZE, s);
    uint64_t *k_in = reinterpret_cast<uint64_t *>(h->d_keys),
             *k_out = reinterpret_cast<uint64_t *>(h->d_keys + 2 * h->cap_pix);
    uint32_t *v_out = h->d_keys + 4 * h->cap_pix;
    int end_bit = 1;
    while ((1u << end_bit) < (uint32_t)(W * H)) end_bit++;
    CK(sort_pending(h->d_pend, (int)npend, k_in, k_out, v_out, h->d_sort_tmp, h->sort_tmp_bytes, end_bit, s));
    launch_finalize(h->d_pend, v_out, (int)npend, leaves_before, h->cfg.leaves_max, h->d_tree, h->d_leaf,
                    plan.frame, h->d_stamp, h->d_queue, h->d_cnt, s);
    launch_parents((int)npend, leaves_before, h->cfg.leaves_max, h->d_tree, h->n, h->d_leaf, h->d_parent, s);
    h->prof.end(pi_fin, 0.0, s);
  }
  h->prof.set_bytes(pi_fin, (double)npend * 8);  // 8 B per new brick
  if (h->pi_insert >= 0) h->prof.set_bytes(h->pi_insert, 16.0 * hc.levels);
  h->leaves_used += npend;
  h->new_leaves = npend;
  bool fuse_now = !plan.one_sync && !skip_update;
  if (h->leaves_used < h->cfg.leaves_max && h->branches_used < h->cfg.branches_max &&
      (hc.box_min[0] < 0 || hc.box_min[1] < 0 || hc.box_min[2] < 0 || hc.box_max[0] >= (int)h->n ||
       hc.box_max[1] >= (int)h->n || hc.box_max[2] >= (int)h->n)) {
    // (with one synchronisation the update stood aside for this); the growth
    // moves leaf positions that the waiting frames' update and updates still
    // in flight read: those run first
    FCK(flush_updates(h));
    CK(join_fuse(h));
    int pi = h->prof.begin(ST_GROW, s);
    const double tree_bytes = (double)h->branches_used * 4 * 2 + (double)h->leaves_used * 8 * 2;
    ff_status st = grow(h, hc.box_min, hc.box_max);
    h->prof.end(pi, tree_bytes, s);  // octree and leaf positions read and written
    if (st != FF_OK) return st;
    // the brick ownership of a part follows the moved positions
    for (int r = 0; r < 3; r++) mf.shift[r] = h->shift[r];
    fuse_now = !skip_update;
  }
  // fuse: every voxel of every queued brick read and written: SDF, weight
  // (4+4 B, or 2+2 B in FP16) and three 16-bit colour channels
  const double brick_bytes = 512.0 * 2 * ((h->cfg.storage == FF_STORAGE_FP16 ? 4 : 8) + 6);
  if (fuse_now && nq) {
    FCK(flush_updates(h));
    CK(join_fuse(h));  // after the previous frames' updates
    // this map's own descriptor, with the host's count (leaf positions may
    // have moved with the growth; the camera parameters are the frame's)
    mf.nq_host = nq;
    h->h_batch->n = 1;
    h->h_batch->max_rounds = 1;
    h->h_batch->tile_end[0] = 0;
    h->h_batch->pix_end[0] = 0;
    h->h_batch->f[0] = mf;
    CK(cudaMemcpyAsync(h->d_batch, h->h_batch, batch_desc_bytes(1), cudaMemcpyHostToDevice, s));
    pi_fuse = h->prof.begin(ST_FUSE, s);
    launch_fuse(h->d_batch, 1, false, h->cfg.storage, h->d_rcp_tab != nullptr, (int)nq, s);
    h->prof.end(pi_fuse, 0.0, s);
    // the descriptor is read by the update: keep it until it has run
    CK(cudaStreamSynchronize(s));
  }
  h->prof.set_bytes(pi_fuse, (double)nq * brick_bytes);
  CK(cudaGetLastError());
  if (h->leaves_used > h->cfg.leaves_max) h->meshing_ok = false;
  h->queued = nq;
  h->d_queue_last = mf.queue;
  h->frames++;
  mesh_note_frame(h->mesh);
  if (queued) *queued = (int32_t)nq;
  if (h->cur_slot >= 0 && plan.one_sync && !skip_update && !fuse_now) {
    // the finalisation marked the frame's bricks: the frame waits for the
    // pass, which reads its slot's images
    FuseSlot &fs_ = h->upd_slot[h->cur_slot];
    fs_.q = mf.q;
    // a sequence's frames are read where the caller keeps them (the call
    // waits for their update); other frames from their ring slot
    fs_.depth = h->seq_images ? mf.depth : h->d_ring_depth + (size_t)h->cur_slot * h->ring_pix;
    fs_.bgr = h->seq_images ? mf.bgr : h->d_ring_bgr + (size_t)h->cur_slot * h->ring_pix * 3;
    fs_.conf = mf.conf;
    fs_.W = plan.W;
    fs_.H = plan.H;
    fs_.scaling = plan.scaling;
    fs_.maxcam = plan.maxcam;
    h->upd_pending = h->cur_slot + 1;
    h->pass_frame_bricks += nq;
    h->fused_frame_bricks += nq;
    if (h->upd_pending >= h->upd_batch) FCK(flush_updates(h));
  } else if (!skip_update) {
    // updated by itself (on the device, gated, or just now after a growth)
    h->fused_frame_bricks += nq;
    h->direct_bricks += nq;
  }
  if (cnn_failed) {
    // the word is kept across frames: clear it once every kernel of the
    // frame that reads it has run
    CK(join_fuse(h));
    CK(cudaStreamSynchronize(s));
    CK(cudaMemsetAsync(&h->d_cnt->cnn_error, 0, sizeof(uint32_t), s));
    CK(cudaStreamSynchronize(s));
    return set_err(h, FF_ERR_TIMEOUT,
                   "a bounded device-side wait gave up in the confidence network; the frame's bricks were "
                   "allocated but not updated");
  }
  if (insert_timeout)
    return set_err(h, FF_ERR_TIMEOUT,
                   "a bounded device-side wait gave up in the octree insert; the frame's bricks found so far "
                   "were allocated but not updated");
  return FF_OK;
}

// The frame, with depth/bgr already on the device (h->d_depth/h->d_bgr or caller memory).
static ff_status add_map_device(ff_handle *h, const uint16_t *d_depth, const uint8_t *d_bgr, bool bgr_pending,
                                int W, int H, const double *K, const double *R, const double *t, float scaling,
                                float maxcam, int32_t *queued) {
  cudaStream_t s = h->stream;
  FramePlan plan;
  MapFrame mf;
  ff_status st = frame_prepare(h, d_depth, d_bgr, W, H, K, R, t, scaling, maxcam, mf, plan, true);
  if (st != FF_OK) return st;
  h->h_batch->f[0] = mf;
  st = frame_launch(h, 1);
  if (st != FF_OK) return st;
  if (bgr_pending) CK(cudaStreamWaitEvent(s, h->ev_bgr_ready, 0));
  int pi_fin = -1, pi_fuse = -1;
  if (plan.one_sync) {
    // the frame returns once its counters are on the host; its leaf
    // finalisation (and, for a deferred frame, the marking of its bricks for
    // the next pass; else its voxel update, gated on the device) keeps
    // running, ordered before anything that follows on the stream
    plan.counters_early = true;
    st = frame_launch_update(h, 1, (uint32_t)(W * H), pi_fin, pi_fuse, h->ev_counters, true, h->cur_slot >= 0);
    if (st != FF_OK) return st;
    CK(wait_event_polling(h->ev_counters));
  } else {
    CK(cudaMemcpyAsync(h->h_cnt, h->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
  }
  st = frame_finish(h, plan, mf, pi_fin, pi_fuse, queued);
  // the previous frame's update has finished reading its images (a deferred
  // frame's images are the ring's copies instead)
  if (st == FF_OK && h->cur_slot < 0 && h->last_fuse >= 0) CK(cudaEventSynchronize(h->ev_fuse[h->set ^ 1]));
  return st;
}

// Whether a single-map frame of W x H pixels waits for a deferred update
// pass: every frame the one-block leaf finalisation takes (it marks the
// frame's bricks), when passes take more than one frame.
static bool deferrable(const ff_handle *h, int W, int H) {
  return h->upd_batch > 1 && finalize_small_fits((uint32_t)W * (uint32_t)H);
}

// Before a single-map frame: its buffer set, free once the update two frames
// back has finished with it.
static ff_status begin_frame(ff_handle *h) {
  const int k = (int)(h->frames & 1u);
  select_set(h, k);
  CK(cudaStreamWaitEvent(h->stream, h->ev_fuse[k], 0));
  return FF_OK;
}

ff_status ff_add_map_u16(ff_handle *h, const uint16_t *depth, int width, int height, size_t depth_pitch,
                         const uint8_t *bgr, size_t bgr_pitch, const double K[4], const double R[9],
                         const double t[3], float scaling, float maxcam, int32_t *queued) {
  if (!h) return FF_ERR_BAD_ARG;
  if (!depth || !bgr || !K || !R || !t || width <= 0 || height <= 0)
    return set_err(h, FF_ERR_BAD_ARG, "ff_add_map_u16: NULL pointer or empty image");
  h->cur_slot = -1;
  CK(cudaSetDevice(h->cfg.device));
  ff_status st = ensure_image(h, width, height);
  if (st != FF_OK) return st;
  const bool defer = deferrable(h, width, height);
  if (defer && (st = ensure_ring(h, width, height)) != FF_OK) return st;
  st = begin_frame(h);
  if (st != FF_OK) return st;
  if (!depth_pitch) depth_pitch = sizeof(uint16_t) * width;
  if (!bgr_pitch) bgr_pitch = 3 * (size_t)width;
  // a deferred frame's images go to its ring slot (free once the last pass
  // that read the ring has run)
  uint16_t *dd = h->d_depth;
  uint8_t *db = h->d_bgr;
  if (defer) {
    h->cur_slot = h->upd_pending;
    dd = h->d_ring_depth + (size_t)h->cur_slot * h->ring_pix;
    db = h->d_ring_bgr + (size_t)h->cur_slot * h->ring_pix * 3;
    if (h->ring_read) {
      CK(cudaStreamWaitEvent(h->stream, h->ev_ring_free, 0));
      CK(cudaStreamWaitEvent(h->copy_stream, h->ev_ring_free, 0));
    }
  }
  CK(cudaMemcpy2DAsync(dd, sizeof(uint16_t) * width, depth, depth_pitch, sizeof(uint16_t) * width, height,
                       cudaMemcpyHostToDevice, h->stream));
  // the colour copy waits for the previous frame's update (the last reader of
  // d_bgr) and overlaps this frame's allocation kernels
  CK(cudaEventRecord(h->ev_bgr_free, h->stream));
  CK(cudaStreamWaitEvent(h->copy_stream, h->ev_bgr_free, 0));
  CK(cudaStreamWaitEvent(h->copy_stream, h->ev_fuse[h->set], 0));  // this set's last reader
  CK(cudaMemcpy2DAsync(db, 3 * (size_t)width, bgr, bgr_pitch, 3 * (size_t)width, height, cudaMemcpyHostToDevice,
                       h->copy_stream));
  CK(cudaEventRecord(h->ev_bgr_ready, h->copy_stream));
  st = add_map_device(h, dd, db, true, width, height, K, R, t, scaling, maxcam, queued);
  h->cur_slot = -1;
  // the caller's image must not be read after return, error paths included
  cudaStreamSynchronize(h->copy_stream);
  return st;
}

ff_status ff_add_map_u16_device(ff_handle *h, const uint16_t *d_depth, const uint8_t *d_bgr, int width, int height,
                                const double K[4], const double R[9], const double t[3], float scaling,
                                float maxcam, int32_t *queued) {
  if (!h) return FF_ERR_BAD_ARG;
  if (!d_depth || !d_bgr || !K || !R || !t || width <= 0 || height <= 0)
    return set_err(h, FF_ERR_BAD_ARG, "ff_add_map_u16_device: NULL pointer or empty image");
  h->cur_slot = -1;
  h->copy_pending = false;
  CK(cudaSetDevice(h->cfg.device));
  ff_status st = ensure_image(h, width, height);
  if (st != FF_OK) return st;
  const bool defer = deferrable(h, width, height);
  if (defer && (st = ensure_ring(h, width, height)) != FF_OK) return st;
  st = begin_frame(h);
  if (st != FF_OK) return st;
  if (defer) {
    // the images are copied into the frame's ring slot (after the work the
    // caller ordered on the map's stream, and after the last pass that read
    // the ring); the call returns once the copies are done
    h->cur_slot = h->upd_pending;
    const size_t npix = (size_t)width * height;
    CK(cudaEventRecord(h->ev_bgr_free, h->stream));
    CK(cudaStreamWaitEvent(h->copy_stream, h->ev_bgr_free, 0));
    if (h->ring_read) CK(cudaStreamWaitEvent(h->copy_stream, h->ev_ring_free, 0));
    CK(cudaMemcpyAsync(h->d_ring_depth + (size_t)h->cur_slot * h->ring_pix, d_depth, 2 * npix,
                       cudaMemcpyDeviceToDevice, h->copy_stream));
    CK(cudaMemcpyAsync(h->d_ring_bgr + (size_t)h->cur_slot * h->ring_pix * 3, d_bgr, 3 * npix,
                       cudaMemcpyDeviceToDevice, h->copy_stream));
    CK(cudaEventRecord(h->ev_copy, h->copy_stream));
    h->copy_pending = true;
  }
  st = add_map_device(h, d_depth, d_bgr, false, width, height, K, R, t, scaling, maxcam, queued);
  if (h->copy_pending) {
    // (an error returned before the counter copy waited for it)
    cudaEventSynchronize(h->ev_copy);
    h->copy_pending = false;
  }
  h->cur_slot = -1;
  return st;
}

// Per-frame buffers of a sequence of up to `frames` frames of W x H pixels.
static ff_status ensure_seq(ff_handle *h, int W, int H, int frames) {
  const size_t pix = (size_t)W * H, bnd = dedupe_boundary_elems(W, H);
  if (frames <= h->seq_frames && pix <= h->seq_pix && bnd <= h->seq_bnd) return FF_OK;
  const int nf = std::max(frames, h->seq_frames);
  const size_t np = std::max(pix, h->seq_pix), nb = std::max(bnd, h->seq_bnd);
  cudaFree(h->d_seq_vox);
  cudaFree(h->d_seq_proc);
  cudaFree(h->d_seq_bnd);
  h->d_seq_vox = nullptr;
  h->d_seq_proc = nullptr;
  h->d_seq_bnd = nullptr;
  h->seq_frames = 0;
  CK(alloc(&h->d_seq_vox, np * nf));
  CK(alloc(&h->d_seq_proc, np * nf));
  CK(alloc(&h->d_seq_bnd, nb * nf));
  if (!h->d_seq_cnt) {
    CK(alloc(&h->d_seq_cnt, (size_t)BATCH_MAX));
    CK(cudaMemset(h->d_seq_cnt, 0, sizeof(Counters) * BATCH_MAX));
    CK(cudaMallocHost((void **)&h->h_seq_cnt, sizeof(Counters) * BATCH_MAX));
  }
  h->seq_frames = nf;
  h->seq_pix = np;
  h->seq_bnd = nb;
  return FF_OK;
}

// One chunk of a sequence: frames [0, c) of the arrays, all de-duplicated in
// one set of cooperative launches, then inserted and finalised frame after
// frame on the device (each finalisation hands the next frame its branch count
// and leaf base, or halts it), one read-back of every frame's counters, and
// the host's bookkeeping frame by frame.  done: frames finished (a frame
// halted by an earlier one that grew the volume is not; the caller runs it
// again).
static ff_status sequence_chunk(ff_handle *h, int c, const uint16_t *const *d_depth, const uint8_t *const *d_bgr,
                                int W, int H, const double *K, const double *R, const double *t, float scaling,
                                float maxcam, int32_t *queued, int &done) {
  done = 0;
  cudaStream_t s = h->stream;
  FCK(ensure_seq(h, W, H, c));
  const size_t pix = (size_t)W * H;
  std::vector<FramePlan> plan(c);
  std::vector<MapFrame> mf(c);
  const uint32_t frame0 = h->frames;
  for (int k = 0; k < c; k++) {
    h->cur_slot = h->upd_pending + k;
    h->d_cnt = h->d_seq_cnt + k;
    h->h_cnt = h->h_seq_cnt + k;
    h->cnn_on_side = true;
    const ff_status sp = frame_prepare(h, d_depth[k], d_bgr[k], W, H, K + 4 * k, R + 9 * k, t + 3 * k, scaling,
                                       maxcam, mf[k], plan[k]);
    h->cnn_on_side = false;
    FCK(sp);
    MapFrame &F = mf[k];
    F.vox = h->d_seq_vox + (size_t)k * h->seq_pix;
    F.proc = h->d_seq_proc + (size_t)k * h->seq_pix;
    F.bnd = h->d_seq_bnd + (size_t)k * h->seq_bnd;
    F.cnt = h->d_seq_cnt + k;
    F.frame = frame0 + 1 + (uint32_t)k;
    F.chain = k > 0 ? 1u : 0u;
    F.next_cnt = k + 1 < c ? h->d_seq_cnt + k + 1 : nullptr;
    h->h_batch->f[k] = F;
  }
  LaunchPlan lp;
  FCK(frame_plan(h, c, lp));
  FCK(frame_issue(h, c, lp, false));
  const int block = h->tune.insert_block > 0 ? h->tune.insert_block : 256;
  std::vector<int> pi_ins(c, -1);
  // The chain's kernels follow one another directly on the stream: each is
  // launched as a programmatic dependent of the one before, so that its
  // launch overlaps that kernel (not with the stage profile's events between
  // them, nor for the first insert, which follows the de-duplication).
  const bool pdl = !h->prof.on;
  for (int k = 0; k < c; k++) {
    int pi = h->prof.begin(ST_INSERT, s);
    pi_ins[k] = pi;
    launch_insert(h->d_batch, (uint32_t)(h->h_batch->pix_end[k] - (k ? h->h_batch->pix_end[k - 1] : 0u)), s, block,
                  k, k + 1, pdl && k > 0);
    h->prof.end(pi, 0.0, s);
    pi = h->prof.begin(ST_FINALIZE, s);
    if (!launch_finalize_small(h->d_batch, 1, (uint32_t)pix, h->cfg.device, s, k, pdl))
      return set_err(h, FF_ERR_CUDA, "leaf finalisation could not be launched");
    h->prof.end(pi, 0.0, s);
  }
  // the parents of every frame's new leaves, once the chain has run
  launch_parents_frames(h->d_batch, c, s, 0, pdl);
  CK(cudaGetLastError());
  if (h->cnn_pending) {
    // the frames' confidence networks report into their counters
    CK(cudaStreamWaitEvent(s, h->ev_cnn_done, 0));
    h->cnn_pending = false;
  }
  CK(cudaMemcpyAsync(h->h_seq_cnt, h->d_seq_cnt, sizeof(Counters) * c, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  h->seq_images = true;
  ff_status st = FF_OK;
  for (int k = 0; k < c; k++) {
    if (h->h_seq_cnt[k].error & ERR_SEQ_HALT) break;
    h->cur_slot = h->upd_pending;
    h->d_cnt = h->d_seq_cnt + k;
    h->h_cnt = h->h_seq_cnt + k;
    plan[k].leaves_before = h->leaves_used;
    plan[k].frame = h->frames + 1;
    plan[k].counters_early = false;  // read after the finalisation: the new leaves are counted
    h->pi_insert = pi_ins[k];        // (its bytes follow from the frame's counters)
    st = frame_finish(h, plan[k], mf[k], -1, -1, queued ? queued + k : nullptr);
    if (st != FF_OK) break;
    done++;
  }
  h->seq_images = false;
  h->pi_insert = -1;
  // the next chunk's counters start clean of this one's halts
  CK(cudaMemsetAsync(h->d_seq_cnt, 0, sizeof(Counters) * c, s));
  return st;
}

ff_status ff_add_map_sequence_u16_device(ff_handle *h, int n, const uint16_t *const *d_depth,
                                         const uint8_t *const *d_bgr, int width, int height, const double *K,
                                         const double *R, const double *t, float scaling, float maxcam,
                                         int32_t *queued) {
  if (!h) return FF_ERR_BAD_ARG;
  if (n < 1 || !d_depth || !d_bgr || !K || !R || !t || width <= 0 || height <= 0)
    return set_err(h, FF_ERR_BAD_ARG, "ff_add_map_sequence_u16_device: bad argument");
  for (int k = 0; k < n; k++)
    if (!d_depth[k] || !d_bgr[k]) return set_err(h, FF_ERR_BAD_ARG, "ff_add_map_sequence_u16_device: NULL image");
  h->cur_slot = -1;
  CK(cudaSetDevice(h->cfg.device));
  if (!deferrable(h, width, height) || n == 1) {
    // frames the one-block finalisation does not take (or deferral is off):
    // one by one
    for (int k = 0; k < n; k++)
      FCK(ff_add_map_u16_device(h, d_depth[k], d_bgr[k], width, height, K + 4 * k, R + 9 * k, t + 3 * k, scaling,
                                maxcam, queued ? queued + k : nullptr));
    return FF_OK;
  }
  FCK(ensure_image(h, width, height));
  FCK(ensure_ring(h, width, height));
  // the single-map frames before: their placement and marking done, their
  // buffers free
  CK(join_fuse(h));
  CK(cudaStreamSynchronize(h->stream));
  h->fin_pending = false;
  select_set(h, 0);
  ff_status st = FF_OK;
  for (int i = 0; i < n && st == FF_OK;) {
    const int c = std::min(n - i, std::min(BATCH_MAX, h->upd_batch));
    if (h->upd_pending + c > h->upd_batch) {
      st = flush_updates(h);
      if (st != FF_OK) break;
    }
    int done = 0;
    st = sequence_chunk(h, c, d_depth + i, d_bgr + i, width, height, K + 4 * i, R + 9 * i, t + 3 * i, scaling,
                        maxcam, queued ? queued + i : nullptr, done);
    i += done;
  }
  // the sequence's frames are read where the caller keeps them: their update
  // runs before the call returns
  const ff_status st2 = flush_updates(h);
  if (st == FF_OK) st = st2;
  if (cudaEventSynchronize(h->ev_ring_free) != cudaSuccess && st == FF_OK)
    st = set_err(h, FF_ERR_CUDA, "the sequence's voxel update failed");
  select_set(h, (int)(h->frames & 1u));
  h->cur_slot = -1;
  return st;
}

ff_status ff_add_map_sequence_u16(ff_handle *h, int n, const uint16_t *const *depth, const uint8_t *const *bgr,
                                  int width, int height, size_t depth_pitch, size_t bgr_pitch, const double *K,
                                  const double *R, const double *t, float scaling, float maxcam,
                                  int32_t *queued) {
  if (!h) return FF_ERR_BAD_ARG;
  if (n < 1 || !depth || !bgr || !K || !R || !t || width <= 0 || height <= 0)
    return set_err(h, FF_ERR_BAD_ARG, "ff_add_map_sequence_u16: bad argument");
  for (int k = 0; k < n; k++)
    if (!depth[k] || !bgr[k]) return set_err(h, FF_ERR_BAD_ARG, "ff_add_map_sequence_u16: NULL image");
  CK(cudaSetDevice(h->cfg.device));
  if (!deferrable(h, width, height) || n == 1) {
    for (int k = 0; k < n; k++)
      FCK(ff_add_map_u16(h, depth[k], width, height, depth_pitch, bgr[k], bgr_pitch, K + 4 * k, R + 9 * k,
                         t + 3 * k, scaling, maxcam, queued ? queued + k : nullptr));
    return FF_OK;
  }
  if (!depth_pitch) depth_pitch = sizeof(uint16_t) * width;
  if (!bgr_pitch) bgr_pitch = 3 * (size_t)width;
  const size_t npix = (size_t)width * height;
  const size_t frames = (size_t)std::min(n, BATCH_MAX);
  if (frames > h->hseq_frames || npix > h->hseq_pix) {
    cudaFree(h->d_hseq_depth);
    cudaFree(h->d_hseq_bgr);
    h->d_hseq_depth = nullptr;
    h->d_hseq_bgr = nullptr;
    h->hseq_frames = h->hseq_pix = 0;
    CK(alloc(&h->d_hseq_depth, frames * npix));
    CK(alloc(&h->d_hseq_bgr, frames * npix * 3));
    h->hseq_frames = frames;
    h->hseq_pix = npix;
  }
  std::vector<const uint16_t *> dd(frames);
  std::vector<const uint8_t *> db(frames);
  ff_status st = FF_OK;
  for (int i = 0; i < n && st == FF_OK;) {
    const int c = std::min(n - i, (int)frames);
    // On the copy stream: the depth images first (the de-duplication reads
    // them: the map's stream waits for these copies only, which meanwhile
    // overlap the map's earlier work, the last mesh update say), then the
    // colour images, overlapping the allocation (the update pass waits for
    // them).  The staging is free: the previous group's call returned after
    // its update pass.
    for (int k = 0; k < c; k++) {
      uint16_t *d = h->d_hseq_depth + (size_t)k * npix;
      CK(cudaMemcpy2DAsync(d, sizeof(uint16_t) * width, depth[i + k], depth_pitch, sizeof(uint16_t) * width, height,
                           cudaMemcpyHostToDevice, h->copy_stream));
      dd[k] = d;
    }
    CK(cudaEventRecord(h->ev_host_depth, h->copy_stream));
    CK(cudaStreamWaitEvent(h->stream, h->ev_host_depth, 0));
    for (int k = 0; k < c; k++) {
      uint8_t *b = h->d_hseq_bgr + (size_t)k * npix * 3;
      CK(cudaMemcpy2DAsync(b, 3 * (size_t)width, bgr[i + k], bgr_pitch, 3 * (size_t)width, height,
                           cudaMemcpyHostToDevice, h->copy_stream));
      db[k] = b;
    }
    CK(cudaEventRecord(h->ev_host_images, h->copy_stream));
    h->host_images_pending = true;
    st = ff_add_map_sequence_u16_device(h, c, dd.data(), db.data(), width, height, K + 4 * i, R + 9 * i, t + 3 * i,
                                        scaling, maxcam, queued ? queued + i : nullptr);
    i += c;
  }
  // the caller's images are not read after the call returns, error paths included
  cudaStreamSynchronize(h->copy_stream);
  h->host_images_pending = false;
  return st;
}

ff_status ff_add_maps_u16_device(ff_handle *const *maps, int n, const uint16_t *const *d_depth,
                                 const uint8_t *const *d_bgr, const int *width, const int *height, const double *K,
                                 const double *R, const double *t, const float *scaling, const float *maxcam,
                                 int32_t *queued) {
  if (!maps || n < 1 || !maps[0]) return FF_ERR_BAD_ARG;
  ff_handle *lead = maps[0];
  ff_handle *h = lead;  // (error reporting)
  if (n > BATCH_MAX) return set_err(lead, FF_ERR_BAD_ARG, "ff_add_maps_u16_device: more maps than a batch holds");
  if (!d_depth || !d_bgr || !width || !height || !K || !R || !t || !scaling || !maxcam)
    return set_err(lead, FF_ERR_BAD_ARG, "ff_add_maps_u16_device: NULL array");
  for (int i = 0; i < n; i++) {
    ff_handle *m = maps[i];
    if (!m || !d_depth[i] || !d_bgr[i] || width[i] <= 0 || height[i] <= 0)
      return set_err(lead, FF_ERR_BAD_ARG, "ff_add_maps_u16_device: NULL map or image, or empty image");
    if (m->cfg.device != lead->cfg.device || m->cfg.storage != lead->cfg.storage ||
        (m->d_rcp_tab != nullptr) != (lead->d_rcp_tab != nullptr))
      return set_err(lead, FF_ERR_BAD_ARG, "ff_add_maps_u16_device: maps differ in device, storage or reciprocal mode");
    for (int j = 0; j < i; j++)
      if (maps[j] == m) return set_err(lead, FF_ERR_BAD_ARG, "ff_add_maps_u16_device: a map appears twice");
  }
  CK(cudaSetDevice(lead->cfg.device));
  // frames whose finalisation needs the sort path (very large images) are
  // fused one by one
  uint32_t max_npix = 0;
  bool all_small = true;
  for (int i = 0; i < n; i++) {
    const uint32_t np = (uint32_t)(width[i] * height[i]);
    max_npix = std::max(max_npix, np);
    all_small = all_small && finalize_small_fits(np);
  }
  if (!all_small) {
    for (int i = 0; i < n; i++) {
      ff_status st = ff_add_map_u16_device(maps[i], d_depth[i], d_bgr[i], width[i], height[i], K + 4 * i, R + 9 * i,
                                           t + 3 * i, scaling[i], maxcam[i], queued ? queued + i : nullptr);
      if (st != FF_OK) return st;
    }
    return FF_OK;
  }
  std::vector<FramePlan> plan(n);
  std::vector<MapFrame> mf(n);
  for (int i = 0; i < n; i++) {
    ff_handle *m = maps[i];
    // single-map frames waiting for their update, or still in flight
    {
      const ff_status st_ = settle(m);
      if (st_ != FF_OK) return set_err(lead, st_, m->err);
    }
    m->cur_slot = -1;
    CK(cudaStreamSynchronize(m->stream));
    ff_status st = ensure_image(m, width[i], height[i]);
    if (st != FF_OK) return st;
    st = frame_prepare(m, d_depth[i], d_bgr[i], width[i], height[i], K + 4 * i, R + 9 * i, t + 3 * i, scaling[i],
                       maxcam[i], mf[i], plan[i]);
    if (st != FF_OK) return st;
  }
  // the counter resets went out on each map's stream; the batch runs on the lead's
  for (int i = 1; i < n; i++) CK(cudaStreamSynchronize(maps[i]->stream));
  for (int i = 0; i < n; i++) lead->h_batch->f[i] = mf[i];
  LaunchPlan lp;
  ff_status st = frame_plan(lead, n, lp);
  if (st != FF_OK) return st;
  int pi_fin = -1, pi_fuse = -1;
  // the device work of the batch: upload, de-duplication, insert,
  // finalisation, gated update, every map's counters back to the host
  auto issue = [&]() -> ff_status {
    ff_status r = frame_issue(lead, n, lp);
    if (r == FF_OK) r = frame_launch_update(lead, n, max_npix, pi_fin, pi_fuse);
    for (int i = 0; i < n && r == FF_OK; i++)
      if (cudaMemcpyAsync(maps[i]->h_cnt, maps[i]->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost,
                          lead->stream) != cudaSuccess)
        r = set_err(lead, FF_ERR_CUDA, "counter copy");
    return r;
  };
  bool use_graph = lead->tune.graph && !lead->prof.on && !lead->graph_failed;
  if (use_graph) {
    // the graph's nodes hold the handles' buffers, the launch shapes and the
    // pixel counts; the descriptor itself is copied from h_batch at replay
    std::vector<uint64_t> key = {(uint64_t)n, (uint64_t)lp.rows, (uint64_t)lp.pix, (uint64_t)max_npix,
                                 (uint64_t)lead->tune.fuse_shape, (uint64_t)lead->tune.fuse_blocks_per_sm,
                                 (uint64_t)lead->tune.insert_block, (uint64_t)(uintptr_t)lead->stream};
    for (int i = 0; i < n; i++) {
      key.push_back((uint64_t)(uintptr_t)maps[i] ^ (uint64_t)maps[i]->set);  // (its buffer set)
      key.push_back(((uint64_t)width[i] << 32) | (uint32_t)height[i]);
    }
    if (!lead->graph_exec || key != lead->graph_key) {
      if (lead->graph_exec) cudaGraphExecDestroy(lead->graph_exec);
      lead->graph_exec = nullptr;
      lead->graph_key.clear();
      if (!finalize_small_prepare(lead->cfg.device))  // (function attributes are set outside the capture)
        return set_err(lead, FF_ERR_CUDA, "leaf finalisation could not be prepared");
      const unsigned long long before = g_own_launches.load();
      CK(cudaStreamBeginCapture(lead->stream, cudaStreamCaptureModeThreadLocal));
      st = issue();
      cudaGraph_t g = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(lead->stream, &g);
      cudaGraphExec_t ex = nullptr;
      if (st != FF_OK || ec != cudaSuccess || !g || cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) {
        // launches that cannot be recorded here: launch them directly from now on
        cudaGetLastError();
        g_own_launches.store(before);
        lead->graph_failed = true;
        use_graph = false;
      } else {
        lead->graph_exec = ex;
        lead->graph_key = key;
        lead->graph_launches = g_own_launches.load() - before;
        g_own_launches.fetch_sub(lead->graph_launches);  // counted when the graph runs
      }
      if (g) cudaGraphDestroy(g);
    }
    if (use_graph) {
      note_launch((unsigned)lead->graph_launches);
      CK(cudaGraphLaunch(lead->graph_exec, lead->stream));
      lead->graph_replays++;
    }
  }
  if (!use_graph) {
    st = issue();
    if (st != FF_OK) return st;
  }
  CK(cudaStreamSynchronize(lead->stream));
  double bricks = 0, pending = 0;
  // every map's frame is finished, also after another map's failure (each
  // map's own state must match what ran on the device); the first failure is
  // reported
  ff_status first = FF_OK;
  std::string first_err;
  for (int i = 0; i < n; i++) {
    st = frame_finish(maps[i], plan[i], mf[i], i == 0 ? pi_fin : -1, i == 0 ? pi_fuse : -1,
                      queued ? queued + i : nullptr);
    if (st != FF_OK && first == FF_OK) {
      first = st;
      first_err = "map " + std::to_string(i) + ": " + maps[i]->err;
    }
    bricks += maps[i]->queued;
    pending += maps[i]->new_leaves;
  }
  // the lead's profile holds the batch's launches: count every map's work
  const double brick_bytes = 512.0 * 2 * ((lead->cfg.storage == FF_STORAGE_FP16 ? 4 : 8) + 6);
  lead->prof.set_bytes(pi_fuse, bricks * brick_bytes);
  lead->prof.set_bytes(pi_fin, pending * 8);
  double levels = 0;
  for (int i = 0; i < n; i++) levels += maps[i]->h_cnt->levels;
  if (lead->pi_insert >= 0) lead->prof.set_bytes(lead->pi_insert, 16.0 * levels);
  if (first != FF_OK) {
    lead->barrier_dirty = true;  // (the batch ran on the lead's barrier words)
    return set_err(lead, first, first_err);
  }
  return FF_OK;
}

ff_status ff_get_stats(ff_handle *h, ff_stats *o) {
  if (!h || !o) return FF_ERR_BAD_ARG;
  memset(o, 0, sizeof(*o));
  o->n = h->n;
  for (int r = 0; r < 3; r++) o->offset[r] = h->offset[r];
  o->leaves_used = h->leaves_used;
  o->leaves_max = h->cfg.leaves_max;
  o->branches_used = h->branches_used;
  o->branches_max = h->cfg.branches_max;
  o->queued = h->queued;
  o->frames = h->frames;
  o->meshing_ok = h->meshing_ok ? 1 : 0;
  o->grows = h->grows;
  o->mesh_vertices = h->mesh.n_vertices;
  o->mesh_faces = h->mesh.n_faces;
  o->mesh_cells = h->mesh.n_cells;
  o->mesh_cells_dirty = h->mesh.n_dirty;
  o->processed_pixels = h->processed;
  o->new_leaves = h->new_leaves;
  o->dedupe_rounds = h->dedupe_rounds;
  o->graph_replays = h->graph_replays;
  o->update_batch = (uint32_t)h->upd_batch;
  o->fused_bricks = *h->h_upd_total + h->direct_bricks;
  o->fused_frame_bricks = h->fused_frame_bricks;
  o->mesh_cells_generated = h->mesh.n_generated;
  o->mesh_top_kept = h->mesh.top_kept ? 1u : 0u;
  return FF_OK;
}

ff_status ff_get_leaves(ff_handle *h, uint16_t *pos, uint16_t *scale, uint32_t *parent) {
  if (!h || !pos || !scale || !parent) return FF_ERR_BAD_ARG;
  CK(cudaSetDevice(h->cfg.device));
  CK(join_fuse(h));
  uint32_t n = std::min(h->leaves_used, h->cfg.leaves_max);
  std::vector<ushort4> tmp(n);
  if (n) {
    CK(cudaMemcpyAsync(tmp.data(), h->d_leaf, sizeof(ushort4) * n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(parent, h->d_parent, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  for (uint32_t i = 0; i < n; i++) {
    pos[3 * i] = tmp[i].x;
    pos[3 * i + 1] = tmp[i].y;
    pos[3 * i + 2] = tmp[i].z;
    scale[i] = tmp[i].w;
  }
  return FF_OK;
}

ff_status ff_get_queue(ff_handle *h, uint32_t *leaves) {
  if (!h || !leaves) return FF_ERR_BAD_ARG;
  CK(cudaSetDevice(h->cfg.device));
  CK(join_fuse(h));
  const uint32_t *q = h->d_queue_last ? h->d_queue_last : h->d_queue;
  if (h->queued) CK(cudaMemcpyAsync(leaves, q, sizeof(uint32_t) * h->queued, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return FF_OK;
}

ff_status ff_get_tree(ff_handle *h, uint32_t *tree) {
  if (!h || !tree) return FF_ERR_BAD_ARG;
  CK(cudaSetDevice(h->cfg.device));
  CK(join_fuse(h));
  CK(cudaMemcpyAsync(tree, h->d_tree, sizeof(uint32_t) * h->branches_used, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return FF_OK;
}

ff_status ff_get_bricks(ff_handle *h, uint32_t first, uint32_t count, float *sdf, float *weight, uint16_t *rgb) {
  if (!h || !sdf || !weight || !rgb) return FF_ERR_BAD_ARG;
  if ((uint64_t)first + count > h->cfg.leaves_max) return set_err(h, FF_ERR_BAD_ARG, "ff_get_bricks: range");
  CK(cudaSetDevice(h->cfg.device));
  FCK(settle(h));
  size_t nv = (size_t)count * 512;
  if (h->cfg.storage == FF_STORAGE_FP16) {
    std::vector<__half> a(nv), b(nv);
    CK(cudaMemcpyAsync(a.data(), h->d_sdf16 + (size_t)first * 512, 2 * nv, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(b.data(), h->d_wgt16 + (size_t)first * 512, 2 * nv, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (size_t i = 0; i < nv; i++) {
      sdf[i] = __half2float(a[i]);
      weight[i] = __half2float(b[i]);
    }
  } else {
    CK(cudaMemcpyAsync(sdf, h->d_sdf + (size_t)first * 512, 4 * nv, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(weight, h->d_wgt + (size_t)first * 512, 4 * nv, cudaMemcpyDeviceToHost, h->stream));
  }
  std::vector<uint16_t> planes(nv * 3);
  CK(cudaMemcpyAsync(planes.data(), h->d_col + (size_t)first * 1536, 2 * nv * 3, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (size_t b = 0; b < count; b++)
    for (int c = 0; c < 3; c++)
      for (int v = 0; v < 512; v++) rgb[(b * 512 + v) * 3 + c] = planes[b * 1536 + c * 512 + v];
  return FF_OK;
}

ff_status ff_set_bricks(ff_handle *h, uint32_t first, uint32_t count, const float *sdf, const float *weight,
                        const uint16_t *rgb) {
  if (!h || !sdf || !weight || !rgb) return FF_ERR_BAD_ARG;
  if ((uint64_t)first + count > h->cfg.leaves_max) return set_err(h, FF_ERR_BAD_ARG, "ff_set_bricks: range");
  CK(cudaSetDevice(h->cfg.device));
  FCK(settle(h));
  size_t nv = (size_t)count * 512;
  if (h->cfg.storage == FF_STORAGE_FP16) {
    std::vector<__half> a(nv), b(nv);
    for (size_t i = 0; i < nv; i++) {
      a[i] = __float2half_rn(sdf[i]);
      b[i] = __float2half_rn(weight[i]);
    }
    CK(cudaMemcpyAsync(h->d_sdf16 + (size_t)first * 512, a.data(), 2 * nv, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_wgt16 + (size_t)first * 512, b.data(), 2 * nv, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  } else {
    CK(cudaMemcpyAsync(h->d_sdf + (size_t)first * 512, sdf, 4 * nv, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_wgt + (size_t)first * 512, weight, 4 * nv, cudaMemcpyHostToDevice, h->stream));
  }
  std::vector<uint16_t> planes(nv * 3);
  for (size_t b = 0; b < count; b++)
    for (int c = 0; c < 3; c++)
      for (int v = 0; v < 512; v++) planes[b * 1536 + c * 512 + v] = rgb[(b * 512 + v) * 3 + c];
  CK(cudaMemcpyAsync(h->d_col + (size_t)first * 1536, planes.data(), 2 * nv * 3, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  mesh_invalidate(h->mesh);
  return FF_OK;
}

ff_status ff_set_state(ff_handle *h, uint32_t n, const float offset[3], const uint32_t *tree, uint32_t branches_used,
                       const uint16_t *pos, const uint16_t *scale, const uint32_t *parent, uint32_t leaves_used,
                       const float *sdf, const float *weight, const uint16_t *rgb) {
  if (!h || !offset || !tree || !pos || !scale || !parent) return FF_ERR_BAD_ARG;
  if (branches_used > h->cfg.branches_max || leaves_used > h->cfg.leaves_max || (branches_used & 15))
    return set_err(h, FF_ERR_BAD_ARG, "ff_set_state: state larger than this map's capacity");
  CK(cudaSetDevice(h->cfg.device));
  FCK(settle(h));
  launch_fill(h->d_tree, h->cfg.branches_max, BRANCHINIT, h->stream);
  CK(cudaMemcpyAsync(h->d_tree, tree, sizeof(uint32_t) * branches_used, cudaMemcpyHostToDevice, h->stream));
  std::vector<ushort4> lp(leaves_used);
  for (uint32_t i = 0; i < leaves_used; i++) lp[i] = make_ushort4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], scale[i]);
  if (leaves_used) {
    CK(cudaMemcpyAsync(h->d_leaf, lp.data(), sizeof(ushort4) * leaves_used, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_parent, parent, sizeof(uint32_t) * leaves_used, cudaMemcpyHostToDevice, h->stream));
  }
  CK(cudaStreamSynchronize(h->stream));
  h->n = n;
  for (int r = 0; r < 3; r++) h->offset[r] = offset[r];
  h->branches_used = branches_used;
  h->leaves_used = leaves_used;
  if (sdf && weight && rgb && leaves_used) {
    ff_status st = ff_set_bricks(h, 0, leaves_used, sdf, weight, rgb);
    if (st != FF_OK) return st;
  }
  mesh_invalidate(h->mesh);
  return FF_OK;
}

// ------------------------------------------------------------- meshing ----

ff_status ff_update_meshes(ff_handle *h, int *updated) {
  if (!h) return FF_ERR_BAD_ARG;
  CK(cudaSetDevice(h->cfg.device));
  FCK(settle(h));
  if (!h->meshing_ok || !h->n) {
    if (updated) *updated = 1;
    return FF_OK;
  }
  // the buffers this update writes (or frees as they grow) only after the
  // asynchronous copies that read them; a copy of the last mesh, which this
  // update only reads, goes on meanwhile
  {
    const void *next[3];
    mesh_next_outputs(h->mesh, &next[0], &next[1], &next[2]);
    for (auto &c : h->mesh_copy) {
      if (!c.pending) continue;
      bool hit = false;
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) hit |= c.src[a] && c.src[a] == next[b];
      if (hit) CK(cudaStreamWaitEvent(h->stream, c.ev, 0));
    }
  }
  MeshInputs in;
  in.tree = h->d_tree;
  in.branches_used = h->branches_used;
  in.leaf = h->d_leaf;
  in.parent = h->d_parent;
  in.sdf = h->d_sdf;
  in.wgt = h->d_wgt;
  in.sdf16 = h->d_sdf16;
  in.wgt16 = h->d_wgt16;
  in.col = h->d_col;
  in.storage = h->cfg.storage;
  in.leaves_used = std::min(h->leaves_used, h->cfg.leaves_max);
  in.leaves_max = h->cfg.leaves_max;
  in.stamp = h->d_stamp;
  in.bstamp = h->d_bstamp;
  in.grows = h->grows;
  in.full_cells = h->full_cells;
  in.top_changed = h->top_changed;
  in.spin_limit = h->spin_limit;
  in.frame = h->frames;
  in.n = h->n;
  for (int r = 0; r < 3; r++) in.offset[r] = h->offset[r];
  in.scale = h->cfg.scale;
  in.cnt = h->d_cnt;
  in.h_cnt = h->h_cnt;
  in.prof = &h->prof;
  in.shard = h->shard;
  in.shards = h->shards;
  for (int r = 0; r < 3; r++) in.shift[r] = h->shift[r];
  std::string err;
  int rc = mesh_update(h->mesh, in, h->stream, err);
  if (rc != 0) return set_err(h, (ff_status)rc, err);
  h->top_changed = false;
  if (updated) *updated = 1;
  return FF_OK;
}

ff_status ff_kernel_launches(uint64_t *own, uint64_t *library) {
  if (!own || !library) return FF_ERR_BAD_ARG;
  *own = g_own_launches.load();
  *library = g_lib_calls.load();
  return FF_OK;
}

ff_status ff_profile(ff_handle *h, int enable) {
  if (!h) return FF_ERR_BAD_ARG;
  CK(cudaSetDevice(h->cfg.device));
  h->prof.reset();
  h->prof.on = enable != 0;
  return FF_OK;
}

ff_status ff_profile_read(ff_handle *h, double *ms, double *bytes, uint64_t *launches) {
  if (!h || !ms || !bytes || !launches) return FF_ERR_BAD_ARG;
  CK(cudaSetDevice(h->cfg.device));
  FCK(settle(h));
  CK(cudaStreamSynchronize(h->fuse_stream));
  h->prof.flush();
  for (int i = 0; i < FF_PROFILE_STAGES; i++) {
    ms[i] = h->prof.ms[i];
    bytes[i] = h->prof.bytes[i];
    launches[i] = h->prof.launches[i];
  }
  return FF_OK;
}

ff_status ff_get_mesh_counts(ff_handle *h, uint64_t *nv, uint64_t *nf) {
  if (!h || !nv || !nf) return FF_ERR_BAD_ARG;
  *nv = h->mesh.n_vertices;
  *nf = h->mesh.n_faces;
  return FF_OK;
}

ff_status ff_get_mesh(ff_handle *h, float *xyz, uint8_t *rgb, uint32_t *faces) {
  if (!h) return FF_ERR_BAD_ARG;
  if ((h->mesh.n_vertices && (!xyz || !rgb)) || (h->mesh.n_faces && !faces))
    return set_err(h, FF_ERR_BAD_ARG, "ff_get_mesh: NULL output buffer");
  CK(cudaSetDevice(h->cfg.device));
  std::string err;
  int rc = mesh_copy_out(h->mesh, xyz, rgb, faces, h->stream, err);
  if (rc != 0) return set_err(h, (ff_status)rc, err);
  return FF_OK;
}

ff_status ff_get_mesh_async(ff_handle *h, float *xyz, uint8_t *rgb, uint32_t *faces) {
  if (!h) return FF_ERR_BAD_ARG;
  const MeshState &M = h->mesh;
  if ((M.n_vertices && (!xyz || !rgb)) || (M.n_faces && !faces))
    return set_err(h, FF_ERR_BAD_ARG, "ff_get_mesh_async: NULL output buffer");
  CK(cudaSetDevice(h->cfg.device));
  // behind the update's device work (its emit pass may still run)
  CK(cudaEventRecord(h->ev_mesh_ready, h->stream));
  CK(cudaStreamWaitEvent(h->mesh_stream, h->ev_mesh_ready, 0));
  if (M.n_vertices) {
    CK(cudaMemcpyAsync(xyz, M.d_xyz, sizeof(float) * 3 * M.n_vertices, cudaMemcpyDeviceToHost, h->mesh_stream));
    CK(cudaMemcpyAsync(rgb, M.d_rgb, 3 * M.n_vertices, cudaMemcpyDeviceToHost, h->mesh_stream));
  }
  if (M.n_faces)
    CK(cudaMemcpyAsync(faces, M.d_faces, sizeof(uint32_t) * 3 * M.n_faces, cudaMemcpyDeviceToHost, h->mesh_stream));
  auto &c = h->mesh_copy[h->mesh_copy_next];
  h->mesh_copy_next ^= 1;
  CK(cudaEventRecord(c.ev, h->mesh_stream));
  c.src[0] = M.d_xyz;
  c.src[1] = M.d_rgb;
  c.src[2] = M.d_faces;
  c.pending = true;
  return FF_OK;
}

ff_status ff_mesh_wait(ff_handle *h) {
  if (!h) return FF_ERR_BAD_ARG;
  CK(cudaSetDevice(h->cfg.device));
  for (auto &c : h->mesh_copy)
    if (c.pending) {
      CK(cudaEventSynchronize(c.ev));
      c.pending = false;
    }
  return FF_OK;
}

ff_status ff_alloc_host(size_t bytes, void **out) {
  if (!out) return FF_ERR_BAD_ARG;
  *out = nullptr;
  if (!bytes) return FF_OK;
  if (cudaHostAlloc(out, bytes, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    *out = nullptr;
    return FF_ERR_CUDA;
  }
  return FF_OK;
}

ff_status ff_free_host(void *p) {
  if (p && cudaFreeHost(p) != cudaSuccess) {
    cudaGetLastError();
    return FF_ERR_CUDA;
  }
  return FF_OK;
}

ff_status ff_get_mesh_cells(ff_handle *h, int32_t *cells, int64_t *ranges) {
  if (!h || (h->mesh.n_cells && (!cells || !ranges))) return FF_ERR_BAD_ARG;
  CK(cudaSetDevice(h->cfg.device));
  std::string err;
  int rc = mesh_copy_cells(h->mesh, cells, ranges, h->stream, err);
  if (rc != 0) return set_err(h, (ff_status)rc, err);
  return FF_OK;
}

ff_status ff_get_mesh_cells_noalloc(ff_handle *h, int32_t *cells, int64_t *ranges) {
  if (!h || (h->mesh.n_cells && (!cells || !ranges))) return FF_ERR_BAD_ARG;
  CK(cudaSetDevice(h->cfg.device));
  std::string err;
  int rc = mesh_copy_cells_noalloc(h->mesh, cells, ranges, h->stream, err);
  if (rc != 0) return set_err(h, (ff_status)rc, err);
  return FF_OK;
}

ff_status ff_get_mesh_device(ff_handle *h, const float **xyz, const uint8_t **rgb, const uint32_t **faces) {
  if (!h || !xyz || !rgb || !faces) return FF_ERR_BAD_ARG;
  *xyz = h->mesh.d_xyz;
  *rgb = h->mesh.d_rgb;
  *faces = h->mesh.d_faces;
  return FF_OK;
}

}  // extern "C"

// ------------------------------------------------- learned confidence weight

// FP32 -> BF16, round to nearest even (NaN kept quiet).
static uint16_t bf16_bits(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7F800000u) == 0x7F800000u && (u & 0x007FFFFFu)) return (uint16_t)((u >> 16) | 0x0040u);
  const uint32_t lsb = (u >> 16) & 1u;
  u += 0x7FFFu + lsb;
  return (uint16_t)(u >> 16);
}

ff_status ff_set_confidence(ff_handle *h, const float *params, int n_params, float tau_m) {
  if (!h) return FF_ERR_BAD_ARG;
  if (!params) {
    h->conf_tau_cm = 0.0f;
    return FF_OK;
  }
  if (n_params != FF_CNN_PARAMS || !(tau_m > 0.0f) || !std::isfinite(tau_m))
    return set_err(h, FF_ERR_BAD_ARG, "ff_set_confidence: expected FF_CNN_PARAMS parameters and tau > 0");
  for (int i = 0; i < n_params; i++)
    if (!std::isfinite(params[i])) return set_err(h, FF_ERR_BAD_ARG, "ff_set_confidence: non-finite parameter");
  CK(cudaSetDevice(h->cfg.device));
  std::vector<uint16_t> b(n_params);
  for (int i = 0; i < n_params; i++) b[i] = bf16_bits(params[i]);
  if (!h->d_cnn_params) CK(alloc(&h->d_cnn_params, (size_t)FF_CNN_PARAMS));
  if (!h->d_cnn_packed) CK(alloc(&h->d_cnn_packed, (size_t)CNN_PACKED_BYTES));
  h->cnn_packed_ready = false;  // packed by the next frame
  CK(cudaMemcpyAsync(h->d_cnn_params, b.data(), sizeof(uint16_t) * n_params, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->conf_tau_cm = tau_m * 100.0f;
  return FF_OK;
}

ff_status ff_get_confidence_map(ff_handle *h, float *out, int *width, int *height) {
  if (!h) return FF_ERR_BAD_ARG;
  if (!(h->conf_tau_cm > 0.0f) || !h->d_conf || !h->conf_w)
    return set_err(h, FF_ERR_BAD_ARG, "ff_get_confidence_map: no learned weight or no frame yet");
  if (width) *width = h->conf_w;
  if (height) *height = h->conf_h;
  if (out) {
    CK(cudaSetDevice(h->cfg.device));
    CK(cudaMemcpyAsync(out, h->d_conf, sizeof(float) * (size_t)h->conf_w * h->conf_h, cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  return FF_OK;
}

ff_status ff_raycast_depth(ff_handle *h, const double K[4], const double R[9], const double t[3],
                           const uint16_t *d_depth, int width, int height, float scaling, float window_m,
                           float step_m, float *d_out) {
  if (!h) return FF_ERR_BAD_ARG;
  if (!K || !R || !t || !d_depth || !d_out || width <= 0 || height <= 0)
    return set_err(h, FF_ERR_BAD_ARG, "ff_raycast_depth: NULL pointer or empty image");
  if (!(window_m > 0.0f && window_m <= 4.0f) || !(step_m >= 1e-4f && step_m <= window_m))
    return set_err(h, FF_ERR_BAD_ARG, "ff_raycast_depth: window must be in (0, 4] m and step in [1e-4, window]");
  if (!h->n) return set_err(h, FF_ERR_BAD_ARG, "ff_raycast_depth: the map holds no frame");
  CK(cudaSetDevice(h->cfg.device));
  FCK(settle(h));
  RaycastMap m;
  m.tree = h->d_tree;
  m.leaf = h->d_leaf;
  m.sdf = h->d_sdf;
  m.wgt = h->d_wgt;
  m.sdf16 = h->d_sdf16;
  m.wgt16 = h->d_wgt16;
  m.n = h->n;
  m.leaves_max = std::min(h->leaves_used, h->cfg.leaves_max);  // leaves with storage
  m.fp16 = h->cfg.storage == FF_STORAGE_FP16;
  m.thr = h->cfg.threshold;
  const CamF p = cam_world_to_grid(h, K, R, t);
  CK(launch_raycast(m, p, width, height, d_depth, scaling, window_m, step_m, d_out, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return FF_OK;
}

// Training entry points: device pointers owned by the caller, work on the
// caller's stream; errors are reported through ff_last_error(NULL).
#define CKN(call)                                                                     \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      g_create_error = std::string(#call) + ": " + cudaGetErrorString(e_);            \
      return FF_ERR_CUDA;                                                             \
    }                                                                                 \
  } while (0)

static ff_status cnn_bad(const char *m) {
  g_create_error = m;
  return FF_ERR_BAD_ARG;
}

ff_status ff_cnn_features(const uint16_t *d_depth, int n, int width, int height, float scaling, const double K[4],
                          void *d_feat, void *stream) {
  if (!d_depth || !K || !d_feat || n <= 0 || width <= 0 || height <= 0) return cnn_bad("ff_cnn_features: bad argument");
  const float kf[4] = {(float)K[0], (float)K[1], (float)K[2], (float)K[3]};
  CKN(cnn_features(d_depth, n, width, height, scaling, kf, (__nv_bfloat16 *)d_feat, (cudaStream_t)stream));
  return FF_OK;
}

ff_status ff_cnn_forward(const void *d_params, void *d_packed, const void *d_feat, int n, int width, int height,
                         void *d_a1, void *d_a2, float *d_out, float tau_m, void *stream) {
  if (!d_params || !d_packed || !d_feat || !d_a1 || !d_a2 || !d_out || n <= 0 || width <= 0 || height <= 0)
    return cnn_bad("ff_cnn_forward: bad argument");
  CKN(cnn_forward((const __nv_bfloat16 *)d_params, (uint8_t *)d_packed, false, (const __nv_bfloat16 *)d_feat, n,
                  width, height, (__nv_bfloat16 *)d_a1, (__nv_bfloat16 *)d_a2, d_out,
                  tau_m > 0.0f ? tau_m * 100.0f : 0.0f, nullptr, (cudaStream_t)stream));
  return FF_OK;
}

ff_status ff_cnn_backward(const void *d_params, const void *d_feat, const void *d_a1, const void *d_a2,
                          const float *d_dpred, int n, int width, int height, float *d_g1, float *d_g2,
                          float *d_grads, void *stream) {
  if (!d_params || !d_feat || !d_a1 || !d_a2 || !d_dpred || !d_g1 || !d_g2 || !d_grads || n <= 0 || width <= 0 ||
      height <= 0)
    return cnn_bad("ff_cnn_backward: bad argument");
  CKN(cnn_backward((const __nv_bfloat16 *)d_params, (const __nv_bfloat16 *)d_feat, (const __nv_bfloat16 *)d_a1,
                   (const __nv_bfloat16 *)d_a2, d_dpred, n, width, height, d_g1, d_g2, d_grads,
                   (cudaStream_t)stream));
  return FF_OK;
}

ff_status ff_cnn_mse(const float *d_pred, const float *d_target, int64_t count, float inv_count, float *d_dpred,
                     double *d_loss, void *stream) {
  if (!d_pred || !d_target || !d_dpred || !d_loss || count <= 0) return cnn_bad("ff_cnn_mse: bad argument");
  CKN(cnn_mse(d_pred, d_target, count, inv_count, d_dpred, d_loss, (cudaStream_t)stream));
  return FF_OK;
}

ff_status ff_cnn_adam(float *d_master, void *d_params, float *d_grads, float *d_m, float *d_v, float lr,
                      float beta1, float beta2, float eps, int step, void *stream) {
  if (!d_master || !d_params || !d_grads || !d_m || !d_v || step < 1) return cnn_bad("ff_cnn_adam: bad argument");
  CKN(cnn_adam(d_master, (__nv_bfloat16 *)d_params, d_grads, d_m, d_v, FF_CNN_PARAMS, lr, beta1, beta2, eps, step,
               (cudaStream_t)stream));
  return FF_OK;
}
