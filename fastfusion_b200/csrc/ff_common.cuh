// Shared device-side definitions of the B200 fusion path.
//
// Data layout in HBM (one map):
//   tree      uint32[branches_max]  16 entries per branch: [0..7] leaf index of
//                                   each octant, [8..15] child branch -- the
//                                   reference's _tree (traversal_functions.cpp:308-395)
//   leaf_pos  ushort4[leaves_max]   x, y, z (voxels), scale (voxel spacing)
//   leaf_par  uint32[leaves_max]    parent leaf (_leafParent)
//   sdf, wgt  float[leaves_max][512]   (or __half with FP16 storage)
//   col       uint16[leaves_max][3][512]  R, G, B planes per brick (x256)
// Voxel v of a brick is (z*8 + y)*8 + x, the reference's order.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

namespace ffb {

// Process-wide counts of this library's own kernel launches and of the CUB
// (library) calls it makes, for launch accounting by callers.
extern std::atomic<unsigned long long> g_own_launches, g_lib_calls;
inline void note_launch(unsigned n = 1) { g_own_launches.fetch_add(n, std::memory_order_relaxed); }
inline void note_lib_call() { g_lib_calls.fetch_add(1, std::memory_order_relaxed); }

// Programmatic dependent launch.  A kernel launched by launch_pdl may be
// scheduled while the kernel before it on the stream still runs, so that its
// launch and ramp-up overlap that kernel's tail; it calls pdl_wait() before
// anything else, which returns once the earlier kernel has completed and its
// writes are visible (and at once in a launch without the attribute).
// pdl_trigger() lets the next kernel of the stream be scheduled early.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_enter() {
  pdl_trigger();
  pdl_wait();
}

// Launch kern on s; with pdl, as a programmatic dependent of the stream's
// previous kernel (which must then be a kernel: the kernel launched here
// starts with pdl_enter()).
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(bool pdl, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

constexpr uint32_t BRANCHINIT = 0xFFFFFFFEu;  // reference definitions.h:128
constexpr uint32_t LOCKED = 0xFFFFFFFDu;      // slot being allocated (device-internal)
constexpr uint32_t PENDING = 0xC0000000u;     // slot holds a leaf created this frame: PENDING + record
constexpr int BL = 8;                         // BRICKLENGTH
constexpr float DIST_W_EPS = 0.005f;          // DISTANCEWEIGHTEPSILON
constexpr float WEIGHT_FACTOR = 3.0f;
constexpr float COLOR_MUL = 256.0f;
// default bound of every device-side wait (iterations); a map can set its
// own (ff_set_spin_limit), down to 0: a wait then gives up at once
constexpr uint32_t SPIN_LIMIT = 1u << 22;

// error bits written by kernels into Counters::error
enum : uint32_t {
  ERR_BRANCH_OVERFLOW = 1u,
  ERR_SPIN_TIMEOUT = 2u,
  ERR_PENDING_OVERFLOW = 4u,
  ERR_CELL_OVERFLOW = 8u,
  ERR_MESH_OVERFLOW = 16u,
  ERR_DEDUPE_NOT_CONVERGED = 32u,
  ERR_CELL_KEY = 64u,  // a mesh cell's origin does not fit its sort key
  ERR_DEDUPE_TIMEOUT = 128u,  // a grid barrier of the de-duplication gave up (nothing was inserted)
  ERR_SEQ_HALT = 256u,        // an earlier frame of a sequence must grow the volume or failed: not run
  ERR_CELL_MERGE = 512u,      // the kept and the new mesh cells share a sort key (the update is redone in full)
  ERR_CELL_TIMEOUT = 1024u,   // a grid barrier of the mesh-cell traversal gave up
};

// Error bits after which a frame's voxel update is skipped: its allocation
// did not complete as the reference's would have.
constexpr uint32_t ERR_FRAME_FAILED = ERR_SPIN_TIMEOUT | ERR_DEDUPE_NOT_CONVERGED | ERR_DEDUPE_TIMEOUT |
                                      ERR_PENDING_OVERFLOW | ERR_SEQ_HALT;
// Error bits of the de-duplication: the insert, the leaf finalisation and the
// update leave such a frame out entirely, so the map stays as it was.
constexpr uint32_t ERR_DEDUPE_FAILED = ERR_DEDUPE_NOT_CONVERGED | ERR_DEDUPE_TIMEOUT;

// Per-map counters kept in device memory; read back once per frame.
struct Counters {
  uint32_t branches_used;
  uint32_t pending;        // new leaves claimed this frame
  uint32_t queued;         // bricks queued this frame (existing + new)
  uint32_t processed;      // pixels that passed de-duplication
  int32_t box_min[3];
  int32_t box_max[3];
  uint32_t error;
  uint32_t dedupe_changed;
  uint32_t dedupe_iters;
  uint32_t n_cells;
  uint32_t n_work;
  uint32_t n_work_next;
  uint64_t mesh_v;
  uint64_t mesh_f;
  uint32_t cnn_error;  // the confidence network's bounded waits (kept by the frame's counter set-up)
  uint32_t levels;     // octree levels the insert probed, summed over the processed pixels
  uint32_t leaves_base;  // a sequence's later frame: leaves before it (set by the previous frame's finalisation)
  uint32_t top_created;  // a branch or leaf was created in a slot within MESH_TOP_LEVELS of the root
};

// The mesher keeps the items of its octree traversal's level MESH_TOP_LEVELS
// from one update to the next; a frame that creates a branch or a leaf in a
// slot that close to the root (depth <= MESH_TOP_LEVELS) makes it build them
// again.
constexpr int MESH_TOP_LEVELS = 4;

// Float camera parameters (the reference's camPamsFloat, definitions.h:71-88).
struct CamF {
  float r[9];
  float t[3];
  float fx, fy, cx, cy;
};

// Ownership in a sharded map (ff_set_shard): every part holds the whole
// octree and leaf table (all parts run the same allocation), updates the
// voxels of the bricks it owns and meshes the cells it owns.  Both are a hash
// of the object's origin in units of its edge, in coordinates that grow()
// does not move (shift: the voxels the grid has been moved by), and of its
// edge (and, for a cell, its type).
__device__ __forceinline__ uint32_t shard_hash(int32_t ox, int32_t oy, int32_t oz, uint32_t edge, uint32_t kind,
                                               const int32_t *shift) {
  const int lg = 31 - __clz(edge);
  const uint32_t kx = (uint32_t)((ox - shift[0]) >> lg);
  const uint32_t ky = (uint32_t)((oy - shift[1]) >> lg);
  const uint32_t kz = (uint32_t)((oz - shift[2]) >> lg);
  uint32_t hsh = kx * 73856093u ^ ky * 19349663u ^ kz * 83492791u ^ (uint32_t)lg * 2654435761u ^ kind * 40503u;
  hsh ^= hsh >> 16;
  hsh *= 0x45d9f3bu;
  hsh ^= hsh >> 16;
  return hsh;
}

// Barrier over all blocks of a cooperative launch (every block resident).
// bar[0] counts arrivals, bar[1] is the generation; both start at zero.
// A wait that exceeds `limit` iterations sets err_bit in *err and stops
// waiting.
__device__ __forceinline__ void grid_barrier_bounded(uint32_t *bar, uint32_t nblocks, uint32_t *err, uint32_t err_bit,
                                                     uint32_t limit) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile uint32_t *gen = bar + 1;
    const uint32_t g = *gen;
    __threadfence();
    if (atomicAdd(bar, 1u) == nblocks - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      uint32_t spins = 0;
      while (*gen == g) {
        if (spins++ >= limit) {
          atomicOr(err, err_bit);
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

}  // namespace ffb
