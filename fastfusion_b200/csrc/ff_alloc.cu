// Brick allocation: per-pixel projection, row/column de-duplication and the
// parallel octree insert that replaces the reference's sequential traversal
// (transformLoopSimPrecalculatedNeg_subtree, traversal_wrapper_functions.cpp:576-694,
//  queryPointDepthSingle_func_subtree / addLeaf, traversal_functions.cpp:185-211, 308-395).
//
// The reference walks pixels in raster order; three of its outcomes depend on
// that order and are reproduced exactly here:
//   * which pixels are processed (the de-duplication recurrence) -- computed
//     by an exact tiled fixed-point solve of the recurrence;
//   * leaf indices -- assigned in order of the first pixel that created each
//     leaf (sort of pending leaves by first pixel);
//   * parent leaves -- the finest ancestor leaf that existed when the leaf was
//     created, i.e. the finest ancestor with a smaller index.
// Branch indices are assigned in arrival order; they are internal.
#include <cub/cub.cuh>

#include "ff_kernels.h"
#include "ff_sort.h"

namespace ffb {

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t *p) { return *(volatile const uint32_t *)p; }

// Octree read on the descent, cached in L1.  Safe without coherence: a valid
// leaf index or child pointer never changes while the insert runs (they are
// written once; grow() runs between kernels), so a cached read that returns
// one is exact; a slot another thread claims meanwhile may still read as
// BRANCHINIT here, and the atomicCAS that follows returns its current value.
__device__ __forceinline__ uint32_t ld_tree(const uint32_t *p) { return __ldca(p); }

// ---------------------------------------------------------------- bbox ----

// computeBoundingboxIntCPU(ushort), geometryfusion_mipmap_cpu.cpp:1270-1303,
// round-to-nearest float arithmetic in the reference's operation order.
__global__ void k_first_bbox(const uint16_t *depth, int W, int H, CamF p, float scaling, float maxcam, int bw,
                             Counters *cnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int mn[3] = {1000000, 1000000, 1000000}, mx[3] = {-1000000, -1000000, -1000000};
  if (i < W * H) {
    int x = i % W, y = i / W;
    float pz = __fmul_rn((float)depth[i], scaling);
    if (pz > 0.0f && pz < maxcam) {
      float px = __fmul_rn(__fdiv_rn(__fsub_rn((float)x, p.cx), p.fx), pz);
      float py = __fmul_rn(__fdiv_rn(__fsub_rn((float)y, p.cy), p.fy), pz);
#pragma unroll
      for (int r = 0; r < 3; r++) {
        float s = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(p.r[3 * r], px), __fmul_rn(p.r[3 * r + 1], py)),
                                      __fmul_rn(p.r[3 * r + 2], pz)),
                            p.t[r]);
        int v = __float2int_rz(s);
        mn[r] = v - bw;
        mx[r] = v + bw;
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 3; r++) {
    int a = mn[r], b = mx[r];
    for (int o = 16; o > 0; o >>= 1) {
      a = min(a, __shfl_xor_sync(0xffffffffu, a, o));
      b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&cnt->box_min[r], a);
      atomicMax(&cnt->box_max[r], b);
    }
  }
}

void launch_first_bbox(const uint16_t *depth, int W, int H, const CamF &p, float scaling, float maxcam, int bw,
                       Counters *cnt, cudaStream_t s) {
  int n = W * H;
  note_launch();
  k_first_bbox<<<(n + 255) / 256, 256, 0, s>>>(depth, W, H, p, scaling, maxcam, bw, cnt);
}

// ------------------------------------------------------------- project ----

// Per pixel: v = (int)(((qx[x] + qy[y]) * depth) * scaling + t), the
// reference's key arithmetic (traversal_wrapper_functions.cpp:613-630,
// addMap's qxp/qyp, geometryfusion_mipmap_cpu.cpp:1807-1822), in
// round-to-nearest with no fused multiply-add.  w = target brick edge in
// voxels, floor(max(depth,1)*8) (leafScaleFunc, inline_functions.hpp:128-145),
// or -1 for invalid depth.
// Voxel coordinates of a pixel's surface point and its target brick scale
// (-1: invalid), under the default rounding: ((qxp+qyp)*d)*scaling + t per
// axis, truncated (traversal_wrapper_functions.cpp:613-630), and
// leafScaleFunc's floor(max(z,1)*8) (inline_functions.hpp:128-145).
__device__ __forceinline__ int4 project_point(float d, float px, float py, const CamF &p, float scaling,
                                              float maxcam) {
  int v[3];
#pragma unroll
  for (int r = 0; r < 3; r++) {
    float qx = __fmul_rn(p.r[3 * r + 0], px);
    float qy = __fadd_rn(__fmul_rn(p.r[3 * r + 1], py), p.r[3 * r + 2]);
    float s = __fadd_rn(__fmul_rn(__fmul_rn(__fadd_rn(qx, qy), d), scaling), p.t[r]);
    v[r] = __float2int_rz(s);
  }
  const float ds = __fmul_rn(d, scaling);
  int target = -1;
  if (ds > 0.0f && ds < maxcam) {
    float f = ds < 1.0f ? 1.0f : ds;
    target = (int)(uint16_t)floorf(__fmul_rn(f, 8.0f));
  }
  return make_int4(v[0], v[1], v[2], target);
}

// ------------------------------------------------------------- dedupe -----
//
// The reference processes pixel (x,y) iff its depth is valid and its brick
// key k = v & -8 differs from s(x,y-1) and from s(x-1,y), where
// s = k if processed and -1 otherwise (traversal_wrapper_functions.cpp:636-639,
// 688-690).  This is a recurrence over the two predecessors only, so it has a
// unique solution.  Each warp solves one 32x32 tile exactly, given the state
// of the column to its left and the row above it, rows top to bottom.  The
// key comparisons never change, so they are made once, as bit masks: per lane
// valid(r), up(r) = k(x,r)==k(x,r-1), left(r) = k(x,r)==k(x-1,r).  In a row,
// a(x) = valid && !(p(x,r-1) && up) and p(x) = a(x) && !(p(x-1) && left(x)):
// p copies a(x) at a lane that is not chained to its left neighbour
// (a(x)==0 or left(x)==0) and alternates along a chain, so one ballot of the
// chained lanes and one of the chain starts give the row.  Tiles exchange
// boundary bits and repeat until no boundary changes; a chain of dependencies
// crosses at most tilesX+tilesY tiles, which bounds the number of rounds.

__device__ __forceinline__ void grid_barrier(uint32_t *bar, uint32_t nblocks, Counters *cnt, uint32_t limit) {
  grid_barrier_bounded(bar, nblocks, &cnt->error, ERR_DEDUPE_TIMEOUT, limit);
}

constexpr int DD_WARPS = 4;  // tiles (warps) per block
// tile height: 16 rows (more, shorter tiles shorten each warp's chain of
// rows), or 32 when the image has more 16-row tiles than resident warps
constexpr int DD_ROWS_SHORT = 16, DD_ROWS_TALL = 32;
constexpr int DD_ROWS_LOW = 8;  // more, shorter tiles again (a tuning choice)

__device__ __forceinline__ bool same3(int a0, int a1, int a2, int b0, int b1, int b2) {
  return a0 == b0 && a1 == b1 && a2 == b2;
}

// Tiles are 32 pixels wide and DD_ROWS high.  bnd layout: right-column keys
// [ntiles][32] int4 (DD_ROWS used), bottom-row keys [ntiles][32]
// int4 (written once, before the first barrier), then processed bits of the
// right column and of the bottom row, [2 rounds][ntiles] uint32 each.
// bar: [0] arrivals, [1] generation, [4..6] per-round change counters (rotating)
// One launch for all frames of a batch: warps are dealt out over the maps'
// tiles in order; the rounds and their barrier are shared (a map whose tiles
// have settled recomputes the same bits until every map has).
// Maps [m0, m1) of the batch (their tiles must all be resident at once).
template <int DD_ROWS>
__device__ __forceinline__ void dedupe_body(const BatchDesc *__restrict__ bd, int m0, int m1, uint32_t *bar) {
  const int lane = threadIdx.x & 31;
  const uint32_t base = m0 ? bd->tile_end[m0 - 1] : 0u;
  const uint32_t gtile = base + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  int m = m0;
  while (m < m1 - 1 && gtile >= bd->tile_end[m]) m++;
  const MapFrame &F = bd->f[m];
  const int tile = (int)(gtile - (m ? bd->tile_end[m - 1] : 0u));
  const bool active = gtile < bd->tile_end[m1 - 1];  // warps past the last tile only join the barriers
  const uint16_t *__restrict__ depth = F.depth;
  const float *__restrict__ pxp = F.pxp;
  const float *__restrict__ pyp = F.pyp;
  const CamF cam = F.p;
  const float scaling = F.scaling, maxcam = F.maxcam;
  int4 *vox = F.vox;
  const int W = F.W, H = F.H, tilesX = F.tilesX, tilesY = F.tilesY;
  int4 *bnd = F.bnd;
  uint8_t *processed = F.proc;
  Counters *cnt = F.cnt;
  const int ntiles = tilesX * tilesY;
  int4 *keyR = bnd, *keyB = bnd + (size_t)ntiles * 32;
  uint32_t *pR = reinterpret_cast<uint32_t *>(bnd + (size_t)2 * ntiles * 32);
  uint32_t *pB = pR + 2 * (size_t)ntiles;
  const int tx = active ? tile % tilesX : 0, ty = active ? tile / tilesX : 0;
  const int x = tx * 32 + lane;
  // each map's counters for this frame (read from the first barrier on)
  if (blockIdx.x == 0 && (int)threadIdx.x < m1 - m0) {
    const MapFrame &G = bd->f[m0 + threadIdx.x];
    Counters *c = G.cnt;
    // (not the confidence network's error word, which that network may be
    // setting meanwhile on another stream)
    constexpr int keep = (int)(offsetof(Counters, cnn_error) / 4);
    uint32_t *w = reinterpret_cast<uint32_t *>(c);
    for (int k = 0; k < (int)(sizeof(Counters) / 4); k++)
      if (k != keep) w[k] = 0;
    c->branches_used = G.branches_init;
    for (int r = 0; r < 3; r++) {
      c->box_min[r] = 0;
      c->box_max[r] = (int)G.n - 1;
    }
  }
  const int rows = active ? min(DD_ROWS, H - ty * DD_ROWS) : 0;
  // project the tile (voxel keys for the insert that follows) and make the
  // key comparisons; the tile's depth and row factors are fetched first so
  // the loads overlap
  uint16_t dv[DD_ROWS];
  const bool col_ok = active && x < W;
#pragma unroll
  for (int r = 0; r < DD_ROWS; r++) dv[r] = (col_ok && r < rows) ? __ldg(&depth[(size_t)(ty * DD_ROWS + r) * W + x]) : 0;
  const float px = col_ok ? __ldg(&pxp[x]) : 0.0f;
  const float py_lane = (active && lane < rows) ? __ldg(&pyp[ty * DD_ROWS + lane]) : 0.0f;
  uint32_t valid = 0, up = 0, left = 0;
  int c0 = 0, c1 = 0, c2 = 0;     // key at (lane 0, row = lane): compared with the left tile
  int t0 = 0, t1 = 0, t2 = 0;     // key at (lane, row 0): compared with the tile above
  int u0 = 0, u1 = 0, u2 = 0;     // key of the previous row
#pragma unroll
  for (int r = 0; r < DD_ROWS; r++) {
    if (r >= rows) break;
    const int y = ty * DD_ROWS + r;
    const float py = __shfl_sync(0xffffffffu, py_lane, r);
    int4 v = make_int4(0, 0, 0, -1);
    if (x < W) {
      v = project_point((float)dv[r], px, py, cam, scaling, maxcam);
      vox[(size_t)y * W + x] = v;
    }
    const int k0 = v.x & -8, k1 = v.y & -8, k2 = v.z & -8;
    const int l0 = __shfl_up_sync(0xffffffffu, k0, 1);
    const int l1 = __shfl_up_sync(0xffffffffu, k1, 1);
    const int l2 = __shfl_up_sync(0xffffffffu, k2, 1);
    const int f0 = __shfl_sync(0xffffffffu, k0, 0);
    const int f1 = __shfl_sync(0xffffffffu, k1, 0);
    const int f2 = __shfl_sync(0xffffffffu, k2, 0);
    if (lane == r) c0 = f0, c1 = f1, c2 = f2;
    if (r == 0) t0 = k0, t1 = k1, t2 = k2;
    if (x < W && v.w >= 0) valid |= 1u << r;
    if (r > 0 && same3(k0, k1, k2, u0, u1, u2)) up |= 1u << r;
    if (lane > 0 && same3(k0, k1, k2, l0, l1, l2)) left |= 1u << r;
    u0 = k0, u1 = k1, u2 = k2;
    if (lane == 31) keyR[(size_t)tile * 32 + r] = make_int4(k0, k1, k2, 0);
    if (r == rows - 1) keyB[(size_t)tile * 32 + lane] = make_int4(k0, k1, k2, 0);
  }
  uint32_t eq_left = 0;  // row bits: lane 0's key equals the left tile's right column
  bool eq_above = false;  // this lane's row-0 key equals the above tile's bottom row
  uint32_t bits = 0, last_r = 0, last_b = 0;
  const int max_rounds = bd->max_rounds;
  volatile uint32_t *chg = bar + 4;
  int round = 0;
  bool converged = false;
  for (; round < max_rounds; round++) {
    const int in = round & 1, out = in ^ 1;
    int changed = 0;
    if (active) {
      uint32_t left_p = 0, above_p = 0;
      if (round > 0) {
        if (round == 1) {
          // boundary keys were published before the first barrier
          bool eq = false;
          if (tx > 0 && lane < rows) {
            const int4 k = keyR[(size_t)(tile - 1) * 32 + lane];
            eq = same3(k.x, k.y, k.z, c0, c1, c2);
          }
          eq_left = __ballot_sync(0xffffffffu, eq);
          if (ty > 0) {
            const int4 k = keyB[(size_t)(tile - tilesX) * 32 + lane];
            eq_above = same3(k.x, k.y, k.z, t0, t1, t2);
          }
        }
        if (tx > 0) left_p = pR[(size_t)in * ntiles + tile - 1];
        if (ty > 0) above_p = pB[(size_t)in * ntiles + tile - tilesX];
      }
      const uint32_t below = (2u << lane) - 1u;  // lanes 0..lane
      int ap = (int)((above_p >> lane) & 1u) & (int)eq_above;  // p above, where its key matches
      bits = 0;
      for (int r = 0; r < rows; r++) {
        const int a = ((valid >> r) & 1u) && !(ap && (r == 0 || ((up >> r) & 1u)));
        const int start_p = lane == 0 ? (a && !(((left_p & eq_left) >> r) & 1u)) : a;
        const uint32_t chained = __ballot_sync(0xffffffffu, lane > 0 && a && ((left >> r) & 1u));
        const uint32_t start_bits = __ballot_sync(0xffffffffu, start_p);
        const int st = 31 - __clz(~chained & below);
        const int p = (int)((start_bits >> st) & 1u) ^ ((lane - st) & 1);
        bits |= (uint32_t)p << r;
        ap = p;
      }
      const uint32_t rb = __shfl_sync(0xffffffffu, bits, 31);
      const uint32_t bb = __ballot_sync(0xffffffffu, (bits >> (rows - 1)) & 1u);
      changed = round == 0 || rb != last_r || bb != last_b;
      last_r = rb;
      last_b = bb;
      if (lane == 0) {
        pR[(size_t)out * ntiles + tile] = rb;
        pB[(size_t)out * ntiles + tile] = bb;
      }
    }
    if (changed && lane == 0) atomicAdd((uint32_t *)&chg[round % 3], 1u);
    // counter (round + 1) % 3 was last read before the previous barrier
    if (blockIdx.x == 0 && threadIdx.x == 0) chg[(round + 1) % 3] = 0;
    // a barrier that gives up marks the first map; every map's frame reports it
    grid_barrier(bar, gridDim.x, bd->f[m0].cnt, bd->f[m0].spin_limit);
    const uint32_t any = chg[round % 3];
    if (!any) {
      converged = true;
      break;
    }
    if (*(volatile uint32_t *)&bd->f[m0].cnt->error & ERR_DEDUPE_TIMEOUT) break;
  }
  // leave the barrier words as the next launch needs them: the arrival count
  // is zero after every completed barrier, counter (round + 1) % 3 was zeroed
  // in this round and counter round % 3 read as zero, and counter
  // (round + 2) % 3 was last read before this round's barrier (after a
  // barrier that gave up or no convergence, the host clears the words)
  if (converged && blockIdx.x == 0 && threadIdx.x == 0) chg[(round + 2) % 3] = 0;
  uint32_t nproc = 0;
  if (active && x < W) {
    for (int r = 0; r < rows; r++) processed[(size_t)(ty * DD_ROWS + r) * W + x] = (uint8_t)((bits >> r) & 1u);
    nproc = (uint32_t)__popc(rows >= 32 ? bits : (bits & ((1u << rows) - 1u)));
  }
  // the frame's processed pixels, counted once per tile (the insert that
  // follows no longer adds them per warp on the counters' cache line)
  nproc = __reduce_add_sync(0xffffffffu, nproc);
  if (active && lane == 0 && nproc) atomicAdd(&F.cnt->processed, nproc);
  if (blockIdx.x == 0 && (int)threadIdx.x < m1 - m0) {
    Counters *c = bd->f[m0 + threadIdx.x].cnt;
    c->dedupe_iters = round + 1;
    if (!converged) atomicOr(&c->error, ERR_DEDUPE_NOT_CONVERGED);
    if (*(volatile uint32_t *)&bd->f[m0].cnt->error & ERR_DEDUPE_TIMEOUT) atomicOr(&c->error, ERR_DEDUPE_TIMEOUT);
  }
}

template <int DD_ROWS>
// (register budget for 6 blocks per SM: a 10-frame sequence of 640x480
// frames fits one cooperative launch)
__global__ void __launch_bounds__(32 * DD_WARPS, 6) k_dedupe(const BatchDesc *__restrict__ bd, int m0, int m1,
                                                          uint32_t *bar) {
  dedupe_body<DD_ROWS>(bd, m0, m1, bar);
}

// One map's frame, its descriptor a launch parameter: block 0 also stores it
// to `out`, where the frame's later kernels read it.
template <int DD_ROWS>
__global__ void __launch_bounds__(32 * DD_WARPS) k_dedupe_one(const __grid_constant__ BatchDesc1 desc,
                                                              BatchDesc *out, uint32_t *bar) {
  if (blockIdx.x == 0) {
    const uint2 *src = reinterpret_cast<const uint2 *>(&desc);
    uint2 *dst = reinterpret_cast<uint2 *>(out);
    for (int k = threadIdx.x; k < (int)(sizeof(BatchDesc1) / 8); k += blockDim.x) dst[k] = src[k];
  }
  dedupe_body<DD_ROWS>(reinterpret_cast<const BatchDesc *>(&desc), 0, 1, bar);
}

int dedupe_tiles(int W, int H, int *tilesX, int *tilesY, int rows) {
  const int tx = (W + 31) / 32, ty = (H + rows - 1) / rows;
  if (tilesX) *tilesX = tx;
  if (tilesY) *tilesY = ty;
  return tx * ty;
}

size_t dedupe_boundary_elems(int W, int H) {
  // sized for the lowest tiles (the largest count)
  const size_t ntiles = (size_t)dedupe_tiles(W, H, nullptr, nullptr, DD_ROWS_LOW);
  return ntiles * 32 * 2 + ntiles;  // keys of the right column and bottom row, then 4 bit words per tile
}

template <int ROWS>
static cudaError_t resident_dedupe_warps(int device, int &warps) {
  static int resident[64] = {};
  const int dslot = device & 63;
  if (!resident[dslot]) {
    int per_sm = 0, per_sm_one = 0, sms = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dedupe<ROWS>, 32 * DD_WARPS, 0);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_one, k_dedupe_one<ROWS>, 32 * DD_WARPS, 0);
    if (e != cudaSuccess) return e;
    per_sm = std::min(per_sm, per_sm_one);  // (both launch forms use one capacity)
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    resident[dslot] = per_sm * sms;
  }
  warps = resident[dslot] * DD_WARPS;
  return cudaSuccess;
}

cudaError_t dedupe_capacity(int device, int rows, uint32_t &tiles) {
  int warps = 0;
  cudaError_t e = rows == DD_ROWS_SHORT  ? resident_dedupe_warps<DD_ROWS_SHORT>(device, warps)
                  : rows == DD_ROWS_LOW ? resident_dedupe_warps<DD_ROWS_LOW>(device, warps)
                                        : resident_dedupe_warps<DD_ROWS_TALL>(device, warps);
  tiles = (uint32_t)warps;
  return e;
}

cudaError_t launch_dedupe(const BatchDesc *d_batch, int m0, int m1, uint32_t tiles, int rows, uint32_t *barrier,
                          int device, cudaStream_t s) {
  uint32_t cap = 0;
  cudaError_t e = dedupe_capacity(device, rows, cap);
  if (e != cudaSuccess) return e;
  // one warp per tile, all resident at once
  const int blocks = (int)((tiles + DD_WARPS - 1) / DD_WARPS);
  if ((uint32_t)blocks * DD_WARPS > cap || blocks < 1) return cudaErrorInvalidConfiguration;
  void *args[] = {(void *)&d_batch, (void *)&m0, (void *)&m1, (void *)&barrier};
  note_launch();
  const void *fn = rows == DD_ROWS_SHORT  ? (const void *)k_dedupe<DD_ROWS_SHORT>
                   : rows == DD_ROWS_LOW ? (const void *)k_dedupe<DD_ROWS_LOW>
                                         : (const void *)k_dedupe<DD_ROWS_TALL>;
  return cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(32 * DD_WARPS), args, 0, s);
}

cudaError_t launch_dedupe_one(const BatchDesc *h_desc, BatchDesc *d_batch, uint32_t tiles, int rows,
                              uint32_t *barrier, int device, cudaStream_t s) {
  uint32_t cap = 0;
  cudaError_t e = dedupe_capacity(device, rows, cap);
  if (e != cudaSuccess) return e;
  const int blocks = (int)((tiles + DD_WARPS - 1) / DD_WARPS);
  if ((uint32_t)blocks * DD_WARPS > cap || blocks < 1 || h_desc->n != 1) return cudaErrorInvalidConfiguration;
  BatchDesc1 d1;
  memcpy(&d1, h_desc, sizeof(BatchDesc1));
  void *args[] = {(void *)&d1, (void *)&d_batch, (void *)&barrier};
  note_launch();
  const void *fn = rows == DD_ROWS_SHORT  ? (const void *)k_dedupe_one<DD_ROWS_SHORT>
                   : rows == DD_ROWS_LOW ? (const void *)k_dedupe_one<DD_ROWS_LOW>
                                         : (const void *)k_dedupe_one<DD_ROWS_TALL>;
  return cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(32 * DD_WARPS), args, 0, s);
}

// -------------------------------------------------------------- insert ----

__device__ __forceinline__ void queue_leaf(uint32_t leaf, uint32_t frame, uint32_t *stamp, uint32_t *queue,
                                           Counters *cnt) {
  // coarse leaves lie on the paths of many pixels: a plain read first keeps
  // those repeats off the atomic unit (the exchange below decides the winner)
  if (ld_volatile(&stamp[leaf]) == frame) return;
  if (atomicExch(&stamp[leaf], frame) != frame) {
    uint32_t q = atomicAdd(&cnt->queued, 1u);
    queue[q] = leaf;
  }
}

// The second half of queue_leaf for a leaf whose stamp was read earlier (st):
// the insert's descent reads a level's stamp, then issues the next level's
// octree loads before it looks at the value, so that the two round trips
// overlap.
__device__ __forceinline__ void queue_leaf_after(uint32_t leaf, uint32_t st, uint32_t frame, uint32_t *stamp,
                                                 uint32_t *queue, Counters *cnt) {
  if (st == frame) return;
  if (atomicExch(&stamp[leaf], frame) != frame) {
    uint32_t q = atomicAdd(&cnt->queued, 1u);
    queue[q] = leaf;
  }
}

// Wait until another thread finished allocating tree[ptr]; bounded.
__device__ __forceinline__ uint32_t wait_unlocked(uint32_t *tree, uint32_t ptr, uint32_t cur, Counters *cnt,
                                                  bool *ok, uint32_t limit) {
  uint32_t spins = 0;
  while (cur == LOCKED) {
    if (spins++ >= limit) {
      atomicOr(&cnt->error, ERR_SPIN_TIMEOUT);
      *ok = false;
      return cur;
    }
    __nanosleep(20);
    cur = ld_volatile(tree + ptr);
  }
  return cur;
}

// Branches on one descent's path: at most one per halving of the volume's
// side (16 bits of voxel coordinates) plus the root.
constexpr int DESCENT_MAX = 18;

// One processed pixel of the frame F (voxel key v): bounding-box growth,
// then (inside the volume) the descent of queryPointDepthSingle_func_subtree:
// queue the existing coarser leaves on the path, allocate missing branches,
// claim the final leaf.  Returns the number of octree levels probed; sets
// *created when this pixel wrote a new branch or leaf slot into the octree,
// and records the branches it passed (root first) in path[0, *npath).
__device__ __forceinline__ uint32_t insert_descend(const MapFrame &F, int i, int4 v, Counters *cnt, bool *created,
                                                   uint32_t *path, int *npath) {
  const uint32_t n = F.n;
  const int bw = (int)F.bw;
  uint32_t *tree = F.tree;
  const uint32_t leaves_max = F.leaves_max, branches_max = F.branches_max, frame = F.frame;
  uint32_t *stamp = F.stamp, *queue = F.queue;
  PendingLeaf *pend = F.pend;
  const uint32_t pend_cap = F.pend_cap;
  uint32_t probed = 0;
  int vv[3] = {v.x, v.y, v.z};
#pragma unroll
  for (int r = 0; r < 3; r++) {
    int lo = vv[r] - bw, hi = vv[r] + bw;
    if (lo < 0) atomicMin(&cnt->box_min[r], lo);
    if (hi >= (int)n) atomicMax(&cnt->box_max[r], hi);
  }
  if (!(v.x >= 0 && (uint16_t)v.x < n && v.y >= 0 && (uint16_t)v.y < n && v.z >= 0 && (uint16_t)v.z < n)) return 0;
  const uint32_t x = (uint16_t)v.x, y = (uint16_t)v.y, z = (uint16_t)v.z;
  const uint32_t target = (uint32_t)v.w;
  uint32_t ox = 0, oy = 0, oz = 0;
  uint32_t half = (uint16_t)(n >> 1);
  uint32_t branch = 0;
  bool ok = true;
  // the previous level's leaf (if any) and its stamp, read but not yet looked at
  uint32_t prev_leaf = BRANCHINIT, prev_st = frame;
  int np = 0;
  while ((half >> 1) >= target) {
    probed++;
    if (np < DESCENT_MAX) path[np++] = branch;
    *npath = np;
    uint32_t co = (x >= ox + half) * 1u + (y >= oy + half) * 2u + (z >= oz + half) * 4u;
    uint32_t ptr = branch + co + 8;
    uint32_t leaf = ld_tree(tree + ptr - 8);
    uint32_t child = ld_tree(tree + ptr);
    if (prev_leaf < leaves_max) queue_leaf_after(prev_leaf, prev_st, frame, stamp, queue, cnt);
    prev_leaf = leaf;
    prev_st = leaf < leaves_max ? ld_volatile(&stamp[leaf]) : frame;
    if (child == BRANCHINIT) {
      uint32_t old = atomicCAS(tree + ptr, BRANCHINIT, LOCKED);
      if (old == BRANCHINIT) {
        uint32_t nb = atomicAdd(&cnt->branches_used, 16u);
        if (nb + 16 > branches_max) {
          atomicOr(&cnt->error, ERR_BRANCH_OVERFLOW);
          atomicExch(tree + ptr, BRANCHINIT);
          if (prev_leaf < leaves_max) queue_leaf_after(prev_leaf, prev_st, frame, stamp, queue, cnt);
          return probed;
        }
        // (no fence: a new branch's slots hold BRANCHINIT since an earlier
        // launch, and nothing else this thread wrote is read through it)
        atomicExch(tree + ptr, nb);
        child = nb;
        *created = true;
        if (probed <= (uint32_t)MESH_TOP_LEVELS) atomicOr(&cnt->top_created, 1u);
      } else {
        child = old;
      }
    }
    child = wait_unlocked(tree, ptr, child, cnt, &ok, F.spin_limit);
    if (!ok || child == BRANCHINIT) {
      if (prev_leaf < leaves_max) queue_leaf_after(prev_leaf, prev_st, frame, stamp, queue, cnt);
      return probed;
    }
    ox += half * ((co & 1) != 0);
    oy += half * ((co & 2) != 0);
    oz += half * ((co & 4) != 0);
    branch = child;
    half >>= 1;
  }
  uint32_t co = (x >= ox + half) * 1u + (y >= oy + half) * 2u + (z >= oz + half) * 4u;
  uint32_t ptr = branch + co;
  probed++;
  if (np < DESCENT_MAX) path[np++] = branch;
  *npath = np;
  uint32_t cur = ld_tree(tree + ptr);
  if (prev_leaf < leaves_max) queue_leaf_after(prev_leaf, prev_st, frame, stamp, queue, cnt);
  if (cur == BRANCHINIT) {
    uint32_t old = atomicCAS(tree + ptr, BRANCHINIT, LOCKED);
    if (old == BRANCHINIT) {
      uint32_t rec = atomicAdd(&cnt->pending, 1u);
      if (rec >= pend_cap) {
        atomicOr(&cnt->error, ERR_PENDING_OVERFLOW);
        atomicExch(tree + ptr, BRANCHINIT);
        return probed;
      }
      PendingLeaf pl;
      pl.slot = ptr;
      pl.first_pixel = (uint32_t)i;
      pl.pos = make_ushort4((uint16_t)(ox + half * ((co & 1) != 0)), (uint16_t)(oy + half * ((co & 2) != 0)),
                            (uint16_t)(oz + half * ((co & 4) != 0)), (uint16_t)(half / BL));
      pend[rec] = pl;
      __threadfence();
      atomicExch(tree + ptr, PENDING + rec);
      *created = true;
      if (probed <= (uint32_t)MESH_TOP_LEVELS) atomicOr(&cnt->top_created, 1u);
      return probed;
    }
    cur = old;
  }
  cur = wait_unlocked(tree, ptr, cur, cnt, &ok, F.spin_limit);
  if (!ok) return probed;
  if (cur >= PENDING && cur < PENDING + pend_cap) {
    atomicMin(&pend[cur - PENDING].first_pixel, (uint32_t)i);
  } else if (cur < leaves_max) {
    queue_leaf(cur, frame, stamp, queue, cnt);
  }
  return probed;
}

// Mark every branch on the descent's path (root first, down to the branch
// that holds the pixel's slot, or to the last one reached when the descent
// stopped early) with the frame: the branches whose subtree gained a branch
// or a leaf.  Only pixels that created something do it; the loads of the
// stamps are independent, so they overlap.
__device__ __forceinline__ void stamp_path(const MapFrame &F, const uint32_t *path, int np) {
  for (int k = 0; k < np; k++) {
    uint32_t *b = F.bstamp + (path[k] >> 4);
    if (*b != F.frame) *b = F.frame;
  }
}

__device__ __forceinline__ uint32_t insert_pixel(const MapFrame &F, int i, int4 v, Counters *cnt) {
  bool created = false;
  uint32_t path[DESCENT_MAX];
  int np = 0;
  const uint32_t probed = insert_descend(F, i, v, cnt, &created, path, &np);
  if (created) stamp_path(F, path, np);
  return probed;
}

// One thread per pixel of every frame of the batch (each map's pixels padded
// to whole warps, so a warp never spans two maps).  At most 40 registers: six
// 256-thread blocks per SM instead of five (a few bytes of spill), for any
// block size the tuning picks.
__global__ void __maxnreg__(40) k_insert(const BatchDesc *__restrict__ bd, int m0, int m1) {
  pdl_enter();
  const int nmaps = min(bd->n, m1);
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x + (m0 ? bd->pix_end[m0 - 1] : 0u);
  if (g >= bd->pix_end[nmaps - 1]) return;
  int mi = m0;
  while (mi < nmaps - 1 && g >= bd->pix_end[mi]) mi++;
  const MapFrame &F = bd->f[mi];
  const int i = (int)(g - (mi ? bd->pix_end[mi - 1] : 0u));
  const int npix = (int)F.npix;
  const int4 *__restrict__ vox = F.vox;
  const uint8_t *__restrict__ processed = F.proc;
  Counters *cnt = F.cnt;
  // a de-duplication that did not complete leaves the frame out, and so does
  // a sequence halted by an earlier frame: the octree is not touched
  if (ld_volatile(&cnt->error) & (ERR_DEDUPE_FAILED | ERR_SEQ_HALT)) return;
  bool act = i < npix && processed[i];
  unsigned m = __ballot_sync(0xffffffffu, act);
  if (!act) return;
  // octree levels this pixel probes on its descent, summed per warp when the
  // stage profile is on (the algorithmic bytes of the insert: 16 B per level
  // -- the node's leaf and child slots, the leaf's frame stamp and its queue
  // entry, 4 B each)
  const uint32_t levels = insert_pixel(F, i, vox[i], cnt);
  if (F.count_levels) {
    const uint32_t sum = __reduce_add_sync(m, levels);
    if ((threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(&cnt->levels, sum);
  }
}

void launch_insert(const BatchDesc *d_batch, uint32_t pix, cudaStream_t s, int block, int m0, int m1, bool pdl) {
  if (!pix) return;
  if (block < 64 || block > 1024 || block % 32) block = 256;
  note_launch();
  launch_pdl(pdl, k_insert, dim3((pix + block - 1) / block), dim3(block), 0, s, d_batch, m0, m1);
}

// ------------------------------------------------- pending leaf order -----

__global__ void k_pending_keys(const PendingLeaf *pend, int npend, uint64_t *keys) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npend) return;
  keys[i] = pend[i].first_pixel;
}

size_t pending_sort_bytes(int n) { return argsort_temp_bytes((uint32_t)std::max(n, 0)); }

cudaError_t sort_pending(const PendingLeaf *pend, int npend, uint64_t *keys, uint64_t *keys_sorted, uint32_t *order,
                         void *tmp, size_t tmp_bytes, int end_bit, cudaStream_t s) {
  if (npend <= 0) return cudaSuccess;
  note_launch();
  k_pending_keys<<<(npend + 255) / 256, 256, 0, s>>>(pend, npend, keys);
  unsigned launches = 0;
  const cudaError_t e = argsort_u64(keys, (uint32_t)npend, end_bit, keys_sorted, order, tmp, tmp_bytes, s, &launches);
  note_launch(launches);
  return e;
}

// Leaf index = leaves_before + rank of first pixel; indices past the pool are
// stored in the tree but get no leaf record, like addLeaf's overflow
// (traversal_functions.cpp:201-210).
__device__ __forceinline__ void finalize_one(const PendingLeaf &p, uint32_t idx, uint32_t leaves_max, uint32_t *tree,
                                             ushort4 *leaf, uint32_t frame, uint32_t *stamp, uint32_t *queue,
                                             Counters *cnt) {
  tree[p.slot] = idx;
  if (idx < leaves_max) {
    leaf[idx] = p.pos;
    queue_leaf(idx, frame, stamp, queue, cnt);
  }
}

// A new leaf of rank r in its frame: index leaves_before + r, queued at
// position q0 + r after the q0 bricks the insert queued (a pending leaf is
// never on the insert's queue), so no atomics; the frame's queue length
// becomes q0 + the number of leaves placed.
__device__ __forceinline__ void finalize_new(const PendingLeaf &p, uint32_t idx, uint32_t qpos, uint32_t leaves_max,
                                             uint32_t *tree, ushort4 *leaf, uint32_t frame, uint32_t *stamp,
                                             uint32_t *queue) {
  tree[p.slot] = idx;
  if (idx < leaves_max) {
    leaf[idx] = p.pos;
    stamp[idx] = frame;
    queue[qpos] = idx;
  }
}

__global__ void k_finalize(const PendingLeaf *pend, const uint32_t *order, int npend, uint32_t leaves_before,
                           uint32_t leaves_max, uint32_t *tree, ushort4 *leaf, uint32_t frame, uint32_t *stamp,
                           uint32_t *queue, Counters *cnt) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= npend) return;
  finalize_one(pend[order[j]], leaves_before + (uint32_t)j, leaves_max, tree, leaf, frame, stamp, queue, cnt);
}

void launch_finalize(const PendingLeaf *pend, const uint32_t *order, int npend, uint32_t leaves_before,
                     uint32_t leaves_max, uint32_t *tree, ushort4 *leaf, uint32_t frame, uint32_t *stamp,
                     uint32_t *queue, Counters *cnt, cudaStream_t s) {
  if (npend <= 0) return;
  note_launch();
  k_finalize<<<(npend + 255) / 256, 256, 0, s>>>(pend, order, npend, leaves_before, leaves_max, tree, leaf, frame,
                                                 stamp, queue, cnt);
}

// parent = finest ancestor leaf that existed when this leaf was created: the
// reference records the last leaf met on the descent (`pl`,
// traversal_functions.cpp:327-333, 376-379); leaves of this frame exist in
// index order, so that is the finest ancestor with a smaller index.
__device__ __forceinline__ uint32_t parent_of(uint32_t idx, uint32_t leaves_max, const uint32_t *tree, uint32_t n,
                                              const ushort4 &p) {
  const uint32_t edge = (uint32_t)p.w * BL;
  uint32_t ox = 0, oy = 0, oz = 0, half = n >> 1, branch = 0, pl = BRANCHINIT;
  while (half > edge) {
    uint32_t co = (p.x >= ox + half) * 1u + (p.y >= oy + half) * 2u + (p.z >= oz + half) * 4u;
    uint32_t l = tree[branch + co];
    if (l < leaves_max && l < idx) pl = l;
    branch = tree[branch + co + 8];
    if (branch >= PENDING) break;  // no child branch (cannot happen for a placed leaf)
    ox += half * ((co & 1) != 0);
    oy += half * ((co & 2) != 0);
    oz += half * ((co & 4) != 0);
    half >>= 1;
  }
  return pl;
}

__global__ void k_parents(int npend, uint32_t leaves_before, uint32_t leaves_max, const uint32_t *tree, uint32_t n,
                          const ushort4 *leaf, uint32_t *parent) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= npend) return;
  const uint32_t idx = leaves_before + (uint32_t)j;
  if (idx >= leaves_max) return;
  parent[idx] = parent_of(idx, leaves_max, tree, n, leaf[idx]);
}

// Parents of the leaves the finalisation of each frame of the descriptor
// placed: blocks PARENT_BLOCKS per frame, striding over its new leaves.  A
// parent is the finest ancestor with a smaller index, so it can be found any
// time after the leaf is placed; off the chain of frames (the next frame's
// insert does not wait for it).  Frames that placed nothing are skipped.
constexpr int PARENT_BLOCKS = 4, PARENT_THREADS = 256;

__global__ void __launch_bounds__(PARENT_THREADS) k_parents_frames(const BatchDesc *__restrict__ bd, int m0) {
  pdl_enter();
  const MapFrame &F = bd->f[m0 + blockIdx.x / PARENT_BLOCKS];
  const Counters *cnt = F.cnt;
  if (ld_volatile(&cnt->error) & (ERR_DEDUPE_FAILED | ERR_PENDING_OVERFLOW | ERR_SEQ_HALT)) return;
  const uint32_t npend = ld_volatile(&cnt->pending);
  const uint32_t leaves_before = F.chain ? ld_volatile(&cnt->leaves_base) : F.leaves_before;
  const uint32_t stride = PARENT_BLOCKS * PARENT_THREADS;
  for (uint32_t j = (blockIdx.x % PARENT_BLOCKS) * PARENT_THREADS + threadIdx.x; j < npend; j += stride) {
    const uint32_t idx = leaves_before + j;
    if (idx >= F.leaves_max) break;
    F.parent[idx] = parent_of(idx, F.leaves_max, F.tree, F.n, F.leaf[idx]);
  }
}

void launch_parents_frames(const BatchDesc *d_batch, int nframes, cudaStream_t s, int m0, bool pdl) {
  if (nframes < 1) return;
  note_launch();
  launch_pdl(pdl, k_parents_frames, dim3(nframes * PARENT_BLOCKS), dim3(PARENT_THREADS), 0, s, d_batch, m0);
}

// The whole frame's pending leaves in one block.  A leaf's creation rank is
// the number of pending leaves with a smaller first pixel; first pixels are
// distinct (a pixel creates at most one leaf), so the rank is a prefix count
// over a bitmap of the image's pixels held in shared memory.  Then indices,
// the leaf table and the parents.
constexpr int FIN_THREADS = 1024;
constexpr size_t FIN_SMEM_MAX = 200 * 1024;
constexpr int FIN_FEW = 1024;  // new leaves ranked by direct count (the dynamic shared memory holds >= 1024 words)

// One block per map of the batch; the pending count is read on the device
// (nothing is done after an allocation error, which the host reports).
// A frame of a sequence hands the next frame its branch count and leaf base,
// or halts it (and so every later frame) when this frame must grow the
// volume, failed or was halted itself: the host runs those frames again after
// the growth, or reports the failure.
__device__ __forceinline__ void chain_next(const MapFrame &F, Counters *cnt, uint32_t leaves_before, bool halt) {
  Counters *nx = F.next_cnt;
  if (!nx) return;
  nx->branches_used = ld_volatile(&cnt->branches_used);
  nx->leaves_base = leaves_before + ld_volatile(&cnt->pending);
  if (halt) atomicOr(&nx->error, ERR_SEQ_HALT);
}

// Deferred update: mark each brick of the frame's queue (nq entries: the
// q0 the insert queued, then the new leaves in rank order, indices from
// leaves_before) with the frame's bit, and list the bricks no earlier frame
// of the pass has marked.  Every thread of the block runs the same number of
// iterations, so the list slots are claimed with one atomic per warp.
__device__ __forceinline__ void finalize_mark(const MapFrame &F, uint32_t q0, uint32_t nq, uint32_t leaves_before,
                                              int t) {
  const uint32_t bit = 1u << F.upd_slot;
  const uint32_t rounds = (nq + FIN_THREADS - 1) / FIN_THREADS;
  for (uint32_t it = 0; it < rounds; it++) {
    const uint32_t j = it * FIN_THREADS + (uint32_t)t;
    bool add = false;
    uint32_t b = 0;
    if (j < nq) {
      b = j < q0 ? F.queue[j] : leaves_before + (j - q0);
      // a part of a sharded map updates the bricks it owns; the queue holds
      // each brick once, so the old mask lacks this bit
      if (F.shards <= 1 || owns_brick(F, F.leaf[b])) add = atomicOr(&F.upd_mask[b], bit) == 0u;
    }
    const unsigned ball = __ballot_sync(0xffffffffu, add);
    uint32_t at = 0;
    if ((t & 31) == 0 && ball) at = atomicAdd(F.upd_count, (uint32_t)__popc(ball));
    at = __shfl_sync(0xffffffffu, at, 0);
    if (add) F.upd_list[at + __popc(ball & ((1u << (t & 31)) - 1u))] = b;
  }
}

__global__ void __launch_bounds__(FIN_THREADS) k_finalize_bitmap(const BatchDesc *__restrict__ bd, int m0) {
  extern __shared__ uint32_t fin_smem[];
  // (the next frame's insert is scheduled once this has started: it overlaps
  // this kernel, not the insert before it)
  pdl_wait();
  pdl_trigger();
  const MapFrame &F = bd->f[m0 + blockIdx.x];
  Counters *cnt = F.cnt;
  if (F.chain || F.next_cnt) {
    // a sequence's frame: everything it reads of the counters was written by
    // earlier kernels (its own insert, the previous finalisation)
    if (ld_volatile(&cnt->error) & (ERR_SEQ_HALT | ERR_DEDUPE_FAILED | ERR_PENDING_OVERFLOW)) {
      if (threadIdx.x == 0) chain_next(F, cnt, F.chain ? ld_volatile(&cnt->leaves_base) : F.leaves_before, true);
      return;
    }
  }
  // After a de-duplication error nothing was inserted.  After an insert whose
  // wait gave up (ERR_SPIN_TIMEOUT) the pending leaves recorded before it are
  // complete records and are placed, so that no octree slot keeps a pending
  // mark; the frame's update is skipped (ERR_FRAME_FAILED).
  if (cnt->error & (ERR_DEDUPE_FAILED | ERR_PENDING_OVERFLOW)) return;
  const int npend = (int)cnt->pending;
  const uint32_t q0 = cnt->queued;  // the insert's queue
  const uint32_t branches_used = cnt->branches_used;
  const PendingLeaf *pend = F.pend;
  const uint32_t leaves_before = F.chain ? ld_volatile(&cnt->leaves_base) : F.leaves_before;
  const uint32_t npix = F.npix, leaves_max = F.leaves_max, frame = F.frame;
  // the new leaves that fit the pool (indices below leaves_max) are queued
  const uint32_t nplaced = leaves_before < leaves_max ? min((uint32_t)npend, leaves_max - leaves_before) : 0u;
  const int t = threadIdx.x;
  // Whether the deferred update takes the frame (not when it failed or the
  // volume must grow first: the host handles those), decided by one thread
  // for the block (the confidence network, on another stream, may set its
  // error word meanwhile).  A map in one part marks its queue at once: the
  // marks need no leaf of this frame placed, so their atomics overlap the
  // ranking below; a part of a sharded map needs the new leaves' positions
  // and marks after it.
  __shared__ int aside_flag;
  if (t == 0) aside_flag = fuse_deferred(F) ? 1 : 0;
  __syncthreads();
  const bool stand_aside = aside_flag != 0;
  const bool mark = F.upd_mask && !stand_aside;
  if (mark && F.shards <= 1) finalize_mark(F, q0, q0 + nplaced, leaves_before, t);
  uint32_t *rank = F.rank, *tree = F.tree, *stamp = F.stamp, *queue = F.queue;
  ushort4 *leaf = F.leaf;
  const uint32_t nwords = (npix + 31) / 32;
  uint32_t *bitmap = fin_smem;
  uint32_t *chunk_base = fin_smem + nwords;  // [FIN_THREADS]
  const uint32_t chunk = (nwords + FIN_THREADS - 1) / FIN_THREADS;
  if (npend <= FIN_FEW) {
    // few new leaves (the usual frame): a leaf's rank counted directly over
    // the others' first pixels in shared memory, without the image bitmap
    uint32_t *fp = fin_smem;
    for (int j = t; j < npend; j += FIN_THREADS) fp[j] = pend[j].first_pixel;
    __syncthreads();
    for (int j = t; j < npend; j += FIN_THREADS) {
      const uint32_t mine_fp = fp[j];
      uint32_t r = 0;
      for (int i = 0; i < npend; i++) r += fp[i] < mine_fp ? 1u : 0u;
      rank[j] = r;
      finalize_new(pend[j], leaves_before + r, q0 + r, leaves_max, tree, leaf, frame, stamp, queue);
    }
  } else {
    for (uint32_t w = t; w < nwords; w += FIN_THREADS) bitmap[w] = 0;
    __syncthreads();
    for (int j = t; j < npend; j += FIN_THREADS) {
      const uint32_t fp = pend[j].first_pixel;
      atomicOr(&bitmap[fp >> 5], 1u << (fp & 31));
    }
    __syncthreads();
    // the image bitmap of first pixels; exclusive prefix of the per-thread
    // chunk counts
    uint32_t mine = 0;
    const uint32_t w0 = (uint32_t)t * chunk, w1 = min(nwords, w0 + chunk);
    for (uint32_t w = w0; w < w1; w++) mine += __popc(bitmap[w]);
    using Scan = cub::BlockScan<uint32_t, FIN_THREADS>;
    __shared__ typename Scan::TempStorage scan_tmp;
    uint32_t before = 0;
    Scan(scan_tmp).ExclusiveSum(mine, before);
    chunk_base[t] = before;
    __syncthreads();
    for (int j = t; j < npend; j += FIN_THREADS) {
      const PendingLeaf p = pend[j];
      const uint32_t w = p.first_pixel >> 5, c = w / chunk;
      uint32_t r = chunk_base[c];
      for (uint32_t k = c * chunk; k < w; k++) r += __popc(bitmap[k]);
      r += __popc(bitmap[w] & ((1u << (p.first_pixel & 31)) - 1u));
      rank[j] = r;
      finalize_new(p, leaves_before + r, q0 + r, leaves_max, tree, leaf, frame, stamp, queue);
    }
  }
  // (the new leaves' parents: k_parents_frames, after this kernel)
  if (mark && F.shards > 1) {
    __syncthreads();  // the new leaves' positions
    finalize_mark(F, q0, q0 + nplaced, leaves_before, t);
  }
  if (t == 0) {
    cnt->queued = q0 + nplaced;
    Counters *nx = F.next_cnt;
    if (nx) {
      // the next frame of a sequence starts from this one's counts
      nx->branches_used = branches_used;
      nx->leaves_base = leaves_before + (uint32_t)npend;
      if (stand_aside) atomicOr(&nx->error, ERR_SEQ_HALT);
    }
  }
}

bool finalize_small_fits(uint32_t npix) {
  return sizeof(uint32_t) * (((size_t)npix + 31) / 32 + FIN_THREADS) <= FIN_SMEM_MAX;
}

bool finalize_small_prepare(int device) {
  static std::atomic<unsigned long long> attr_devices{0};
  const unsigned long long bit = 1ull << (device & 63);
  if (!(attr_devices.load() & bit)) {
    if (cudaFuncSetAttribute(k_finalize_bitmap, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FIN_SMEM_MAX) !=
        cudaSuccess)
      return false;
    attr_devices.fetch_or(bit);
  }
  return true;
}

bool launch_finalize_small(const BatchDesc *d_batch, int nmaps, uint32_t max_npix, int device, cudaStream_t s,
                           int m0, bool pdl) {
  const size_t smem = sizeof(uint32_t) * (((size_t)max_npix + 31) / 32 + FIN_THREADS);
  if (smem > FIN_SMEM_MAX || nmaps < 1) return false;
  if (!finalize_small_prepare(device)) return false;
  note_launch();
  return launch_pdl(pdl, k_finalize_bitmap, dim3(nmaps), dim3(FIN_THREADS), smem, s, d_batch, m0) == cudaSuccess;
}

void launch_parents(int npend, uint32_t leaves_before, uint32_t leaves_max, const uint32_t *tree, uint32_t n,
                    const ushort4 *leaf, uint32_t *parent, cudaStream_t s) {
  if (npend <= 0) return;
  note_launch();
  k_parents<<<(npend + 255) / 256, 256, 0, s>>>(npend, leaves_before, leaves_max, tree, n, leaf, parent);
}

// ---------------------------------------------------------------- grow ----

__global__ void k_shift_branches(uint32_t *tree, uint32_t used, uint32_t shift) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= used) return;
  if ((i & 15) >= 8 && tree[i] != BRANCHINIT) tree[i] += shift;
}

void launch_shift_branches(uint32_t *tree, uint32_t used, uint32_t shift, cudaStream_t s) {
  if (!used) return;
  note_launch();
  k_shift_branches<<<(used + 255) / 256, 256, 0, s>>>(tree, used, shift);
}

__global__ void k_shift_leaves(ushort4 *leaf, uint32_t n, ushort3 add) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  ushort4 p = leaf[i];
  p.x = (uint16_t)(p.x + add.x);
  p.y = (uint16_t)(p.y + add.y);
  p.z = (uint16_t)(p.z + add.z);
  leaf[i] = p;
}

void launch_shift_leaves(ushort4 *leaf, uint32_t n, ushort3 add, cudaStream_t s) {
  if (!n) return;
  note_launch();
  k_shift_leaves<<<(n + 255) / 256, 256, 0, s>>>(leaf, n, add);
}

__global__ void k_fill(uint32_t *p, size_t n, uint32_t v) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t stride = (size_t)gridDim.x * blockDim.x;
  for (; i < n; i += stride) p[i] = v;
}

void launch_fill(uint32_t *p, size_t n, uint32_t v, cudaStream_t s) {
  if (!n) return;
  size_t blocks = (n + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  note_launch();
  k_fill<<<(unsigned)blocks, 256, 0, s>>>(p, n, v);
}

// Load this file's kernels now (modules load lazily on first launch, which
// would otherwise land inside the first frame that needs a kernel).
cudaError_t prewarm_alloc_kernels() {
  const void *fns[] = {(const void *)k_first_bbox, (const void *)k_dedupe<DD_ROWS_SHORT>,
                       (const void *)k_dedupe_one<DD_ROWS_SHORT>, (const void *)k_dedupe_one<DD_ROWS_LOW>,
                       (const void *)k_dedupe_one<DD_ROWS_TALL>,
                       (const void *)k_dedupe<DD_ROWS_LOW>,
                       (const void *)k_dedupe<DD_ROWS_TALL>, (const void *)k_insert,
                       (const void *)k_pending_keys, (const void *)k_finalize, (const void *)k_parents, (const void *)k_parents_frames,
                       (const void *)k_finalize_bitmap, (const void *)k_shift_branches,
                       (const void *)k_shift_leaves, (const void *)k_fill};
  for (const void *f : fns) {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, f);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace ffb
