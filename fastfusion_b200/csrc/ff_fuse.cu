// Per-voxel SDF / weight / colour fusion of the queued bricks.
//
// Restates update8AddLoopAVXSingleInteger (reference update_functions.cpp:1187-1444)
// as run by updateWrapperInteger (:1633-1732): every operation in
// round-toward-zero (the reference sets MXCSR=RZ, :1678-1679) with the
// reference's operation order, voxel positions accumulated the way the
// reference's loops accumulate them (z steps, then y steps, then x * step),
// and the reference's three reciprocals either exactly as the host CPU's
// RCPPS computes them (FF_RCP_HOST: table of the instruction's mantissa map,
// bit-identical to the reference binary on that host) or as exact RZ
// reciprocals (FF_RCP_EXACT: __frcp_rz, host-independent).
// Every voxel of every queued brick is read and written, like the reference.
//
// One CTA per brick, one thread per voxel: the 512 SDF and weight words of a
// brick and its three 512-entry colour planes are contiguous, so each load and
// store is a fully coalesced 2 KB / 1 KB segment.
#include <string.h>

#include <vector>
#if defined(__x86_64__) || defined(_M_X64)
#include <xmmintrin.h>
#endif

#include "ff_kernels.h"

namespace ffb {

// x86 float->int32 under round-toward-zero (truncation; 0x80000000 when out
// of range), the behaviour of _mm256_cvtps_epi32 with MXCSR=RZ.
__device__ __forceinline__ int cvt_x86_rz(float f) {
  if (!(f > -2147483904.0f && f < 2147483648.0f)) return (int)0x80000000;
  return __float2int_rz(f);
}

// Reciprocal as the host CPU's RCPPS computes it: the result mantissa is a
// function of the input mantissa alone -- in practice of its top 23 - shift
// bits (tab, measured from the instruction for x in [1,2)) --, the exponent
// is negated; zero and denormal inputs give
// infinity, infinity gives zero, results below the normal range are flushed
// to zero, NaN stays NaN -- the behaviour checked when the table is built.
__device__ __forceinline__ float rcp_host(float x, const uint32_t *__restrict__ tab, int shift) {
  const uint32_t u = __float_as_uint(x);
  const uint32_t sgn = u & 0x80000000u;
  const int e = (int)((u >> 23) & 255u);
  const uint32_t m = u & 0x7fffffu;
  if (e == 255) return m ? __uint_as_float(u | 0x400000u) : __uint_as_float(sgn);
  if (e == 0) return __uint_as_float(sgn | 0x7f800000u);
  const uint32_t t = __ldg(tab + (m >> shift));
  const int te = (int)((t >> 23) & 255u) - (e - 127);
  if (te <= 0) return __uint_as_float(sgn);
  return __uint_as_float(sgn | (t & 0x7fffffu) | ((uint32_t)te << 23));
}

template <bool RCP_HOST>
__device__ __forceinline__ float rcp_upd(float x, const uint32_t *tab, int shift) {
  return RCP_HOST ? rcp_host(x, tab, shift) : __frcp_rz(x);
}

template <bool FP16, bool RCP_HOST>
__device__ __forceinline__ void fuse_brick(const uint32_t brick, const ushort4 *__restrict__ leaf,
                                           float *__restrict__ sdf, float *__restrict__ wgt,
                                           __half *__restrict__ sdf16, __half *__restrict__ wgt16,
                                           uint16_t *__restrict__ col, const uint16_t *__restrict__ depth,
                                           const uint8_t *__restrict__ bgr, int W, int H, const CamF &q, float scale,
                                           float thr, float scaling, float maxcam, const uint32_t *__restrict__ rtab,
                                           int rshift, const float *__restrict__ conf, const int v) {
  const int x = v & 7, y = (v >> 3) & 7, z = v >> 6;
  const ushort4 o = leaf[brick];
  // the voxel's stored state does not depend on the projection: load it first
  // so that its latency overlaps the arithmetic and the image gathers
  const size_t vi = (size_t)brick * 512 + v;
  float wAcc, dAcc;
  if (FP16) {
    wAcc = __half2float(wgt16[vi]);
    dAcc = __half2float(sdf16[vi]);
  } else {
    wAcc = wgt[vi];
    dAcc = sdf[vi];
  }
  uint16_t *cb = col + (size_t)brick * 1536 + v;
  const uint16_t acc0 = cb[0], acc1 = cb[512], acc2 = cb[1024];
  const float *M = q.r;
  const float ls = (float)o.w;
  const float fls = __fmul_rz(ls, scale);
  const float fo0 = (float)o.x, fo1 = (float)o.y, fo2 = (float)o.z;
  // brick origin in camera coordinates
  float pzx = __fadd_rz(__fmul_rz(__fadd_rz(__fadd_rz(__fmul_rz(M[0], fo0), __fmul_rz(M[1], fo1)), __fmul_rz(M[2], fo2)), scale), q.t[0]);
  float pzy = __fadd_rz(__fmul_rz(__fadd_rz(__fadd_rz(__fmul_rz(M[3], fo0), __fmul_rz(M[4], fo1)), __fmul_rz(M[5], fo2)), scale), q.t[1]);
  float pzz = __fadd_rz(__fmul_rz(__fadd_rz(__fadd_rz(__fmul_rz(M[6], fo0), __fmul_rz(M[7], fo1)), __fmul_rz(M[8], fo2)), scale), q.t[2]);
  const float d11 = __fmul_rz(M[0], fls), d21 = __fmul_rz(M[3], fls), d31 = __fmul_rz(M[6], fls);
  const float d12 = __fmul_rz(M[1], fls), d22 = __fmul_rz(M[4], fls), d32 = __fmul_rz(M[7], fls);
  const float d13 = __fmul_rz(M[2], fls), d23 = __fmul_rz(M[5], fls), d33 = __fmul_rz(M[8], fls);
  // the reference walks z, then y, adding one step per iteration
  for (int i = 0; i < z; i++) {
    pzx = __fadd_rz(pzx, d13);
    pzy = __fadd_rz(pzy, d23);
    pzz = __fadd_rz(pzz, d33);
  }
  for (int i = 0; i < y; i++) {
    pzx = __fadd_rz(pzx, d12);
    pzy = __fadd_rz(pzy, d22);
    pzz = __fadd_rz(pzz, d32);
  }
  // lane offsets 0, d, 2d, ..., 7d of the 8-wide rows
  const float fx_ = (float)x;
  const float kx = x == 0 ? 0.0f : (x == 1 ? d11 : __fmul_rz(fx_, d11));
  const float ky = x == 0 ? 0.0f : (x == 1 ? d21 : __fmul_rz(fx_, d21));
  const float kz = x == 0 ? 0.0f : (x == 1 ? d31 : __fmul_rz(fx_, d31));
  const float px = __fadd_rz(pzx, kx), py = __fadd_rz(pzy, ky), pz = __fadd_rz(pzz, kz);

  const float len = __fsqrt_rz(__fadd_rz(__fadd_rz(__fmul_rz(px, px), __fmul_rz(py, py)), __fmul_rz(pz, pz)));
  const float rc = rcp_upd<RCP_HOST>(pz, rtab, rshift);
  const int imx = cvt_x86_rz(__fadd_rz(q.cx, __fmul_rz(q.fx, __fmul_rz(px, rc))));
  const int imy = cvt_x86_rz(__fadd_rz(q.cy, __fmul_rz(q.fy, __fmul_rz(py, rc))));
  const int cyi = max(min(imy, H - 1), 0);
  const int cxi = max(min(imx, W - 1), 0);
  const int ii = W * cyi + cxi;
  // every gather at the pixel is issued before any of them is used
  const uint16_t draw = __ldg(depth + ii);
  const uint8_t *p8 = bgr + 3 * (size_t)ii;
  const uint8_t cr = __ldg(p8 + 2), cg = __ldg(p8 + 1), cbl = __ldg(p8 + 0);
  const float cw = conf ? __ldg(conf + ii) : 1.0f;
  const float h = __fmul_rz(scaling, (float)draw);
  const float dInc = __fsub_rz(len, __fmul_rz(__fmul_rz(len, rc), h));
  const bool mask = pz > 0.0f && imy < H && imy > -1 && imx < W && imx > -1 && h < maxcam;
  const float thrD = __fmul_rz(thr, ls);
  const float thrW = __fmul_rz(__fmul_rz(WEIGHT_FACTOR, thr), ls);
  const float front = dInc < DIST_W_EPS ? 1.0f : 0.0f;
  const float back = (dInc >= DIST_W_EPS && dInc < thrW) ? 1.0f : 0.0f;
  const float fall = __fmul_rz(__fsub_rz(thrW, dInc), rcp_upd<RCP_HOST>(__fsub_rz(thrW, DIST_W_EPS), rtab, rshift));
  float wInc = mask ? __fadd_rz(front, __fmul_rz(fall, back)) : 0.0f;
  // learned weight: the ramp's increment scaled by the pixel's confidence
  if (conf) wInc = __fmul_rz(wInc, cw);

  const float wNew = __fadd_rz(wAcc, wInc);
  const float factor = rcp_upd<RCP_HOST>(__fadd_rz(wNew, wNew <= 0.0f ? 1.0f : 0.0f), rtab, rshift);
  float tr = dInc < thrD ? dInc : thrD;
  const float lo = -thrD;
  tr = tr > lo ? tr : lo;
  const float add = mask ? __fmul_rz(tr, wInc) : 0.0f;
  const float dNew = __fmul_rz(__fadd_rz(__fmul_rz(dAcc, wAcc), add), factor);
  if (FP16) {
    sdf16[vi] = __float2half_rn(dNew);
    wgt16[vi] = __float2half_rn(wNew);
  } else {
    sdf[vi] = dNew;
    wgt[vi] = wNew;
  }
  const float inc[3] = {__fmul_rz((float)cr, COLOR_MUL), __fmul_rz((float)cg, COLOR_MUL),
                        __fmul_rz((float)cbl, COLOR_MUL)};
  const uint16_t accs[3] = {acc0, acc1, acc2};
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float acc = (float)accs[c];
    float val = __fmul_rz(__fadd_rz(__fmul_rz(acc, wAcc), __fmul_rz(inc[c], wInc)), factor);
    val = val < 65280.0f ? val : 65280.0f;
    cb[c * 512] = (uint16_t)__float2int_rz(val);
  }
}

// BPC bricks per block of 512 BPC threads, one thread per voxel, blocks
// looping over the bricks of every map of the batch in order.  Gated: each
// map's count is read on the device; otherwise the host's count (nq_host)
// is used.  Every map's camera parameters are staged in shared memory once.
template <bool FP16, bool RCP_HOST, int BPC, int MINB>
__global__ void __launch_bounds__(512 * BPC, MINB) k_fuse(const BatchDesc *__restrict__ bd, int gated) {
  __shared__ uint32_t end[BATCH_MAX];  // inclusive prefix of the maps' brick counts
  __shared__ CamF sq[BATCH_MAX];
  const int nmaps = bd->n;
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int m = 0; m < nmaps; m++) {
      const MapFrame &F = bd->f[m];
      acc += gated ? (fuse_deferred(F) ? 0u : F.cnt->queued) : F.nq_host;
      end[m] = acc;
    }
  }
  constexpr int CF = sizeof(CamF) / sizeof(float);
  for (int i = threadIdx.x; i < nmaps * CF; i += blockDim.x)
    reinterpret_cast<float *>(sq)[i] = reinterpret_cast<const float *>(&bd->f[i / CF].q)[i % CF];
  __syncthreads();
  const uint32_t total = end[nmaps - 1];
  const int sub = threadIdx.x >> 9, v = threadIdx.x & 511;
  int m = 0;
  for (uint32_t b = blockIdx.x * BPC + sub; b < total; b += gridDim.x * BPC) {
    while (b >= end[m]) m++;
    const MapFrame &F = bd->f[m];
    const uint32_t local = b - (m ? end[m - 1] : 0u);
    const uint32_t brick = F.queue[local];
    // a part of a sharded map updates the bricks it owns
    if (F.shards > 1 && !owns_brick(F, F.leaf[brick])) continue;
    fuse_brick<FP16, RCP_HOST>(brick, F.leaf, F.sdf, F.wgt, F.sdf16, F.wgt16, F.col, F.depth, F.bgr, F.W, F.H, sq[m],
                               F.scale, F.thr, F.scaling, F.maxcam, F.rcp_tab, F.rcp_shift, F.conf, v);
  }
}

// ---------------------------------------------------------------------------
// Deferred update: one pass over the bricks of several frames.
//
// The reference updates every queued brick once per frame.  A voxel's update
// depends only on its own stored state and on the frame (camera parameters,
// depth, colour, confidence), so the frames of a batch can be applied to a
// voxel one after another in a single pass: load the state once, apply each
// frame that queued the brick, in frame order, with the same round-toward-zero
// operations, and store once.  Between two frames the state is rounded exactly
// as a store and a load would round it (colour truncated to uint16; SDF and
// weight to half with FP16 storage), so every bit equals the frame-by-frame
// update.  The brick's state is read and written once per pass instead of
// once per frame.
//
// One block of 512 threads per brick (one thread per voxel), blocks striding
// over the pass's brick list.  Per brick and frame, the start positions of
// the 64 voxel rows -- the reference's loop accumulation, z steps then y
// steps -- are made once, by 64 threads, into shared memory.
// ---------------------------------------------------------------------------

constexpr int FUSE_MULTI_BLOCKS_PER_SM = 2;

template <bool FP16, bool RCP_HOST>
__global__ void __launch_bounds__(512, FUSE_MULTI_BLOCKS_PER_SM) k_fuse_multi(const __grid_constant__ FuseBatch fb) {
  __shared__ float3 rows[FUSE_SLOTS_MAX][64];  // per frame: (z, y) row start in camera coordinates
  __shared__ float3 xstep[FUSE_SLOTS_MAX];     // per frame: d11, d21, d31 (one voxel along x)
  __shared__ int order[FUSE_SLOTS_MAX];        // the brick's frames, in frame order
  __shared__ uint32_t s_mask;
  __shared__ ushort4 s_leaf;
  const int v = threadIdx.x;
  const int x = v & 7, y = (v >> 3) & 7, z = v >> 6;
  const uint32_t total = *fb.count;
  const float scale = fb.scale, thr = fb.thr;
  const uint32_t *__restrict__ rtab = fb.rcp_tab;
  const int rshift = fb.rcp_shift;
  for (uint32_t bi = blockIdx.x; bi < total; bi += gridDim.x) {
    const uint32_t brick = fb.list[bi];
    if (v == 0) {
      s_mask = fb.mask[brick];
      s_leaf = fb.leaf[brick];
    }
    __syncthreads();
    const uint32_t mask = s_mask;
    const ushort4 o = s_leaf;
    const int nk = __popc(mask);
    if (v < 32 && ((mask >> v) & 1u)) order[__popc(mask & ((1u << v) - 1u))] = v;
    // the voxel's stored state, loaded while the row starts are made
    const size_t vi = (size_t)brick * 512 + v;
    float wAcc, dAcc;
    if (FP16) {
      wAcc = __half2float(fb.wgt16[vi]);
      dAcc = __half2float(fb.sdf16[vi]);
    } else {
      wAcc = fb.wgt[vi];
      dAcc = fb.sdf[vi];
    }
    uint16_t *cb = fb.col + (size_t)brick * 1536 + v;
    uint16_t acc[3] = {cb[0], cb[512], cb[1024]};
    __syncthreads();
    const float ls = (float)o.w;
    const float fls = __fmul_rz(ls, scale);
    const float fo0 = (float)o.x, fo1 = (float)o.y, fo2 = (float)o.z;
    for (int k0 = 0; k0 < nk; k0 += 8) {
      const int k = k0 + (v >> 6);
      if (k < nk) {
        const int j = order[k];
        const CamF &q = fb.s[j].q;
        const float *M = q.r;
        // brick origin in camera coordinates, then z steps and y steps as
        // the reference's loops add them
        float pzx = __fadd_rz(__fmul_rz(__fadd_rz(__fadd_rz(__fmul_rz(M[0], fo0), __fmul_rz(M[1], fo1)), __fmul_rz(M[2], fo2)), scale), q.t[0]);
        float pzy = __fadd_rz(__fmul_rz(__fadd_rz(__fadd_rz(__fmul_rz(M[3], fo0), __fmul_rz(M[4], fo1)), __fmul_rz(M[5], fo2)), scale), q.t[1]);
        float pzz = __fadd_rz(__fmul_rz(__fadd_rz(__fadd_rz(__fmul_rz(M[6], fo0), __fmul_rz(M[7], fo1)), __fmul_rz(M[8], fo2)), scale), q.t[2]);
        const float d12 = __fmul_rz(M[1], fls), d22 = __fmul_rz(M[4], fls), d32 = __fmul_rz(M[7], fls);
        const float d13 = __fmul_rz(M[2], fls), d23 = __fmul_rz(M[5], fls), d33 = __fmul_rz(M[8], fls);
        const int r = v & 63, rz = r >> 3, ry = r & 7;
        for (int i = 0; i < rz; i++) {
          pzx = __fadd_rz(pzx, d13);
          pzy = __fadd_rz(pzy, d23);
          pzz = __fadd_rz(pzz, d33);
        }
        for (int i = 0; i < ry; i++) {
          pzx = __fadd_rz(pzx, d12);
          pzy = __fadd_rz(pzy, d22);
          pzz = __fadd_rz(pzz, d32);
        }
        rows[j][r] = make_float3(pzx, pzy, pzz);
        if (r == 0) xstep[j] = make_float3(__fmul_rz(M[0], fls), __fmul_rz(M[3], fls), __fmul_rz(M[6], fls));
      }
    }
    __syncthreads();
    const float thrD = __fmul_rz(thr, ls);
    const float thrW = __fmul_rz(__fmul_rz(WEIGHT_FACTOR, thr), ls);
    // the fall-off's reciprocal depends on the brick only, not on the frame
    const float rcp_fall = rcp_upd<RCP_HOST>(__fsub_rz(thrW, DIST_W_EPS), rtab, rshift);
    const float fx_ = (float)x;
    // Frame k's sample of this voxel: the projection and the image reads,
    // issued one frame ahead so that they overlap the previous frame's
    // update (which they do not depend on).
    struct Sample {
      float len, rc;
      bool in;  // in front of the camera and inside the image
      uint16_t draw;
      uint8_t cr, cg, cb;
      float cw;
    };
    auto fetch = [&](int k, Sample &sm) {
      const int j = order[k];
      const FuseSlot &S = fb.s[j];
      const float3 rb = rows[j][z * 8 + y];
      const float3 d1 = xstep[j];
      // lane offsets 0, d, 2d, ..., 7d of the 8-wide rows
      const float kx = x == 0 ? 0.0f : (x == 1 ? d1.x : __fmul_rz(fx_, d1.x));
      const float ky = x == 0 ? 0.0f : (x == 1 ? d1.y : __fmul_rz(fx_, d1.y));
      const float kz = x == 0 ? 0.0f : (x == 1 ? d1.z : __fmul_rz(fx_, d1.z));
      const float px = __fadd_rz(rb.x, kx), py = __fadd_rz(rb.y, ky), pz = __fadd_rz(rb.z, kz);
      const int W = S.W, H = S.H;
      sm.len = __fsqrt_rz(__fadd_rz(__fadd_rz(__fmul_rz(px, px), __fmul_rz(py, py)), __fmul_rz(pz, pz)));
      sm.rc = rcp_upd<RCP_HOST>(pz, rtab, rshift);
      const int imx = cvt_x86_rz(__fadd_rz(S.q.cx, __fmul_rz(S.q.fx, __fmul_rz(px, sm.rc))));
      const int imy = cvt_x86_rz(__fadd_rz(S.q.cy, __fmul_rz(S.q.fy, __fmul_rz(py, sm.rc))));
      sm.in = pz > 0.0f && imy < H && imy > -1 && imx < W && imx > -1;
      const int cyi = max(min(imy, H - 1), 0);
      const int cxi = max(min(imx, W - 1), 0);
      const int ii = W * cyi + cxi;
      sm.draw = __ldg(S.depth + ii);
      const uint8_t *p8 = S.bgr + 3 * (size_t)ii;
      sm.cr = __ldg(p8 + 2);
      sm.cg = __ldg(p8 + 1);
      sm.cb = __ldg(p8 + 0);
      sm.cw = S.conf ? __ldg(S.conf + ii) : 1.0f;
    };
    Sample cur, nxt;
    if (nk > 0) fetch(0, cur);
    for (int k = 0; k < nk; k++) {
      if (k + 1 < nk) fetch(k + 1, nxt);
      const FuseSlot &S = fb.s[order[k]];
      const float len = cur.len, rc = cur.rc;
      const float h = __fmul_rz(S.scaling, (float)cur.draw);
      const float dInc = __fsub_rz(len, __fmul_rz(__fmul_rz(len, rc), h));
      const bool msk = cur.in && h < S.maxcam;
      const float front = dInc < DIST_W_EPS ? 1.0f : 0.0f;
      const float back = (dInc >= DIST_W_EPS && dInc < thrW) ? 1.0f : 0.0f;
      const float fall = __fmul_rz(__fsub_rz(thrW, dInc), rcp_fall);
      float wInc = msk ? __fadd_rz(front, __fmul_rz(fall, back)) : 0.0f;
      if (S.conf) wInc = __fmul_rz(wInc, cur.cw);
      const float wNew = __fadd_rz(wAcc, wInc);
      const float factor = rcp_upd<RCP_HOST>(__fadd_rz(wNew, wNew <= 0.0f ? 1.0f : 0.0f), rtab, rshift);
      float tr = dInc < thrD ? dInc : thrD;
      const float lo = -thrD;
      tr = tr > lo ? tr : lo;
      const float add = msk ? __fmul_rz(tr, wInc) : 0.0f;
      const float dNew = __fmul_rz(__fadd_rz(__fmul_rz(dAcc, wAcc), add), factor);
      const float inc[3] = {__fmul_rz((float)cur.cr, COLOR_MUL), __fmul_rz((float)cur.cg, COLOR_MUL),
                            __fmul_rz((float)cur.cb, COLOR_MUL)};
#pragma unroll
      for (int c = 0; c < 3; c++) {
        float val = __fmul_rz(__fadd_rz(__fmul_rz((float)acc[c], wAcc), __fmul_rz(inc[c], wInc)), factor);
        val = val < 65280.0f ? val : 65280.0f;
        acc[c] = (uint16_t)__float2int_rz(val);
      }
      // the state as the next frame would load it
      if (FP16) {
        dAcc = __half2float(__float2half_rn(dNew));
        wAcc = __half2float(__float2half_rn(wNew));
      } else {
        dAcc = dNew;
        wAcc = wNew;
      }
      cur = nxt;
    }
    if (FP16) {
      fb.sdf16[vi] = __float2half_rn(dAcc);
      fb.wgt16[vi] = __float2half_rn(wAcc);
    } else {
      fb.sdf[vi] = dAcc;
      fb.wgt[vi] = wAcc;
    }
    cb[0] = acc[0];
    cb[512] = acc[1];
    cb[1024] = acc[2];
    if (v == 0) fb.mask[brick] = 0u;  // the next pass starts from an empty mask
    __syncthreads();                   // (shared state of this brick reused by the next)
  }
  if (blockIdx.x == 0 && v == 0) atomicAdd(fb.total, (unsigned long long)total);
}

void launch_fuse_multi(const FuseBatch &fb, int storage, bool rcp_host, int grid, cudaStream_t s) {
  if (grid <= 0) return;
  note_launch();
  if (storage == 1) {
    if (rcp_host) k_fuse_multi<true, true><<<grid, 512, 0, s>>>(fb);
    else k_fuse_multi<true, false><<<grid, 512, 0, s>>>(fb);
  } else {
    if (rcp_host) k_fuse_multi<false, true><<<grid, 512, 0, s>>>(fb);
    else k_fuse_multi<false, false><<<grid, 512, 0, s>>>(fb);
  }
}

// ---------------------------------------------------------------------------
// Halo exchange of a sharded map: the bricks a part owns whose voxels changed
// since its last export, as records (uint32 leaf index, 12 bytes of padding,
// then SDF, weight and colour planes as the pool stores them), and their
// import into another part's pool.
// ---------------------------------------------------------------------------

size_t halo_record_bytes(bool fp16) { return 16 + 512 * (fp16 ? 4 : 8) + 512 * 6; }

__global__ void k_halo_select(const ushort4 *__restrict__ leaf, const uint32_t *__restrict__ stamp, uint32_t nleaves,
                              uint32_t since, uint32_t shard, uint32_t shards, int3 shift, uint32_t *list,
                              uint32_t *count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  bool take = false;
  if (i < nleaves && stamp[i] > since) {
    const ushort4 p = leaf[i];
    const int32_t sh[3] = {shift.x, shift.y, shift.z};
    take = shards <= 1 || shard_hash(p.x, p.y, p.z, (uint32_t)p.w * 8u, 0u, sh) % shards == shard;
  }
  // one claim per warp
  const unsigned b = __ballot_sync(0xffffffffu, take);
  if (!b) return;
  const int lane = threadIdx.x & 31, leader = __ffs(b) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(b));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (take) list[base + __popc(b & ((1u << lane) - 1u))] = i;
}

template <bool FP16>
__global__ void __launch_bounds__(512) k_halo_pack(const uint32_t *__restrict__ list, uint32_t n,
                                                   const float *__restrict__ sdf, const float *__restrict__ wgt,
                                                   const __half *__restrict__ sdf16,
                                                   const __half *__restrict__ wgt16,
                                                   const uint16_t *__restrict__ col, uint8_t *out, size_t rec) {
  const int t = threadIdx.x;
  for (uint32_t r = blockIdx.x; r < n; r += gridDim.x) {
    const uint32_t b = list[r];
    uint8_t *p = out + (size_t)r * rec;
    if (t < 4) reinterpret_cast<uint32_t *>(p)[t] = t == 0 ? b : 0u;
    const size_t vi = (size_t)b * 512 + t;
    uint8_t *q = p + 16;
    if (FP16) {
      reinterpret_cast<__half *>(q)[t] = sdf16[vi];
      reinterpret_cast<__half *>(q + 1024)[t] = wgt16[vi];
      q += 2048;
    } else {
      reinterpret_cast<float *>(q)[t] = sdf[vi];
      reinterpret_cast<float *>(q + 2048)[t] = wgt[vi];
      q += 4096;
    }
    const uint16_t *cb = col + (size_t)b * 1536;
    uint16_t *cq = reinterpret_cast<uint16_t *>(q);
    cq[t] = cb[t];
    cq[512 + t] = cb[512 + t];
    cq[1024 + t] = cb[1024 + t];
  }
}

template <bool FP16>
__global__ void __launch_bounds__(512) k_halo_unpack(const uint8_t *in, uint64_t n, uint32_t leaves_max, float *sdf,
                                                     float *wgt, __half *sdf16, __half *wgt16, uint16_t *col,
                                                     size_t rec) {
  const int t = threadIdx.x;
  for (uint64_t r = blockIdx.x; r < n; r += gridDim.x) {
    const uint8_t *p = in + (size_t)r * rec;
    const uint32_t b = reinterpret_cast<const uint32_t *>(p)[0];
    if (b >= leaves_max) continue;  // not a brick of this map's pool
    const size_t vi = (size_t)b * 512 + t;
    const uint8_t *q = p + 16;
    if (FP16) {
      sdf16[vi] = reinterpret_cast<const __half *>(q)[t];
      wgt16[vi] = reinterpret_cast<const __half *>(q + 1024)[t];
      q += 2048;
    } else {
      sdf[vi] = reinterpret_cast<const float *>(q)[t];
      wgt[vi] = reinterpret_cast<const float *>(q + 2048)[t];
      q += 4096;
    }
    const uint16_t *cq = reinterpret_cast<const uint16_t *>(q);
    uint16_t *cb = col + (size_t)b * 1536;
    cb[t] = cq[t];
    cb[512 + t] = cq[512 + t];
    cb[1024 + t] = cq[1024 + t];
  }
}

void launch_halo_select(const ushort4 *leaf, const uint32_t *stamp, uint32_t nleaves, uint32_t since,
                        uint32_t shard, uint32_t shards, const int32_t shift[3], uint32_t *list, uint32_t *count,
                        cudaStream_t s) {
  if (!nleaves) return;
  note_launch();
  k_halo_select<<<(nleaves + 255) / 256, 256, 0, s>>>(leaf, stamp, nleaves, since, shard, shards,
                                                      make_int3(shift[0], shift[1], shift[2]), list, count);
}

void launch_halo_pack(const uint32_t *list, uint32_t n, const float *sdf, const float *wgt, const __half *sdf16,
                      const __half *wgt16, const uint16_t *col, void *out, bool fp16, int grid, cudaStream_t s) {
  if (!n) return;
  note_launch();
  const size_t rec = halo_record_bytes(fp16);
  if (fp16)
    k_halo_pack<true><<<grid, 512, 0, s>>>(list, n, sdf, wgt, sdf16, wgt16, col, (uint8_t *)out, rec);
  else
    k_halo_pack<false><<<grid, 512, 0, s>>>(list, n, sdf, wgt, sdf16, wgt16, col, (uint8_t *)out, rec);
}

void launch_halo_unpack(const void *in, uint64_t n, uint32_t leaves_max, float *sdf, float *wgt, __half *sdf16,
                        __half *wgt16, uint16_t *col, bool fp16, int grid, cudaStream_t s) {
  if (!n) return;
  note_launch();
  const size_t rec = halo_record_bytes(fp16);
  if (fp16)
    k_halo_unpack<true><<<grid, 512, 0, s>>>((const uint8_t *)in, n, leaves_max, sdf, wgt, sdf16, wgt16, col, rec);
  else
    k_halo_unpack<false><<<grid, 512, 0, s>>>((const uint8_t *)in, n, leaves_max, sdf, wgt, sdf16, wgt16, col, rec);
}

// ---------------------------------------------------------------------------
// Loop closure: removing a fused frame's contribution into separate loop
// arrays (the reference's deleteOldLoopPoses, geometryfusion_mipmap_cpu.cpp:
// 3933-4025, with updateWrapper_deleteloop / update8AddLoopSSESingleDeleteloop,
// loopclosure.cpp:15-309).
// ---------------------------------------------------------------------------

// Slots of the frame's queued bricks in the loop arrays, in queue order: a
// brick without a slot gets the next one (updateWrapper_deleteloop,
// loopclosure.cpp:281-289).  When the slots run out, that entry and every
// later one are left out (the reference returns there).  One block;
// st[0] = slots in use (in and out), st[1] = entries taken.
__global__ void __launch_bounds__(1024) k_loop_slots(const uint32_t *__restrict__ queue, uint32_t nq, uint32_t *map,
                                                     uint32_t capacity, uint32_t *slots, uint32_t *st) {
  __shared__ uint32_t warp_sum[32];
  __shared__ uint32_t s_base, s_stop;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  if (t == 0) {
    s_base = st[0];
    s_stop = nq;
  }
  __syncthreads();
  for (uint32_t c0 = 0; c0 < nq; c0 += 1024) {
    const uint32_t i = c0 + t;
    uint32_t b = 0, cur = 0;
    bool fresh = false;
    if (i < nq) {
      b = queue[i];
      cur = map[b];
      fresh = cur >= s_base;  // no slot yet (slots below the count in use are taken)
    }
    // exclusive prefix of the fresh entries of this chunk
    const unsigned bal = __ballot_sync(0xffffffffu, fresh);
    if (lane == 0) warp_sum[w] = __popc(bal);
    __syncthreads();
    if (w == 0) {
      uint32_t v = warp_sum[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
      }
      warp_sum[lane] = v;  // inclusive
    }
    __syncthreads();
    const uint32_t before = (w ? warp_sum[w - 1] : 0u) + __popc(bal & ((1u << lane) - 1u));
    const uint32_t chunk_fresh = warp_sum[31];
    if (i < nq) {
      const uint32_t base = s_base;
      if (fresh) {
        const uint32_t slot = base + before;
        if (slot >= capacity) {
          atomicMin(&s_stop, i);
        } else {
          map[b] = slot;
          slots[i] = slot;
        }
      } else {
        slots[i] = cur;
      }
    }
    __syncthreads();
    // slots are handed out consecutively, so the ones given are exactly those
    // below the capacity; entries past the first one that found none are left
    // out (fresh ones there received no slot)
    if (t == 0) s_base = min(s_base + chunk_fresh, capacity);
    __syncthreads();
    if (s_stop < nq) break;
  }
  if (t == 0) {
    st[0] = s_base;
    st[1] = s_stop;
  }
}

template <bool RCP_HOST>
__global__ void __launch_bounds__(512) k_loop_delete(LoopFrame L) {
  const int v = threadIdx.x;
  const int x = v & 7, y = (v >> 3) & 7, z = v >> 6;
  const uint32_t n = *L.taken;
  const CamF &q = L.q;
  const float *M = q.r;
  for (uint32_t e = blockIdx.x; e < n; e += gridDim.x) {
    const uint32_t brick = L.queue[e];
    const uint32_t slot = L.slots[e];
    const ushort4 o = L.leaf[brick];
    const float ls = (float)o.w;
    const float fls = __fmul_rz(ls, L.scale);
    const float fo0 = (float)o.x, fo1 = (float)o.y, fo2 = (float)o.z;
    float pzx = __fadd_rz(__fmul_rz(__fadd_rz(__fadd_rz(__fmul_rz(M[0], fo0), __fmul_rz(M[1], fo1)), __fmul_rz(M[2], fo2)), L.scale), q.t[0]);
    float pzy = __fadd_rz(__fmul_rz(__fadd_rz(__fadd_rz(__fmul_rz(M[3], fo0), __fmul_rz(M[4], fo1)), __fmul_rz(M[5], fo2)), L.scale), q.t[1]);
    float pzz = __fadd_rz(__fmul_rz(__fadd_rz(__fadd_rz(__fmul_rz(M[6], fo0), __fmul_rz(M[7], fo1)), __fmul_rz(M[8], fo2)), L.scale), q.t[2]);
    const float d11 = __fmul_rz(M[0], fls), d21 = __fmul_rz(M[3], fls), d31 = __fmul_rz(M[6], fls);
    const float d12 = __fmul_rz(M[1], fls), d22 = __fmul_rz(M[4], fls), d32 = __fmul_rz(M[7], fls);
    const float d13 = __fmul_rz(M[2], fls), d23 = __fmul_rz(M[5], fls), d33 = __fmul_rz(M[8], fls);
    for (int i = 0; i < z; i++) {
      pzx = __fadd_rz(pzx, d13);
      pzy = __fadd_rz(pzy, d23);
      pzz = __fadd_rz(pzz, d33);
    }
    for (int i = 0; i < y; i++) {
      pzx = __fadd_rz(pzx, d12);
      pzy = __fadd_rz(pzy, d22);
      pzz = __fadd_rz(pzz, d32);
    }
    // 4-wide rows: lanes 0, d, 2d, 3d from the row start, the second half
    // from the start advanced by 4d (loopclosure.cpp:40-60)
    if (x >= 4) {
      pzx = __fadd_rz(pzx, __fmul_rz(d11, 4.0f));
      pzy = __fadd_rz(pzy, __fmul_rz(d21, 4.0f));
      pzz = __fadd_rz(pzz, __fmul_rz(d31, 4.0f));
    }
    const int l = x & 3;
    const float kx = l == 0 ? 0.0f : (l == 1 ? d11 : __fmul_rz((float)l, d11));
    const float ky = l == 0 ? 0.0f : (l == 1 ? d21 : __fmul_rz((float)l, d21));
    const float kz = l == 0 ? 0.0f : (l == 1 ? d31 : __fmul_rz((float)l, d31));
    const float px = __fadd_rz(pzx, kx), py = __fadd_rz(pzy, ky), pz = __fadd_rz(pzz, kz);
    const int W = L.W, H = L.H;
    const float len = __fsqrt_rz(__fadd_rz(__fadd_rz(__fmul_rz(px, px), __fmul_rz(py, py)), __fmul_rz(pz, pz)));
    const float rc = rcp_upd<RCP_HOST>(pz, L.rcp_tab, L.rcp_shift);
    const int imx = cvt_x86_rz(__fadd_rz(q.cx, __fmul_rz(q.fx, __fmul_rz(px, rc))));
    const int imy = cvt_x86_rz(__fadd_rz(q.cy, __fmul_rz(q.fy, __fmul_rz(py, rc))));
    const int ii = W * max(min(imy, H - 1), 0) + max(min(imx, W - 1), 0);
    const float h = __ldg(L.depth + ii);
    const float rI = __fmul_rz((float)__ldg(L.red + ii), COLOR_MUL);
    const float gI = __fmul_rz((float)__ldg(L.green + ii), COLOR_MUL);
    const float bI = __fmul_rz((float)__ldg(L.blue + ii), COLOR_MUL);
    const float dInc = __fsub_rz(len, __fmul_rz(__fmul_rz(len, rc), h));
    // no maximum distance here; a hole (NaN depth) fails the ordered test
    const bool msk = pz > 0.0f && imy < H && imy > -1 && imx < W && imx > -1 && !isnan(dInc);
    const float thrD = __fmul_rz(L.thr, ls);
    const float thrW = __fmul_rz(__fmul_rz(WEIGHT_FACTOR, L.thr), ls);
    const float front = dInc < DIST_W_EPS ? 1.0f : 0.0f;
    const float back = (dInc >= DIST_W_EPS && dInc < thrW) ? 1.0f : 0.0f;
    // the fall-off with its sign turned (loopclosure.cpp:166-172)
    const float fall =
        __fmul_rz(__fsub_rz(dInc, thrW), rcp_upd<RCP_HOST>(__fsub_rz(thrW, DIST_W_EPS), L.rcp_tab, L.rcp_shift));
    const float wInc = msk ? __fadd_rz(front, __fmul_rz(fall, back)) : 0.0f;
    const size_t vi = (size_t)slot * 512 + v;
    const float wAcc = L.wgt[vi], dAcc = L.sdf[vi];
    const float wNew = __fadd_rz(wAcc, wInc);
    const float factor = rcp_upd<RCP_HOST>(__fadd_rz(wNew, wNew <= 0.0f ? 1.0f : 0.0f), L.rcp_tab, L.rcp_shift);
    const float mn = thrD < dInc ? thrD : dInc;                    // _mm_min_ps(thrD, dInc)
    const float lo = __fmul_rz(-1.0f, thrD);
    const float tr = lo > mn ? lo : mn;                            // _mm_max_ps(-thrD, min)
    const float add = msk ? __fmul_rz(tr, wInc) : 0.0f;
    L.sdf[vi] = __fmul_rz(__fadd_rz(__fmul_rz(dAcc, wAcc), add), factor);
    L.wgt[vi] = wNew;
    uint16_t *cb = L.col + (size_t)slot * 1536 + v;
    const float inc[3] = {rI, gI, bI};
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float acc = (float)cb[c * 512];
      const float val = __fmul_rz(__fadd_rz(__fmul_rz(acc, wAcc), __fmul_rz(inc[c], wInc)), factor);
      // the float -> unsigned short store of the reference (no clamp): a
      // truncating conversion to int, of which the low 16 bits are kept
      cb[c * 512] = (uint16_t)cvt_x86_rz(val);
    }
  }
}

void launch_loop_slots(const uint32_t *queue, uint32_t nq, uint32_t *map, uint32_t capacity, uint32_t *slots,
                       uint32_t *st, cudaStream_t s) {
  note_launch();
  k_loop_slots<<<1, 1024, 0, s>>>(queue, nq, map, capacity, slots, st);
}

void launch_loop_delete(const LoopFrame &L, bool rcp_host, int grid, cudaStream_t s) {
  note_launch();
  if (rcp_host) k_loop_delete<true><<<grid, 512, 0, s>>>(L);
  else k_loop_delete<false><<<grid, 512, 0, s>>>(L);
}

// Block shapes of the voxel update: (bricks per block, blocks per SM the
// register budget is cut for).  Shape 0 is the default.
static const int FUSE_SHAPES[FUSE_SHAPE_COUNT][2] = {{1, 4}, {1, 3}, {2, 2}, {2, 1}};

template <bool F16, bool RH>
static void launch_fuse_shape(const BatchDesc *d_batch, int g, int grid, int shape, cudaStream_t s) {
  switch (shape) {
    case 1: k_fuse<F16, RH, 1, 3><<<grid, 512, 0, s>>>(d_batch, g); break;
    case 2: k_fuse<F16, RH, 2, 2><<<grid, 1024, 0, s>>>(d_batch, g); break;
    case 3: k_fuse<F16, RH, 2, 1><<<grid, 1024, 0, s>>>(d_batch, g); break;
    default: k_fuse<F16, RH, 1, 4><<<grid, 512, 0, s>>>(d_batch, g); break;
  }
}

void launch_fuse(const BatchDesc *d_batch, int nmaps, bool gated, int storage, bool rcp_host, int grid,
                 cudaStream_t s, int shape) {
  if (grid <= 0 || nmaps < 1) return;
  const int g = gated ? 1 : 0;
  note_launch();
  if (storage == 1) {
    if (rcp_host) launch_fuse_shape<true, true>(d_batch, g, grid, shape, s);
    else launch_fuse_shape<true, false>(d_batch, g, grid, shape, s);
  } else {
    if (rcp_host) launch_fuse_shape<false, true>(d_batch, g, grid, shape, s);
    else launch_fuse_shape<false, false>(d_batch, g, grid, shape, s);
  }
}

int fuse_shape_bricks(int shape) { return FUSE_SHAPES[(shape >= 0 && shape < FUSE_SHAPE_COUNT) ? shape : 0][0]; }

// Measure the host CPU's RCPPS for every mantissa of [1,2) and check the
// exponent/sign/special-value rules that rcp_host() relies on.
bool build_rcp_table(std::vector<uint32_t> &tab, int &shift) {
#if defined(__x86_64__) || defined(_M_X64)
  tab.resize(1u << 23);
  for (uint32_t m = 0; m < (1u << 23); m += 4) {
    float x[4];
    for (int k = 0; k < 4; k++) {
      uint32_t u = (127u << 23) | (m + k);
      memcpy(&x[k], &u, 4);
    }
    __m128 r = _mm_rcp_ps(_mm_loadu_ps(x));
    _mm_storeu_ps(reinterpret_cast<float *>(&tab[m]), r);
  }
  auto bits = [](float f) { uint32_t u; memcpy(&u, &f, 4); return u; };
  auto rcp1 = [](float f) { return _mm_cvtss_f32(_mm_rcp_ss(_mm_set_ss(f))); };
  for (int e = 1; e < 255; e += 7) {
    for (uint32_t m = 0; m < (1u << 23); m += 65537) {
      uint32_t u = ((uint32_t)e << 23) | m;
      float x;
      memcpy(&x, &u, 4);
      uint32_t t = tab[m];
      int te = (int)((t >> 23) & 255u) - (e - 127);
      uint32_t pred = te <= 0 ? 0u : ((t & 0x7fffffu) | ((uint32_t)te << 23));
      if (bits(rcp1(x)) != pred || bits(rcp1(-x)) != (pred | 0x80000000u)) return false;
    }
  }
  if (bits(rcp1(0.0f)) != 0x7f800000u || bits(rcp1(1e-40f)) != 0x7f800000u) return false;
  if (bits(rcp1(__builtin_inff())) != 0u) return false;
  // keep only the mantissa bits the result depends on (the instruction is a
  // table lookup on the leading bits: 11 of them on recent Intel cores), so
  // the device table stays small enough to live in L1
  shift = 0;
  for (int sh = 23; sh > 0; sh--) {
    const uint32_t low = (1u << sh) - 1u;
    bool same = true;
    for (uint32_t m = 0; m < (1u << 23) && same; m++) same = tab[m] == tab[m & ~low];
    if (same) {
      shift = sh;
      break;
    }
  }
  if (shift) {
    std::vector<uint32_t> c(1u << (23 - shift));
    for (uint32_t i = 0; i < c.size(); i++) c[i] = tab[(size_t)i << shift];
    tab.swap(c);
  }
  return true;
#else
  (void)tab;
  shift = 0;
  return false;
#endif
}

cudaError_t prewarm_fuse_kernels() {
  const void *fns[] = {(const void *)k_fuse<false, false, 1, 4>, (const void *)k_fuse<false, true, 1, 4>,
                       (const void *)k_fuse<true, false, 1, 4>,  (const void *)k_fuse<true, true, 1, 4>,
                       (const void *)k_fuse_multi<false, false>, (const void *)k_fuse_multi<false, true>,
                       (const void *)k_fuse_multi<true, false>,  (const void *)k_fuse_multi<true, true>};
  for (const void *f : fns) {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, f);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace ffb
