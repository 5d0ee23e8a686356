// Per-voxel SDF / weight / colour fusion of the queued bricks.
//
// Restates update8AddLoopAVXSingleInteger (reference update_functions.cpp:1187-1444)
// as run by updateWrapperInteger (:1633-1732): every operation in
// round-toward-zero (the reference sets MXCSR=RZ, :1678-1679) with the
// reference's operation order, voxel positions accumulated the way the
// reference's loops accumulate them (z steps, then y steps, then x * step),
// and exact RZ reciprocals (__frcp_rz) in place of _mm256_rcp_ps.
// Every voxel of every queued brick is read and written, like the reference.
//
// One CTA per brick, one thread per voxel: the 512 SDF and weight words of a
// brick and its three 512-entry colour planes are contiguous, so each load and
// store is a fully coalesced 2 KB / 1 KB segment.
#include "ff_kernels.h"

namespace ffb {

// x86 float->int32 under round-toward-zero (truncation; 0x80000000 when out
// of range), the behaviour of _mm256_cvtps_epi32 with MXCSR=RZ.
__device__ __forceinline__ int cvt_x86_rz(float f) {
  if (!(f > -2147483904.0f && f < 2147483648.0f)) return (int)0x80000000;
  return __float2int_rz(f);
}

template <bool FP16>
__global__ void __launch_bounds__(512) k_fuse(const uint32_t *__restrict__ queue, const ushort4 *__restrict__ leaf,
                                              float *__restrict__ sdf, float *__restrict__ wgt,
                                              __half *__restrict__ sdf16, __half *__restrict__ wgt16,
                                              uint16_t *__restrict__ col, uint32_t leaves_max,
                                              const uint16_t *__restrict__ depth, const uint8_t *__restrict__ bgr,
                                              int W, int H, CamF q, float scale, float thr, float scaling,
                                              float maxcam) {
  const uint32_t brick = queue[blockIdx.x];
  const int v = threadIdx.x;
  const int x = v & 7, y = (v >> 3) & 7, z = v >> 6;
  const ushort4 o = leaf[brick];
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
  const float rc = __frcp_rz(pz);
  const int imx = cvt_x86_rz(__fadd_rz(q.cx, __fmul_rz(q.fx, __fmul_rz(px, rc))));
  const int imy = cvt_x86_rz(__fadd_rz(q.cy, __fmul_rz(q.fy, __fmul_rz(py, rc))));
  const int cyi = max(min(imy, H - 1), 0);
  const int cxi = max(min(imx, W - 1), 0);
  const int ii = W * cyi + cxi;
  const float h = __fmul_rz(scaling, (float)__ldg(depth + ii));
  const float dInc = __fsub_rz(len, __fmul_rz(__fmul_rz(len, rc), h));
  const bool mask = pz > 0.0f && imy < H && imy > -1 && imx < W && imx > -1 && h < maxcam;
  const float thrD = __fmul_rz(thr, ls);
  const float thrW = __fmul_rz(__fmul_rz(WEIGHT_FACTOR, thr), ls);
  const float front = dInc < DIST_W_EPS ? 1.0f : 0.0f;
  const float back = (dInc >= DIST_W_EPS && dInc < thrW) ? 1.0f : 0.0f;
  const float fall = __fmul_rz(__fsub_rz(thrW, dInc), __frcp_rz(__fsub_rz(thrW, DIST_W_EPS)));
  const float wInc = mask ? __fadd_rz(front, __fmul_rz(fall, back)) : 0.0f;

  const size_t vi = (size_t)brick * 512 + v;
  float wAcc, dAcc;
  if (FP16) {
    wAcc = __half2float(wgt16[vi]);
    dAcc = __half2float(sdf16[vi]);
  } else {
    wAcc = wgt[vi];
    dAcc = sdf[vi];
  }
  const float wNew = __fadd_rz(wAcc, wInc);
  const float factor = __frcp_rz(__fadd_rz(wNew, wNew <= 0.0f ? 1.0f : 0.0f));
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
  const uint8_t *p8 = bgr + 3 * (size_t)ii;
  const float inc[3] = {__fmul_rz((float)__ldg(p8 + 2), COLOR_MUL), __fmul_rz((float)__ldg(p8 + 1), COLOR_MUL),
                        __fmul_rz((float)__ldg(p8 + 0), COLOR_MUL)};
  uint16_t *cb = col + (size_t)brick * 1536 + v;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float acc = (float)cb[c * 512];
    float val = __fmul_rz(__fadd_rz(__fmul_rz(acc, wAcc), __fmul_rz(inc[c], wInc)), factor);
    val = val < 65280.0f ? val : 65280.0f;
    cb[c * 512] = (uint16_t)__float2int_rz(val);
  }
}

void launch_fuse(const uint32_t *queue, int nq, const ushort4 *leaf, float *sdf, float *wgt, __half *sdf16,
                 __half *wgt16, uint16_t *col, int storage, uint32_t leaves_max, const uint16_t *depth,
                 const uint8_t *bgr, int W, int H, const CamF &q, float scale, float thr, float scaling,
                 float maxcam, cudaStream_t s) {
  if (nq <= 0) return;
  if (storage == 1)
    k_fuse<true><<<nq, 512, 0, s>>>(queue, leaf, sdf, wgt, sdf16, wgt16, col, leaves_max, depth, bgr, W, H, q,
                                    scale, thr, scaling, maxcam);
  else
    k_fuse<false><<<nq, 512, 0, s>>>(queue, leaf, sdf, wgt, sdf16, wgt16, col, leaves_max, depth, bgr, W, H, q,
                                     scale, thr, scaling, maxcam);
}

}  // namespace ffb
