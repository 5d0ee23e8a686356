// Learned per-pixel confidence weight: a 3-layer 5x5 CNN (16 channels) with
// BF16 weights and activations and FP32 accumulation, its training kernels
// (backward of every layer, MSE loss, Adam), the input features, and a
// raycaster of the fused volume that gives the training targets.
//
// There is no counterpart in the reference: its fusion weight is the fixed
// distance ramp of update_functions.cpp:1187-1444.  The learned weight
// multiplies that ramp's weight increment per pixel; with no network set the
// update is the reference's, bit for bit.
//
// Layout in HBM (n images of W x H, pixel-major, channels innermost):
//   features  bf16 [n][H][W][8]   depth (m), normal (x, y, z), valid, 0, 0, 0
//   a1, a2    bf16 [n][H][W][16]  post-ReLU activations of layers 1 and 2
//   pred      f32  [n][H][W]      layer 3 output: predicted |depth residual| in cm
//   params    bf16 [8833]         W1[16][5][25] b1[16] W2[16][16][25] b2[16] W3[1][16][25] b3[1]
// Convolutions are 'same' 5x5 correlations with zero padding per image.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <mutex>

#include "ff_common.cuh"
#include "ff_kernels.h"

namespace ffb {

constexpr int CNN_HID = 16;
constexpr int CNN_IN = 5;
constexpr int CNN_IN_STRIDE = 8;
constexpr int TAPS = 25;
constexpr int P_W1 = 0, P_B1 = P_W1 + CNN_HID * CNN_IN * TAPS, P_W2 = P_B1 + CNN_HID,
              P_B2 = P_W2 + CNN_HID * CNN_HID * TAPS, P_W3 = P_B2 + CNN_HID, P_B3 = P_W3 + CNN_HID * TAPS,
              P_TOTAL = P_B3 + 1;
static_assert(P_TOTAL == CNN_PARAMS && CNN_HID == CNN_HIDDEN && CNN_IN_STRIDE == CNN_FEAT_CH, "parameter layout");
static_assert(CNN_PACKED_BYTES == 65 * 512, "packed operand bytes");

// output tile of a convolution block: 32 x 16 pixels, 256 threads, two
// pixels (rows ty and ty + 8) per thread; input tile with a 2-pixel halo,
// one plane per channel, planes padded to an odd length so that threads
// reading different channels hit different banks
constexpr int TX = 32, TY = 16, SX = TX + 4, SY = TY + 4, PLANE = SX * SY + 1;
constexpr int GPLANE = TX * TY + 1;

enum ConvMode { CONV_RELU_BF16 = 0, CONV_F32 = 1, CONV_CONF = 2, CONV_MASK_F32 = 3 };

__device__ __forceinline__ float to_f(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float to_f(float v) { return v; }

// KIN channels of one pixel (CSTR elements apart) into v[]
template <int KIN, int CSTR, typename T>
__device__ __forceinline__ void load_px(const T *__restrict__ p, float *v) {
  if constexpr (sizeof(T) == 2 && CSTR % 8 == 0) {
    constexpr int NV = (KIN + 7) / 8;
#pragma unroll
    for (int k = 0; k < NV; k++) {
      const uint4 u = __ldg(reinterpret_cast<const uint4 *>(p) + k);
      const __nv_bfloat16 *b = reinterpret_cast<const __nv_bfloat16 *>(&u);
#pragma unroll
      for (int j = 0; j < 8; j++)
        if (k * 8 + j < KIN) v[k * 8 + j] = __bfloat162float(b[j]);
    }
  } else if constexpr (sizeof(T) == 4 && CSTR % 4 == 0 && KIN % 4 == 0) {
#pragma unroll
    for (int k = 0; k < KIN / 4; k++) {
      const float4 u = __ldg(reinterpret_cast<const float4 *>(p) + k);
      v[4 * k] = u.x;
      v[4 * k + 1] = u.y;
      v[4 * k + 2] = u.z;
      v[4 * k + 3] = u.w;
    }
  } else {
#pragma unroll
    for (int c = 0; c < KIN; c++) v[c] = to_f(p[c]);
  }
}

// The input tile of block (x0, y0) of image img: KIN planes of SX x SYT
// (PLANET floats apart).
template <int KIN, int CSTR, typename T, int SYT = SY, int PLANET = PLANE>
__device__ __forceinline__ void load_tile(const T *__restrict__ in, int img, int W, int H, int x0, int y0,
                                          float *s_in) {
  const size_t base = (size_t)img * W * H;
  for (int i = threadIdx.x; i < SX * SYT; i += blockDim.x) {
    const int gx = x0 + i % SX - 2, gy = y0 + i / SX - 2;
    float v[KIN];
    if (gx >= 0 && gx < W && gy >= 0 && gy < H) {
      load_px<KIN, CSTR>(in + (base + (size_t)gy * W + gx) * CSTR, v);
    } else {
#pragma unroll
      for (int c = 0; c < KIN; c++) v[c] = 0.0f;
    }
#pragma unroll
    for (int c = 0; c < KIN; c++) s_in[c * PLANET + i] = v[c];
  }
}

// Convolution tiles: 32 x (8 * RPT) output pixels, RPT rows per thread.
constexpr int CONV_RPT = 4;
__host__ __device__ constexpr int conv_ty(int rpt) { return 8 * rpt; }
__host__ __device__ constexpr int conv_plane(int rpt) { return SX * (conv_ty(rpt) + 4) + 1; }
__host__ __device__ constexpr int w_offset(int kin, int rpt) { return (kin * conv_plane(rpt) + 3) & ~3; }

template <int KIN, int KOUT>
constexpr size_t conv_smem_bytes() {
  return sizeof(float) * ((size_t)w_offset(KIN, CONV_RPT) + (size_t)KIN * TAPS * KOUT);
}

// One 5x5 convolution layer over a 32 x (8 RPT) tile, each thread RPT
// pixels of one column (rows ty, ty + 8, ...).  KIN channels are read, KOUT
// produced.  TRANS: the gradient of a layer's input -- the layer (KOUT in,
// KIN out) applied transposed, i.e. a correlation with its weights flipped.
// Modes: ReLU to BF16 (forward hidden layers), FP32 (network output), the
// confidence weight (inference), FP32 masked by the ReLU of an activation
// (backward).  FP32 accumulation in channel-major, row, column order; the
// weights of a tap are read as float4 broadcasts shared by the RPT pixels.
template <int KIN, int KOUT, int CSTR, typename TIN, bool TRANS, int MODE>
__global__ void __launch_bounds__(256) k_conv(const TIN *__restrict__ in, int W, int H,
                                              const __nv_bfloat16 *__restrict__ w,
                                              const __nv_bfloat16 *__restrict__ bias, void *__restrict__ out,
                                              const __nv_bfloat16 *__restrict__ act, float inv_tau) {
  constexpr int RPT = CONV_RPT, TYC = conv_ty(RPT), PL = conv_plane(RPT);
  extern __shared__ __align__(16) float smem[];
  float *s_in = smem;
  float *s_w = smem + w_offset(KIN, RPT);  // [KIN][25][KOUT]
  const int img = blockIdx.z;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TYC;
  for (int i = threadIdx.x; i < KIN * TAPS * KOUT; i += blockDim.x) {
    const int co = i % KOUT, rest = i / KOUT, tap = rest % TAPS, ci = rest / TAPS;
    s_w[i] = TRANS ? __bfloat162float(w[(ci * KOUT + co) * TAPS + (TAPS - 1 - tap)])
                   : __bfloat162float(w[(co * KIN + ci) * TAPS + tap]);
  }
  load_tile<KIN, CSTR, TIN, TYC + 4, PL>(in, img, W, H, x0, y0, s_in);
  __syncthreads();
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  float acc[RPT][KOUT];
#pragma unroll
  for (int r = 0; r < RPT; r++)
#pragma unroll
    for (int co = 0; co < KOUT; co++) acc[r][co] = (MODE == CONV_MASK_F32) ? 0.0f : __bfloat162float(bias[co]);
#pragma unroll 1
  for (int ci = 0; ci < KIN; ci++) {
    const float *pl = s_in + ci * PL + ty * SX + tx;
    const float *wc = s_w + ci * TAPS * KOUT;
#pragma unroll
    for (int ky = 0; ky < 5; ky++) {
#pragma unroll
      for (int kx = 0; kx < 5; kx++) {
        float u[RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++) u[r] = pl[(ky + 8 * r) * SX + kx];
        const float *wp = wc + (ky * 5 + kx) * KOUT;
        if constexpr (KOUT % 4 == 0) {
#pragma unroll
          for (int co = 0; co < KOUT; co += 4) {
            const float4 w4 = *reinterpret_cast<const float4 *>(wp + co);
#pragma unroll
            for (int r = 0; r < RPT; r++) {
              acc[r][co] = fmaf(w4.x, u[r], acc[r][co]);
              acc[r][co + 1] = fmaf(w4.y, u[r], acc[r][co + 1]);
              acc[r][co + 2] = fmaf(w4.z, u[r], acc[r][co + 2]);
              acc[r][co + 3] = fmaf(w4.w, u[r], acc[r][co + 3]);
            }
          }
        } else {
#pragma unroll
          for (int co = 0; co < KOUT; co++) {
            const float wv = wp[co];
#pragma unroll
            for (int r = 0; r < RPT; r++) acc[r][co] = fmaf(wv, u[r], acc[r][co]);
          }
        }
      }
    }
  }
  const int gx = x0 + tx;
#pragma unroll
  for (int r = 0; r < RPT; r++) {
    const int gy = y0 + ty + 8 * r;
    if (gx >= W || gy >= H) continue;
    const float *a = acc[r];
    const size_t px = ((size_t)img * H + gy) * W + gx;
    if constexpr (MODE == CONV_RELU_BF16) {
      static_assert(KOUT % 8 == 0, "vector store");
#pragma unroll
      for (int k = 0; k < KOUT / 8; k++) {
        uint4 v;
        __nv_bfloat16 *b = reinterpret_cast<__nv_bfloat16 *>(&v);
#pragma unroll
        for (int j = 0; j < 8; j++) b[j] = __float2bfloat16_rn(fmaxf(a[8 * k + j], 0.0f));
        reinterpret_cast<uint4 *>(reinterpret_cast<__nv_bfloat16 *>(out) + px * KOUT)[k] = v;
      }
    } else if constexpr (MODE == CONV_F32) {
#pragma unroll
      for (int co = 0; co < KOUT; co++) reinterpret_cast<float *>(out)[px * KOUT + co] = a[co];
    } else if constexpr (MODE == CONV_CONF) {
      static_assert(KOUT == 1, "confidence from one channel");
      // (1 - r/tau)^2 on [0, tau], 0 beyond: weight falls to exactly zero for
      // pixels whose predicted residual reaches tau
      const float c = fmaxf(1.0f - fmaxf(a[0], 0.0f) * inv_tau, 0.0f);
      reinterpret_cast<float *>(out)[px] = c * c;
    } else {
      static_assert(KOUT % 8 == 0, "vector load");
#pragma unroll
      for (int k = 0; k < KOUT / 8; k++) {
        const uint4 v = __ldg(reinterpret_cast<const uint4 *>(act + px * KOUT) + k);
        const __nv_bfloat16 *b = reinterpret_cast<const __nv_bfloat16 *>(&v);
        float4 o0, o1;
        o0.x = __bfloat162float(b[0]) > 0.0f ? a[8 * k + 0] : 0.0f;
        o0.y = __bfloat162float(b[1]) > 0.0f ? a[8 * k + 1] : 0.0f;
        o0.z = __bfloat162float(b[2]) > 0.0f ? a[8 * k + 2] : 0.0f;
        o0.w = __bfloat162float(b[3]) > 0.0f ? a[8 * k + 3] : 0.0f;
        o1.x = __bfloat162float(b[4]) > 0.0f ? a[8 * k + 4] : 0.0f;
        o1.y = __bfloat162float(b[5]) > 0.0f ? a[8 * k + 5] : 0.0f;
        o1.z = __bfloat162float(b[6]) > 0.0f ? a[8 * k + 6] : 0.0f;
        o1.w = __bfloat162float(b[7]) > 0.0f ? a[8 * k + 7] : 0.0f;
        float4 *o = reinterpret_cast<float4 *>(reinterpret_cast<float *>(out) + px * KOUT) + 2 * k;
        o[0] = o0;
        o[1] = o1;
      }
    }
  }
}

// ------------------------------------------------ tensor-core convolution
//
// The forward layers as implicit GEMMs on the 5th-generation tensor cores:
// per output row of a 128-pixel strip, D[128 pixels x 16] (FP32, in tensor
// memory) accumulates one tcgen05.mma (M=128, N=16, K=16, BF16) per
// tap (C = 16 input channels: the 16 channels of the tap) or per pair of
// horizontally adjacent taps (C = 8: the 8 channels of two neighbouring
// pixels).  Operands are read by the tensor core straight from shared
// memory through descriptors of the K-major, unswizzled canonical layout:
// 8 x 16-byte core matrices, rows (pixels) 16 bytes apart, 8-row groups 128
// bytes apart (SBO), the two K halves LBO apart -- the two channel planes of
// the tile (C = 16) or the next pixel (C = 8).  A tap's shift is the
// descriptor's start address.  Layer 3 (16 -> 1) runs with N = 16 (the
// smallest N of an M = 128 MMA): output channel 0 real, 1..15 zero weights.
//
// CTA: 128 threads, output tile 128 x TC_ROWS pixels; input tile
// (TC_ROWS + 4) x TC_COLS pixels per plane, brought in with cp.async (zero
// fill outside the image).  One thread issues the MMAs; all wait on an
// mbarrier (bounded) and read the accumulators back with tcgen05.ld (warp
// w: pixels 32w..32w+31).

constexpr int TC_ROWS = 8;               // output rows per CTA
constexpr int TC_COLS = 136;             // 128 + 4 halo + 4 (the pair of taps 4 and 5 reads one more pixel)
constexpr int TC_TILE_ROWS = TC_ROWS + 4;
constexpr int TC_PLANE = TC_TILE_ROWS * TC_COLS * 16;  // bytes of one 8-channel plane
constexpr int TC_WAIT_LIMIT = 1 << 24;

template <int C>
__host__ __device__ constexpr int tc_mmas_per_row() { return C == 16 ? 25 : 15; }
template <int N>
__host__ __device__ constexpr int tc_b_bytes() { return N * 32; }  // one K=16 x N operand (512 B)
// at least 57 KB, so that at most 4 CTAs share an SM: 4 x 128 columns fill
// the 512 of tensor memory, and no allocation has to wait for another CTA
template <int C, int N>
constexpr size_t tc_smem_bytes() {
  return std::max<size_t>((size_t)(C / 8) * TC_PLANE + (size_t)tc_mmas_per_row<C>() * tc_b_bytes<N>() + 64,
                          57 * 1024);
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: K-major, no swizzle (sm_100 version 1)
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

// instruction descriptor: D FP32, A and B BF16, both K-major, M = 128
template <int N>
__host__ __device__ constexpr uint32_t tc_idesc() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((128u >> 4) << 24);
}

// TMA tile loads and a bulk copy, completing on an mbarrier (transaction bytes)
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap *m, int c0, int c1, int c2, int c3,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap *m, int c0, int c1, int c2, int c3,
                                            int c4, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
      "%6}], [%7];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(m)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ uint32_t mbar_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok = 0;
  for (int it = 0; it < TC_WAIT_LIMIT && !ok; it++) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
  }
  return ok;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0) : "memory");
}

// Weight of operand element (n, k) of MMA j: layer with C input channels
// (C = 8: taps paired along x), output channel n.
template <int C>
__device__ __forceinline__ float tc_weight(const __nv_bfloat16 *__restrict__ w, int cin, int cout, int j, int n,
                                           int k) {
  if (n >= cout) return 0.0f;
  if (C == 16) return __bfloat162float(__ldg(w + (n * cin + k) * TAPS + j));
  const int ky = j / 3, kx = 2 * (j % 3) + (k >> 3), ci = k & 7;
  return (kx < 5 && ci < cin) ? __bfloat162float(__ldg(w + (n * cin + ci) * TAPS + ky * 5 + kx)) : 0.0f;
}

// The B operands of all three layers in their shared-memory layout (element
// (n, k) of MMA j at j*512 + (k/8)*256 + (n/8)*128 + (n%8)*16 + (k%8)*2),
// written once per parameter set by k_pack_tc and copied by each CTA.
constexpr int TC_PACK_L1 = 0, TC_PACK_L2 = 15 * 512, TC_PACK_L3 = TC_PACK_L2 + 25 * 512,
              TC_PACK_BYTES = TC_PACK_L3 + 25 * 512;

__global__ void k_pack_tc(const __nv_bfloat16 *__restrict__ params, __nv_bfloat16 *__restrict__ packed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= TC_PACK_BYTES / 2) return;
  const int byte = 2 * i;
  float v;
  int rel, layer;
  if (byte < TC_PACK_L2) rel = byte, layer = 1;
  else if (byte < TC_PACK_L3) rel = byte - TC_PACK_L2, layer = 2;
  else rel = byte - TC_PACK_L3, layer = 3;
  const int j = rel / 512, q = rel % 512;
  const int k = ((q / 256) << 3) | ((q % 16) / 2), n = ((q / 128) % 2) * 8 + (q % 128) / 16;
  if (layer == 1) v = tc_weight<8>(params + P_W1, CNN_IN, CNN_HID, j, n, k);
  else if (layer == 2) v = tc_weight<16>(params + P_W2, CNN_HID, CNN_HID, j, n, k);
  else v = tc_weight<16>(params + P_W3, CNN_HID, 1, j, n, k);
  packed[i] = __float2bfloat16_rn(v);
}

template <int C, int N, int MODE>
__global__ void __launch_bounds__(128) k_conv_tc(const __grid_constant__ CUtensorMap tile, int W, int H,
                                                 const uint8_t *__restrict__ wpack,
                                                 const __nv_bfloat16 *__restrict__ bias, void *__restrict__ out,
                                                 float inv_tau, uint32_t *__restrict__ err) {
  constexpr int NP = C / 8;  // channel planes
  constexpr int NM = tc_mmas_per_row<C>();
  constexpr int BB = tc_b_bytes<N>();
  static_assert(N == 16, "M = 128 MMAs take N in steps of 16");
  constexpr int TMEM_COLS = TC_ROWS * N;  // 128
  extern __shared__ __align__(1024) uint8_t tsm[];
  uint8_t *planes = tsm;                  // NP x [TC_TILE_ROWS][TC_COLS][8] bf16
  uint8_t *wsm = tsm + NP * TC_PLANE;     // NM x [k half][N][8] bf16
  uint64_t *mbar = reinterpret_cast<uint64_t *>(wsm + NM * BB);  // [0], [1]: MMA stages; [2]: loads
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(wsm + NM * BB + 24);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int img = blockIdx.z;
  const int x0 = blockIdx.x * 128, y0 = blockIdx.y * TC_ROWS;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    // stage barriers: one arrival per issuing warp (two warps per stage)
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 2;" ::"r"(smem_addr(mbar)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 2;" ::"r"(smem_addr(mbar + 1)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar + 2)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const size_t img_base = (size_t)img * W * H;
  const uint32_t pbase = smem_addr(planes), wbase = smem_addr(wsm), ld_bar = smem_addr(mbar + 2);
  // the input tile (zero outside the image) and the weight operands, by the
  // tensor-memory-access unit: one tile copy per 8-channel plane, one bulk copy
  if (tid == 0) {
    const uint32_t bytes = (uint32_t)(NP * TC_PLANE + NM * BB);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(ld_bar), "r"(bytes) : "memory");
    if constexpr (C == 16) {
      tma_load_5d(pbase, &tile, 0, 0, x0 - 2, y0 - 2, img, ld_bar);
      tma_load_5d(pbase + TC_PLANE, &tile, 0, 1, x0 - 2, y0 - 2, img, ld_bar);
    } else {
      tma_load_4d(pbase, &tile, 0, x0 - 2, y0 - 2, img, ld_bar);
    }
    bulk_load(wbase, wpack, (uint32_t)(NM * BB), ld_bar);
  }
  const uint32_t loaded = mbar_wait(ld_bar, 0);
  if (!loaded && tid == 0 && err) atomicOr(err, ERR_SPIN_TIMEOUT);

  // MMAs in two stages (output rows 0-3, then 4-7), one mbarrier each, so the
  // read-back of the first overlaps the MMAs of the second; each warp's
  // first lane issues the MMAs of two rows (four issuers share the tensor core)
  auto issue = [&](int r0, int r1, uint64_t *bar) {
    const uint32_t lbo = C == 16 ? (uint32_t)TC_PLANE : 16u;
    for (int r = r0; r < r1; r++) {
      for (int j = 0; j < NM; j++) {
        const int ky = C == 16 ? j / 5 : j / 3;
        const int kx = C == 16 ? j % 5 : 2 * (j % 3);
        const uint64_t ad = tc_desc(pbase + (uint32_t)(((r + ky) * TC_COLS + kx) * 16), lbo, 128);
        const uint64_t bd = tc_desc(wbase + (uint32_t)(j * BB), BB / 2, 128);
        const uint32_t acc = j > 0 ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.u32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem + (uint32_t)(r * N)),
            "l"(ad), "l"(bd), "r"(tc_idesc<N>()), "r"(acc));
      }
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
  };
  static_assert(TC_ROWS == 8, "two rows per warp, two warps per stage");
  if (lane == 0 && loaded) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    issue(2 * warp, 2 * warp + 2, mbar + (warp >> 1));
  }

  auto wait_bar = [&](uint64_t *bar) -> uint32_t {
    const uint32_t ok = loaded ? mbar_wait(smem_addr(bar), 0) : 0u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok && tid == 0 && err) atomicOr(err, ERR_SPIN_TIMEOUT);
    return ok;
  };
  const int gx = x0 + 32 * warp + lane;
  const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
  // read back and store output rows [r0, r1) once their MMAs are done
  auto epilogue = [&](int r0, int r1, uint32_t done) {
    if constexpr (MODE == CONV_RELU_BF16) {
      float b[16];
#pragma unroll
      for (int c = 0; c < 16; c++) b[c] = __bfloat162float(bias[c]);
#pragma unroll 1
      for (int r = r0; r < r1; r++) {
        uint32_t v[16];
        if (done) {
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
              : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
              : "r"(trow + (uint32_t)(r * N)));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        } else {
#pragma unroll
          for (int c = 0; c < 16; c++) v[c] = 0x7FC00000u;  // NaN: the accumulators were not read
        }
        const int gy = y0 + r;
        if (gx < W && gy < H) {
          uint4 o[2];
          __nv_bfloat16 *ob = reinterpret_cast<__nv_bfloat16 *>(o);
#pragma unroll
          for (int c = 0; c < 16; c++) ob[c] = __float2bfloat16_rn(fmaxf(__uint_as_float(v[c]) + b[c], 0.0f));
          uint4 *dst = reinterpret_cast<uint4 *>(reinterpret_cast<__nv_bfloat16 *>(out) +
                                                 (img_base + (size_t)gy * W + gx) * 16);
          dst[0] = o[0];
          dst[1] = o[1];
        }
      }
    } else {
      const float b0 = __bfloat162float(bias[0]);
      constexpr int HALF = TC_ROWS / 2;
      uint32_t v[HALF];
      if (done) {
        // column 0 (output channel 0) of each row's accumulator
#pragma unroll
        for (int k = 0; k < HALF; k++)
          asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];"
                       : "=r"(v[k])
                       : "r"(trow + (uint32_t)((r0 + k) * N)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      } else {
#pragma unroll
        for (int k = 0; k < HALF; k++) v[k] = 0x7FC00000u;
      }
#pragma unroll
      for (int k = 0; k < HALF; k++) {
        const int gy = y0 + r0 + k;
        if (gx >= W || gy >= H) continue;
        const float a = __uint_as_float(v[k]) + b0;
        float o = a;
        if (MODE == CONV_CONF) {
          const float c = fmaxf(1.0f - fmaxf(a, 0.0f) * inv_tau, 0.0f);
          o = c * c;
        }
        reinterpret_cast<float *>(out)[img_base + (size_t)gy * W + gx] = o;
      }
    }
  };
  const uint32_t done0 = wait_bar(mbar);
  epilogue(0, TC_ROWS / 2, done0);
  const uint32_t done1 = wait_bar(mbar + 1);
  epilogue(TC_ROWS / 2, TC_ROWS, done1);
  // A wait that gave up may leave the tile copies or the MMAs in flight,
  // writing this block's shared and tensor memory: wait for them once more
  // (bounded again) before both are given back.  If that wait gives up too,
  // the frame is already reported failed and its confidence map is not used.
  if (!loaded) {
    mbar_wait(ld_bar, 0);
  } else {
    if (!done0) mbar_wait(smem_addr(mbar), 0);
    if (!done1) mbar_wait(smem_addr(mbar + 1), 0);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

template <int CIN, int COUT>
constexpr size_t wgrad_smem_bytes() {
  return sizeof(float) * ((size_t)CIN * PLANE + (size_t)COUT * GPLANE);
}

// Weight and bias gradients of a layer (CIN in, COUT out): dW[co][ci][tap] =
// sum over pixels of x[p + tap] * dy[p][co], db[co] = sum of dy[co].  Each
// thread owns one (co, ci) pair and a share of the tile's pixels, blocks
// stride over the tiles of all images and add their sums once at the end.
template <int CIN, int COUT, int CSTR>
__global__ void __launch_bounds__(256) k_conv_wgrad(const __nv_bfloat16 *__restrict__ x,
                                                    const float *__restrict__ dy, int W, int H, int n_img,
                                                    float *__restrict__ dw, float *__restrict__ db) {
  extern __shared__ __align__(16) float smem[];
  float *s_x = smem;
  float *s_g = smem + CIN * PLANE;
  constexpr int P = CIN * COUT;
  static_assert(P <= 256, "one pair per thread");
  constexpr int G = 256 / P;
  const int pair = threadIdx.x % P, grp = threadIdx.x / P;
  const bool active = grp < G;
  const int co = pair / CIN, ci = pair % CIN;
  float acc[TAPS];
#pragma unroll
  for (int k = 0; k < TAPS; k++) acc[k] = 0.0f;
  float accb = 0.0f;
  const int tiles_x = (W + TX - 1) / TX, tiles_y = (H + TY - 1) / TY;
  const int total = tiles_x * tiles_y * n_img;
  for (int tile = blockIdx.x; tile < total; tile += gridDim.x) {
    const int img = tile / (tiles_x * tiles_y), rest = tile % (tiles_x * tiles_y);
    const int x0 = (rest % tiles_x) * TX, y0 = (rest / tiles_x) * TY;
    __syncthreads();
    load_tile<CIN, CSTR>(x, img, W, H, x0, y0, s_x);
    for (int i = threadIdx.x; i < TX * TY; i += blockDim.x) {
      const int gx = x0 + i % TX, gy = y0 + i / TX;
      float v[COUT];
      if (gx < W && gy < H) {
        load_px<COUT, COUT>(dy + (((size_t)img * H + gy) * W + gx) * COUT, v);
      } else {
#pragma unroll
        for (int c = 0; c < COUT; c++) v[c] = 0.0f;
      }
#pragma unroll
      for (int c = 0; c < COUT; c++) s_g[c * GPLANE + i] = v[c];
    }
    __syncthreads();
    if (active) {
      const float *pg = s_g + co * GPLANE;
      const float *px = s_x + ci * PLANE;
      for (int p = grp; p < TX * TY; p += G) {
        const float g = pg[p];
        const float *q = px + (p / TX) * SX + (p % TX);
#pragma unroll
        for (int ky = 0; ky < 5; ky++)
#pragma unroll
          for (int kx = 0; kx < 5; kx++) acc[ky * 5 + kx] = fmaf(q[ky * SX + kx], g, acc[ky * 5 + kx]);
        accb += g;
      }
    }
  }
  if (active) {
#pragma unroll
    for (int k = 0; k < TAPS; k++) atomicAdd(dw + (co * CIN + ci) * TAPS + k, acc[k]);
    if (ci == 0) atomicAdd(db + co, accb);
  }
}

// Network input per pixel: depth z (m), the unit normal from central
// differences of the back-projected neighbours (zero unless all four are
// valid), and the validity flag.
__global__ void k_cnn_features(const uint16_t *__restrict__ depth, int W, int H, float scaling, float fx, float fy,
                               float cx, float cy, __nv_bfloat16 *__restrict__ feat) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, img = blockIdx.z;
  if (x >= W) return;
  const uint16_t *d = depth + (size_t)img * W * H;
  auto zat = [&](int xx, int yy) -> float {
    return (xx < 0 || yy < 0 || xx >= W || yy >= H) ? 0.0f : scaling * (float)__ldg(d + (size_t)yy * W + xx);
  };
  const float z = zat(x, y);
  const float zl = zat(x - 1, y), zr = zat(x + 1, y), zu = zat(x, y - 1), zd = zat(x, y + 1);
  float nx = 0.0f, ny = 0.0f, nz = 0.0f;
  if (z > 0.0f && zl > 0.0f && zr > 0.0f && zu > 0.0f && zd > 0.0f) {
    // a = P(x+1) - P(x-1), b = P(y+1) - P(y-1); n = b x a faces the camera
    const float ax = ((float)(x + 1) - cx) * zr / fx - ((float)(x - 1) - cx) * zl / fx;
    const float ay = ((float)y - cy) * (zr - zl) / fy;
    const float az = zr - zl;
    const float bx = ((float)x - cx) * (zd - zu) / fx;
    const float by = ((float)(y + 1) - cy) * zd / fy - ((float)(y - 1) - cy) * zu / fy;
    const float bz = zd - zu;
    nx = by * az - bz * ay;
    ny = bz * ax - bx * az;
    nz = bx * ay - by * ax;
    const float len = sqrtf(nx * nx + ny * ny + nz * nz);
    if (len > 0.0f) {
      nx /= len;
      ny /= len;
      nz /= len;
    } else {
      nx = ny = nz = 0.0f;
    }
  }
  uint4 u;
  __nv_bfloat16 *b = reinterpret_cast<__nv_bfloat16 *>(&u);
  b[0] = __float2bfloat16_rn(z);
  b[1] = __float2bfloat16_rn(nx);
  b[2] = __float2bfloat16_rn(ny);
  b[3] = __float2bfloat16_rn(nz);
  b[4] = __float2bfloat16_rn(z > 0.0f ? 1.0f : 0.0f);
  b[5] = b[6] = b[7] = __float2bfloat16_rn(0.0f);
  reinterpret_cast<uint4 *>(feat)[((size_t)img * H + y) * W + x] = u;
}

// Mean squared error over labelled pixels (target >= 0; negative = no
// label): dpred = 2 (pred - target) * inv_count, loss += sum * inv_count.
__global__ void k_cnn_mse(const float *__restrict__ pred, const float *__restrict__ target, int64_t n,
                          float inv_count, float *__restrict__ dpred, double *__restrict__ loss) {
  double local = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float y = target[i];
    float g = 0.0f;
    if (y >= 0.0f) {
      const float e = pred[i] - y;
      g = 2.0f * e * inv_count;
      local += (double)e * (double)e;
    }
    dpred[i] = g;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && local != 0.0) atomicAdd(loss, local * (double)inv_count);
}

// Adam on the FP32 master weights; the BF16 copy the kernels use is written
// from the updated master, and the gradient is cleared for the next step.
__global__ void k_cnn_adam(float *__restrict__ master, __nv_bfloat16 *__restrict__ params, float *__restrict__ grad,
                           float *__restrict__ m, float *__restrict__ v, int n, float lr, float b1, float b2,
                           float eps, float bc1, float bc2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = grad[i];
  const float mi = b1 * m[i] + (1.0f - b1) * g;
  const float vi = b2 * v[i] + (1.0f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float w = master[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  master[i] = w;
  params[i] = __float2bfloat16_rn(w);
  grad[i] = 0.0f;
}

// ------------------------------------------------------------------ raycast

constexpr int RAYCAST_MAX_STEPS = 4096;

// The finest leaf holding voxel (x, y, z), or UINT32_MAX.
__device__ __forceinline__ uint32_t finest_leaf(const uint32_t *__restrict__ tree, uint32_t n, uint32_t leaves_max,
                                                uint32_t x, uint32_t y, uint32_t z) {
  uint32_t ox = 0, oy = 0, oz = 0, half = n >> 1, branch = 0, best = UINT32_MAX;
  for (int level = 0; level < 16 && half >= (uint32_t)BL; level++) {
    const uint32_t co = (x >= ox + half) * 1u + (y >= oy + half) * 2u + (z >= oz + half) * 4u;
    const uint32_t leaf = __ldg(tree + branch + co);
    if (leaf < leaves_max) best = leaf;
    const uint32_t child = __ldg(tree + branch + co + 8);
    if (child >= PENDING) break;  // BRANCHINIT (no child)
    ox += half * ((co & 1) != 0);
    oy += half * ((co & 2) != 0);
    oz += half * ((co & 4) != 0);
    branch = child;
    half >>= 1;
  }
  return best;
}

// Depth (m) of the first surface crossing of pixel (x, y)'s ray within
// +-window of its measured depth: the fused SDF of the finest brick
// (trilinear where the 8 surrounding voxels lie in the brick and are
// weighted, else the nearest voxel) sampled every `step` metres of depth,
// a change from negative (in front of the surface) to non-negative, both
// samples weighted, linearly interpolated -- or, entering a weighted band
// from unallocated space with 0 <= s < the truncation distance, t - s.
// 0 where the pixel has no depth, -1 where no surface lies in the window.
__global__ void k_raycast(RaycastMap m, CamF p, int W, int H, const uint16_t *__restrict__ depth, float scaling,
                          float window, float step, float *__restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const float d0 = scaling * (float)__ldg(depth + (size_t)y * W + x);
  float res = 0.0f;
  if (d0 > 0.0f) {
    res = -1.0f;
    const float rx = ((float)x - p.cx) / p.fx, ry = ((float)y - p.cy) / p.fy;
    const float t0 = fmaxf(d0 - window, 0.05f), t1 = d0 + window;
    bool prev_ok = false;
    float prev_s = 0.0f, prev_t = 0.0f, band = 0.0f;
    const int nsteps = min((int)((t1 - t0) / step) + 1, RAYCAST_MAX_STEPS);
    for (int k = 0; k < nsteps; k++) {
      const float t = t0 + (float)k * step;
      const float cxm = rx * t, cym = ry * t;
      const float gx = p.r[0] * cxm + p.r[1] * cym + p.r[2] * t + p.t[0];
      const float gy = p.r[3] * cxm + p.r[4] * cym + p.r[5] * t + p.t[1];
      const float gz = p.r[6] * cxm + p.r[7] * cym + p.r[8] * t + p.t[2];
      bool ok = false;
      float s = 0.0f;
      const int ix = __float2int_rn(gx), iy = __float2int_rn(gy), iz = __float2int_rn(gz);
      if (ix >= 0 && iy >= 0 && iz >= 0 && ix < (int)m.n && iy < (int)m.n && iz < (int)m.n) {
        const uint32_t leaf = finest_leaf(m.tree, m.n, m.leaves_max, ix, iy, iz);
        if (leaf != UINT32_MAX) {
          const ushort4 o = __ldg(m.leaf + leaf);
          const float ls = (float)o.w;
          band = 0.99f * m.thr * ls;
          const float ux = (gx - (float)o.x) / ls, uy = (gy - (float)o.y) / ls, uz = (gz - (float)o.z) / ls;
          const int fx0 = (int)floorf(ux), fy0 = (int)floorf(uy), fz0 = (int)floorf(uz);
          const size_t base = (size_t)leaf * 512;
          if (fx0 >= 0 && fy0 >= 0 && fz0 >= 0 && fx0 < 7 && fy0 < 7 && fz0 < 7) {
            // trilinear inside the brick when its 8 voxels are all weighted
            const float ax = ux - (float)fx0, ay = uy - (float)fy0, az = uz - (float)fz0;
            float acc = 0.0f;
            bool all = true;
#pragma unroll
            for (int c = 0; c < 8; c++) {
              const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
              const size_t vi = base + ((fz0 + dz) * 8 + fy0 + dy) * 8 + fx0 + dx;
              const float w = m.fp16 ? __half2float(m.wgt16[vi]) : m.wgt[vi];
              const float v = m.fp16 ? __half2float(m.sdf16[vi]) : m.sdf[vi];
              all = all && w > 0.0f;
              acc += (dx ? ax : 1.0f - ax) * (dy ? ay : 1.0f - ay) * (dz ? az : 1.0f - az) * v;
            }
            if (all) {
              s = acc;
              ok = true;
            }
          }
          if (!ok) {  // nearest voxel
            const int lx = min(max(__float2int_rn(ux), 0), 7);
            const int ly = min(max(__float2int_rn(uy), 0), 7);
            const int lz = min(max(__float2int_rn(uz), 0), 7);
            const size_t vi = base + (lz * 8 + ly) * 8 + lx;
            const float w = m.fp16 ? __half2float(m.wgt16[vi]) : m.wgt[vi];
            if (w > 0.0f) {
              s = m.fp16 ? __half2float(m.sdf16[vi]) : m.sdf[vi];
              ok = true;
            }
          }
        }
      }
      if (ok && prev_ok && prev_s < 0.0f && s >= 0.0f) {
        res = prev_t + step * (-prev_s) / (s - prev_s);
        break;
      }
      // entering the band of a surface from unallocated space (its front
      // side lies in a brick no sample allocated): the along-ray SDF places
      // the surface at t - s
      if (ok && !prev_ok && k > 0 && s >= 0.0f && s < band) {
        res = t - s;
        break;
      }
      prev_ok = ok;
      prev_s = s;
      prev_t = t;
    }
  }
  out[(size_t)y * W + x] = res;
}

// ---------------------------------------------------------------- launchers

namespace {
std::mutex g_attr_mu;
unsigned long long g_attr_done = 0;  // devices whose kernels have their shared-memory limits set

template <int KIN, int KOUT, int CSTR, typename TIN, bool TRANS, int MODE>
cudaError_t set_conv_attr() {
  return cudaFuncSetAttribute(k_conv<KIN, KOUT, CSTR, TIN, TRANS, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)conv_smem_bytes<KIN, KOUT>());
}
template <int C, int N, int MODE>
cudaError_t set_tc_attr() {
  return cudaFuncSetAttribute(k_conv_tc<C, N, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)tc_smem_bytes<C, N>());
}
template <int CIN, int COUT, int CSTR>
cudaError_t set_wgrad_attr() {
  return cudaFuncSetAttribute(k_conv_wgrad<CIN, COUT, CSTR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)wgrad_smem_bytes<CIN, COUT>());
}

cudaError_t ensure_attrs() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_attr_mu);
  const unsigned long long bit = 1ull << (dev & 63);
  if (g_attr_done & bit) return cudaSuccess;
  cudaError_t r[] = {
      set_tc_attr<CNN_IN_STRIDE, 16, CONV_RELU_BF16>(),
      set_tc_attr<CNN_HID, 16, CONV_RELU_BF16>(),
      set_tc_attr<CNN_HID, 16, CONV_F32>(),
      set_tc_attr<CNN_HID, 16, CONV_CONF>(),
      set_conv_attr<1, CNN_HID, 1, float, true, CONV_MASK_F32>(),
      set_conv_attr<CNN_HID, CNN_HID, CNN_HID, float, true, CONV_MASK_F32>(),
      set_wgrad_attr<CNN_HID, 1, CNN_HID>(),
      set_wgrad_attr<CNN_HID, CNN_HID, CNN_HID>(),
      set_wgrad_attr<CNN_IN, CNN_HID, CNN_IN_STRIDE>(),
  };
  for (cudaError_t x : r)
    if (x != cudaSuccess) return x;
  g_attr_done |= bit;
  return cudaSuccess;
}

// Tensor-map encoder of the driver, looked up once (the library does not
// link the driver library itself).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// The tile of a k_conv_tc block over n images of W x H pixels, C = 8 or 16
// BF16 channels per pixel: a (TC_ROWS + 4) x TC_COLS box of one 8-channel
// plane, zero outside the image (dimensions: 8 channels, [plane], x, y, image).
cudaError_t tile_map(CUtensorMap *m, const void *base, int C, int W, int H, int n) {
  const EncodeTiledFn f = encode_tiled();
  if (!f) return cudaErrorNotSupported;
  cuuint64_t dims[5], strides[4];
  cuuint32_t box[5], es[5] = {1, 1, 1, 1, 1};
  cuuint32_t rank;
  if (C == 16) {
    rank = 5;
    const cuuint64_t d[5] = {8, 2, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)n};
    const cuuint64_t st[4] = {16, 32, (cuuint64_t)W * 32, (cuuint64_t)W * H * 32};
    const cuuint32_t b[5] = {8, 1, TC_COLS, TC_TILE_ROWS, 1};
    for (int i = 0; i < 5; i++) dims[i] = d[i], box[i] = b[i];
    for (int i = 0; i < 4; i++) strides[i] = st[i];
  } else {
    rank = 4;
    const cuuint64_t d[4] = {8, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)n};
    const cuuint64_t st[3] = {16, (cuuint64_t)W * 16, (cuuint64_t)W * H * 16};
    const cuuint32_t b[4] = {8, TC_COLS, TC_TILE_ROWS, 1};
    for (int i = 0; i < 4; i++) dims[i] = d[i], box[i] = b[i];
    for (int i = 0; i < 3; i++) strides[i] = st[i];
  }
  const CUresult r = f(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, rank, const_cast<void *>(base), dims, strides, box, es,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

dim3 conv_grid(int W, int H, int n) {
  return dim3((W + TX - 1) / TX, (H + conv_ty(CONV_RPT) - 1) / conv_ty(CONV_RPT), n);
}

template <int KIN, int KOUT, int CSTR, typename TIN, bool TRANS, int MODE>
void conv(const TIN *in, int n, int W, int H, const __nv_bfloat16 *w, const __nv_bfloat16 *b, void *out,
          const __nv_bfloat16 *act, float inv_tau, cudaStream_t s) {
  note_launch();
  k_conv<KIN, KOUT, CSTR, TIN, TRANS, MODE>
      <<<conv_grid(W, H, n), 256, conv_smem_bytes<KIN, KOUT>(), s>>>(in, W, H, w, b, out, act, inv_tau);
}

template <int CIN, int COUT, int CSTR>
void wgrad(const __nv_bfloat16 *x, const float *dy, int n, int W, int H, float *dw, float *db, cudaStream_t s) {
  const int tiles = ((W + TX - 1) / TX) * ((H + TY - 1) / TY) * n;
  note_launch();
  k_conv_wgrad<CIN, COUT, CSTR>
      <<<std::min(tiles, 148 * 2), 256, wgrad_smem_bytes<CIN, COUT>(), s>>>(x, dy, W, H, n, dw, db);
}
}  // namespace

cudaError_t cnn_features(const uint16_t *depth, int n, int W, int H, float scaling, const float K[4],
                         __nv_bfloat16 *feat, cudaStream_t s) {
  note_launch();
  k_cnn_features<<<dim3((W + 127) / 128, H, n), 128, 0, s>>>(depth, W, H, scaling, K[0], K[1], K[2], K[3], feat);
  return cudaGetLastError();
}

cudaError_t cnn_forward(const __nv_bfloat16 *params, uint8_t *packed, bool packed_ready, const __nv_bfloat16 *feat,
                        int n, int W, int H, __nv_bfloat16 *a1, __nv_bfloat16 *a2, float *out, float tau_cm,
                        uint32_t *err, cudaStream_t s) {
  cudaError_t e = ensure_attrs();
  if (e != cudaSuccess) return e;
  if (!packed_ready) {
    note_launch();
    k_pack_tc<<<(TC_PACK_BYTES / 2 + 255) / 256, 256, 0, s>>>(params, reinterpret_cast<__nv_bfloat16 *>(packed));
  }
  CUtensorMap m_feat, m_a1, m_a2;
  if ((e = tile_map(&m_feat, feat, CNN_IN_STRIDE, W, H, n)) != cudaSuccess ||
      (e = tile_map(&m_a1, a1, CNN_HID, W, H, n)) != cudaSuccess ||
      (e = tile_map(&m_a2, a2, CNN_HID, W, H, n)) != cudaSuccess)
    return e;
  const dim3 tg((W + 127) / 128, (H + TC_ROWS - 1) / TC_ROWS, n);
  note_launch(3);
  k_conv_tc<CNN_IN_STRIDE, 16, CONV_RELU_BF16><<<tg, 128, tc_smem_bytes<CNN_IN_STRIDE, 16>(), s>>>(
      m_feat, W, H, packed + TC_PACK_L1, params + P_B1, a1, 0.0f, err);
  k_conv_tc<CNN_HID, 16, CONV_RELU_BF16><<<tg, 128, tc_smem_bytes<CNN_HID, 16>(), s>>>(
      m_a1, W, H, packed + TC_PACK_L2, params + P_B2, a2, 0.0f, err);
  if (tau_cm > 0.0f)
    k_conv_tc<CNN_HID, 16, CONV_CONF><<<tg, 128, tc_smem_bytes<CNN_HID, 16>(), s>>>(
        m_a2, W, H, packed + TC_PACK_L3, params + P_B3, out, 1.0f / tau_cm, err);
  else
    k_conv_tc<CNN_HID, 16, CONV_F32><<<tg, 128, tc_smem_bytes<CNN_HID, 16>(), s>>>(
        m_a2, W, H, packed + TC_PACK_L3, params + P_B3, out, 0.0f, err);
  return cudaGetLastError();
}

cudaError_t cnn_backward(const __nv_bfloat16 *params, const __nv_bfloat16 *feat, const __nv_bfloat16 *a1,
                         const __nv_bfloat16 *a2, const float *dpred, int n, int W, int H, float *g1, float *g2,
                         float *grads, cudaStream_t s) {
  cudaError_t e = ensure_attrs();
  if (e != cudaSuccess) return e;
  // layer 3
  wgrad<CNN_HID, 1, CNN_HID>(a2, dpred, n, W, H, grads + P_W3, grads + P_B3, s);
  conv<1, CNN_HID, 1, float, true, CONV_MASK_F32>(dpred, n, W, H, params + P_W3, nullptr, g2, a2, 0.0f, s);
  // layer 2
  wgrad<CNN_HID, CNN_HID, CNN_HID>(a1, g2, n, W, H, grads + P_W2, grads + P_B2, s);
  conv<CNN_HID, CNN_HID, CNN_HID, float, true, CONV_MASK_F32>(g2, n, W, H, params + P_W2, nullptr, g1, a1, 0.0f, s);
  // layer 1 (no gradient of the input)
  wgrad<CNN_IN, CNN_HID, CNN_IN_STRIDE>(feat, g1, n, W, H, grads + P_W1, grads + P_B1, s);
  return cudaGetLastError();
}

cudaError_t cnn_mse(const float *pred, const float *target, int64_t count, float inv_count, float *dpred,
                    double *loss, cudaStream_t s) {
  const int blocks = (int)std::min<int64_t>((count + 255) / 256, 148 * 8);
  note_launch();
  k_cnn_mse<<<std::max(blocks, 1), 256, 0, s>>>(pred, target, count, inv_count, dpred, loss);
  return cudaGetLastError();
}

cudaError_t cnn_adam(float *master, __nv_bfloat16 *params, float *grads, float *m, float *v, int n, float lr,
                     float b1, float b2, float eps, int step, cudaStream_t s) {
  const float bc1 = 1.0f - powf(b1, (float)step), bc2 = 1.0f - powf(b2, (float)step);
  note_launch();
  k_cnn_adam<<<(n + 255) / 256, 256, 0, s>>>(master, params, grads, m, v, n, lr, b1, b2, eps, bc1, bc2);
  return cudaGetLastError();
}

cudaError_t launch_raycast(const RaycastMap &m, const CamF &p, int W, int H, const uint16_t *depth, float scaling,
                           float window, float step, float *out, cudaStream_t s) {
  note_launch();
  k_raycast<<<dim3((W + 127) / 128, H), 128, 0, s>>>(m, p, W, H, depth, scaling, window, step, out);
  return cudaGetLastError();
}

}  // namespace ffb
