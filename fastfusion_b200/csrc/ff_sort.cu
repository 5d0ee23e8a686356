// Sorting of 64-bit keys with their original positions (an argsort), for the
// mesh-cell list (keys of type, size and origin) and the order of a frame's
// new leaves (first pixel).  Ascending; equal keys keep their input order.
//
//  * up to SORT_SMALL keys whose bits and position fit one 64-bit word: one
//    block sorts the packed words (key << 14 | position) in shared memory by
//    a bitonic network (one launch);
//  * otherwise a least-significant-digit radix sort, 8 bits per pass: per
//    tile of 2048 keys a digit histogram, an exclusive scan of the histograms
//    in digit-major order (the output base of every (digit, tile)), and a
//    stable scatter that ranks each tile's keys digit by digit in input order
//    (warp match + per-warp counters in shared memory).
#include <algorithm>
#include <cstdint>

#include "ff_common.cuh"
#include "ff_sort.h"

namespace ffb {

constexpr int SORT_SMALL_THREADS = 1024;
constexpr int SORT_SMALL_POS_BITS = 14;  // positions < SORT_SMALL = 2^14
constexpr int RS_THREADS = 256, RS_ITEMS = 8, RS_TILE = RS_THREADS * RS_ITEMS, RS_BINS = 256;
constexpr int SCAN_BLOCK = 1024;

static_assert(SORT_SMALL == (1u << SORT_SMALL_POS_BITS), "positions of the small sort fill its position bits");
static_assert(RS_BINS == RS_THREADS, "one digit per thread in the scatter's digit loops");

// ----------------------------------------------------------- small sort ----

__global__ void __launch_bounds__(SORT_SMALL_THREADS) k_sort_small(const uint64_t *__restrict__ keys, uint32_t n,
                                                                  uint32_t p2, uint64_t *keys_out,
                                                                  uint32_t *pos_out) {
  extern __shared__ uint64_t w[];
  for (uint32_t i = threadIdx.x; i < p2; i += SORT_SMALL_THREADS)
    w[i] = i < n ? (keys[i] << SORT_SMALL_POS_BITS) | i : ~0ull;
  __syncthreads();
  for (uint32_t k = 2; k <= p2; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < p2; i += SORT_SMALL_THREADS) {
        const uint32_t m = i ^ j;
        if (m > i) {
          const uint64_t a = w[i], b = w[m];
          const bool up = (i & k) == 0;
          if ((a > b) == up) {
            w[i] = b;
            w[m] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  for (uint32_t i = threadIdx.x; i < n; i += SORT_SMALL_THREADS) {
    const uint64_t v = w[i];
    keys_out[i] = v >> SORT_SMALL_POS_BITS;
    pos_out[i] = (uint32_t)(v & (SORT_SMALL - 1u));
  }
}

// The same network with E packed words per thread in registers, thread t
// holding words [E t, E t + E) of P = 1024 E: compare-exchanges of words
// less than E apart are within a thread, less than 32 E apart between the
// lanes of a warp (shuffles), the rest through shared memory -- 15 block
// barriers for P = 16384 instead of 105.
__device__ __forceinline__ void cx(uint64_t &lo, uint64_t &hi, bool up) {
  const uint64_t a = lo, b = hi;
  const bool sw = (a > b) == up;
  lo = sw ? b : a;
  hi = sw ? a : b;
}

// compare-exchanges J apart within a thread's E words (J < E)
template <int E, int J>
__device__ __forceinline__ void stage_in(uint64_t (&v)[E], uint32_t base, uint32_t k) {
#pragma unroll
  for (int e = 0; e < E; e++)
    if ((e ^ J) > e) cx(v[e], v[e ^ J], ((base + (uint32_t)e) & k) == 0);
}

template <int E>
__global__ void __launch_bounds__(SORT_SMALL_THREADS) k_sort_small_reg(const uint64_t *__restrict__ keys, uint32_t n,
                                                                      uint64_t *keys_out, uint32_t *pos_out) {
  pdl_enter();
  extern __shared__ uint64_t w[];
  constexpr uint32_t P = SORT_SMALL_THREADS * E;
  const uint32_t t = threadIdx.x, base = t * E;
  uint64_t v[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const uint32_t i = base + e;
    v[e] = i < n ? (keys[i] << SORT_SMALL_POS_BITS) | i : ~0ull;
  }
  for (uint32_t k = 2; k <= P; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      if (j < (uint32_t)E) {
        // within the thread
        if (j == 1) stage_in<E, (E > 1 ? 1 : 0)>(v, base, k);
        if constexpr (E > 2) {
          if (j == 2) stage_in<E, 2>(v, base, k);
        }
        if constexpr (E > 4) {
          if (j == 4) stage_in<E, 4>(v, base, k);
        }
        if constexpr (E > 8) {
          if (j == 8) stage_in<E, 8>(v, base, k);
        }
      } else {
        // the partner word is word e of thread t ^ (j / E); this thread keeps
        // the smaller of the two where its index is the lower one of an
        // ascending pair (or the upper one of a descending pair)
        const uint32_t tj = j / E;
        const bool up = (base & k) == 0;  // (k > j >= E: the same for all E words)
        const bool lower = (t & tj) == 0;
        const bool keep_min = lower == up;
        if (tj < 32) {
#pragma unroll
          for (int e = 0; e < E; e++) {
            const uint64_t o = __shfl_xor_sync(0xffffffffu, v[e], (int)tj);
            v[e] = keep_min ? (o < v[e] ? o : v[e]) : (o > v[e] ? o : v[e]);
          }
        } else {
          __syncthreads();  // (the previous exchange's reads are done)
#pragma unroll
          for (int e = 0; e < E; e++) w[base + e] = v[e];
          __syncthreads();
          const uint32_t ob = (t ^ tj) * E;
#pragma unroll
          for (int e = 0; e < E; e++) {
            const uint64_t o = w[ob + e];
            v[e] = keep_min ? (o < v[e] ? o : v[e]) : (o > v[e] ? o : v[e]);
          }
        }
      }
    }
  }
#pragma unroll
  for (int e = 0; e < E; e++) {
    const uint32_t i = base + e;
    if (i < n) {
      keys_out[i] = v[e] >> SORT_SMALL_POS_BITS;
      pos_out[i] = (uint32_t)(v[e] & (SORT_SMALL - 1u));
    }
  }
}

// ----------------------------------------------------------- radix sort ----

// digit histogram of each tile, digit-major: hist[d * ntiles + tile]
__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const uint64_t *__restrict__ keys, uint32_t n, int shift,
                                                        uint32_t *hist, uint32_t ntiles) {
  __shared__ uint32_t h[RS_BINS];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t base = blockIdx.x * RS_TILE;
#pragma unroll
  for (int r = 0; r < RS_ITEMS; r++) {
    const uint32_t i = base + r * RS_THREADS + threadIdx.x;
    if (i < n) atomicAdd(&h[(uint32_t)(keys[i] >> shift) & (RS_BINS - 1)], 1u);
  }
  __syncthreads();
  hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// exclusive prefix over a SCAN_BLOCK-thread block of one value per thread;
// the block's total in *total
__device__ __forceinline__ uint32_t block_scan_1024(uint32_t v, uint32_t *total) {
  __shared__ uint32_t ws[SCAN_BLOCK / 32];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t u = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += u;
  }
  if (lane == 31) ws[wi] = x;
  __syncthreads();
  if (wi == 0) {
    uint32_t y = ws[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, y, o);
      if (lane >= o) y += u;
    }
    ws[lane] = y;  // inclusive over warps
  }
  __syncthreads();
  const uint32_t r = (wi ? ws[wi - 1] : 0u) + x - v;
  *total = ws[SCAN_BLOCK / 32 - 1];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_sums(const uint32_t *__restrict__ v, uint32_t n, uint32_t *sums) {
  const uint32_t i = blockIdx.x * SCAN_BLOCK + threadIdx.x;
  uint32_t total;
  (void)block_scan_1024(i < n ? v[i] : 0u, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// exclusive scan of the block sums in one block, in chunks of SCAN_BLOCK
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_top(uint32_t *sums, uint32_t nsums) {
  uint32_t carry = 0;
  for (uint32_t base = 0; base < nsums; base += SCAN_BLOCK) {
    const uint32_t i = base + threadIdx.x;
    uint32_t total;
    const uint32_t ex = block_scan_1024(i < nsums ? sums[i] : 0u, &total);
    if (i < nsums) sums[i] = carry + ex;
    carry += total;
  }
}

__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_apply(uint32_t *v, uint32_t n, const uint32_t *__restrict__ sums) {
  const uint32_t i = blockIdx.x * SCAN_BLOCK + threadIdx.x;
  uint32_t total;
  const uint32_t ex = block_scan_1024(i < n ? v[i] : 0u, &total);
  if (i < n) v[i] = ex + sums[blockIdx.x];
}

// Stable scatter of one tile by the digit at `shift`: the tile's keys are
// taken RS_THREADS at a time in input order; within such a round a key's
// rank among equal digits is its lane rank in its warp plus the counts of
// the warps before it, after the counts of the earlier rounds.  vals null:
// the values are the input positions.
__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const uint64_t *__restrict__ keys,
                                                           const uint32_t *__restrict__ vals, uint32_t n, int shift,
                                                           const uint32_t *__restrict__ offs, uint32_t ntiles,
                                                           uint64_t *keys_out, uint32_t *vals_out) {
  __shared__ uint32_t run[RS_BINS];
  __shared__ uint32_t wc[RS_THREADS / 32][RS_BINS];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  run[threadIdx.x] = offs[(size_t)threadIdx.x * ntiles + blockIdx.x];
  const uint32_t base = blockIdx.x * RS_TILE;
  for (int r = 0; r < RS_ITEMS; r++) {
#pragma unroll
    for (int k = 0; k < RS_THREADS / 32; k++) wc[k][threadIdx.x] = 0;
    __syncthreads();
    const uint32_t i = base + r * RS_THREADS + threadIdx.x;
    const bool ok = i < n;
    const uint64_t key = ok ? keys[i] : 0ull;
    const uint32_t val = ok ? (vals ? vals[i] : i) : 0u;
    const uint32_t dig = ok ? ((uint32_t)(key >> shift) & (RS_BINS - 1)) : (uint32_t)RS_BINS;
    const unsigned peers = __match_any_sync(0xffffffffu, dig);
    const uint32_t rank = (uint32_t)__popc(peers & ((1u << lane) - 1u));
    if (ok && lane == __ffs(peers) - 1) wc[wi][dig] = (uint32_t)__popc(peers);
    __syncthreads();
    {
      uint32_t acc = run[threadIdx.x];
#pragma unroll
      for (int k = 0; k < RS_THREADS / 32; k++) {
        const uint32_t c = wc[k][threadIdx.x];
        wc[k][threadIdx.x] = acc;
        acc += c;
      }
      run[threadIdx.x] = acc;
    }
    __syncthreads();
    if (ok) {
      const uint32_t pos = wc[wi][dig] + rank;
      keys_out[pos] = key;
      vals_out[pos] = val;
    }
    __syncthreads();
  }
}

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

static uint32_t tiles_of(uint32_t n) { return (n + RS_TILE - 1) / RS_TILE; }

// packed words below the all-ones padding: end_bit + 14 < 64
static bool small_path(uint32_t n, int end_bit) { return n <= SORT_SMALL && end_bit + SORT_SMALL_POS_BITS < 64; }

size_t argsort_temp_bytes(uint32_t n) {
  const size_t ntiles = tiles_of(n), nh = ntiles * RS_BINS, nsums = (nh + SCAN_BLOCK - 1) / SCAN_BLOCK;
  return align256((size_t)n * 8) + align256((size_t)n * 4) + align256(nh * 4) + align256(std::max<size_t>(nsums, 1) * 4);
}

cudaError_t argsort_u64(const uint64_t *keys, uint32_t n, int end_bit, uint64_t *keys_out, uint32_t *pos_out,
                        void *tmp, size_t tmp_bytes, cudaStream_t s, unsigned *launches, bool pdl) {
  if (!n) return cudaSuccess;
  if (end_bit < 1 || end_bit > 64) return cudaErrorInvalidValue;
  if (small_path(n, end_bit)) {
    static bool attr_set[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (!attr_set[dev & 63]) {
      const int most = (int)(SORT_SMALL * sizeof(uint64_t));
      if ((e = cudaFuncSetAttribute(k_sort_small_reg<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, most)) !=
              cudaSuccess ||
          (e = cudaFuncSetAttribute(k_sort_small_reg<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, most)) !=
              cudaSuccess)
        return e;
      attr_set[dev & 63] = true;
    }
    // words per thread: the smallest power of two with 1024 E >= n
    const size_t per = sizeof(uint64_t) * SORT_SMALL_THREADS;
    const dim3 one(1), blk(SORT_SMALL_THREADS);
    cudaError_t le;
    if (n <= 1024u)
      le = launch_pdl(pdl, k_sort_small_reg<1>, one, blk, per, s, keys, n, keys_out, pos_out);
    else if (n <= 2048u)
      le = launch_pdl(pdl, k_sort_small_reg<2>, one, blk, 2 * per, s, keys, n, keys_out, pos_out);
    else if (n <= 4096u)
      le = launch_pdl(pdl, k_sort_small_reg<4>, one, blk, 4 * per, s, keys, n, keys_out, pos_out);
    else if (n <= 8192u)
      le = launch_pdl(pdl, k_sort_small_reg<8>, one, blk, 8 * per, s, keys, n, keys_out, pos_out);
    else
      le = launch_pdl(pdl, k_sort_small_reg<16>, one, blk, 16 * per, s, keys, n, keys_out, pos_out);
    if (le != cudaSuccess) return le;
    if (launches) *launches += 1;
    return cudaGetLastError();
  }
  if (tmp_bytes < argsort_temp_bytes(n)) return cudaErrorInvalidValue;
  const uint32_t ntiles = tiles_of(n);
  const uint32_t nh = ntiles * RS_BINS, nsums = (nh + SCAN_BLOCK - 1) / SCAN_BLOCK;
  char *t = static_cast<char *>(tmp);
  uint64_t *tk = reinterpret_cast<uint64_t *>(t);
  t += align256((size_t)n * 8);
  uint32_t *tv = reinterpret_cast<uint32_t *>(t);
  t += align256((size_t)n * 4);
  uint32_t *hist = reinterpret_cast<uint32_t *>(t);
  t += align256((size_t)nh * 4);
  uint32_t *sums = reinterpret_cast<uint32_t *>(t);
  const int passes = (end_bit + 7) / 8;
  const uint64_t *in_k = keys;
  const uint32_t *in_v = nullptr;
  for (int p = 0; p < passes; p++) {
    // the last pass lands in the outputs; passes before it alternate back
    // from there through the temporary pair
    const bool to_out = ((passes - 1 - p) & 1) == 0;
    uint64_t *ok = to_out ? keys_out : tk;
    uint32_t *ov = to_out ? pos_out : tv;
    const int shift = 8 * p;
    k_rs_hist<<<ntiles, RS_THREADS, 0, s>>>(in_k, n, shift, hist, ntiles);
    k_scan_sums<<<nsums, SCAN_BLOCK, 0, s>>>(hist, nh, sums);
    k_scan_top<<<1, SCAN_BLOCK, 0, s>>>(sums, nsums);
    k_scan_apply<<<nsums, SCAN_BLOCK, 0, s>>>(hist, nh, sums);
    k_rs_scatter<<<ntiles, RS_THREADS, 0, s>>>(in_k, in_v, n, shift, hist, ntiles, ok, ov);
    if (launches) *launches += 5;
    in_k = ok;
    in_v = ov;
  }
  return cudaGetLastError();
}

cudaError_t prewarm_sort_kernels() {
  const void *fns[] = {(const void *)k_sort_small, (const void *)k_rs_hist, (const void *)k_scan_sums,
                       (const void *)k_scan_top, (const void *)k_scan_apply, (const void *)k_rs_scatter};
  for (const void *f : fns) {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, f);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace ffb
