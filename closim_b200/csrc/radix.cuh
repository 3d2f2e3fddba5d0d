// Stable LSD radix sort of (key, payload) records on the device, hand-written.
//
// Keys are KW 32-bit words, most significant word first (word 0); each pass
// sorts one 8-bit digit: a per-tile histogram, one exclusive scan over
// (digit, tile), then a stable scatter in which each tile ranks its elements
// with warp match + per-warp digit counters. Passes run from the least
// significant digit up, so equal keys keep their input order (a stable sort,
// which is what makes the (key, index) orders of the reference reproducible).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cs {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;                        // rows per tile
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 elements

template <int KW>
struct Key {
  uint32_t w[KW];
};

template <int KW>
__device__ __forceinline__ uint32_t digit_of(const Key<KW>& k, int pass) {
  // pass 0 = least significant byte of the last word
  const int word = KW - 1 - pass / 4;
  return (k.w[word] >> ((pass % 4) * 8)) & 0xffu;
}

// dn (optional): the element count, read on the device when the launch was
// sized for a capacity n (graph-captured steps, where the host does not know it).
template <int KW>
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const Key<KW>* keys, int n, int pass, uint32_t* hist,
                                                             int ntiles, const int* dn = nullptr) {
  if (dn) n = min(n, *dn);
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int base = blockIdx.x * kSortTile;
  for (int r = 0; r < kSortItems; r++) {
    const int i = base + r * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[digit_of(keys[i], pass)], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of `n` u32 in place by one block: chunks of 4096 (4 per
// thread), warp-shuffle scans of the thread totals, one running carry.
static __global__ void __launch_bounds__(1024) k_scan_exclusive(uint32_t* a, int n, uint32_t* total) {
  __shared__ uint32_t wsum[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t carry = 0;
  for (int base = 0; base < n; base += 4096) {
    const int i0 = base + threadIdx.x * 4;
    uint32_t v[4];
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = i0 + k < n ? a[i0 + k] : 0u;
    const uint32_t t = v[0] + v[1] + v[2] + v[3];
    uint32_t incl = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      wsum[lane] = w;
    }
    __syncthreads();
    uint32_t excl = carry + (warp > 0 ? wsum[warp - 1] : 0u) + incl - t;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      if (i0 + k < n) a[i0 + k] = excl;
      excl += v[k];
    }
    carry += wsum[31];
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

template <int KW>
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const Key<KW>* kin, const uint32_t* pin, Key<KW>* kout,
                                                                uint32_t* pout, int n, int pass, const uint32_t* offs,
                                                                int ntiles, const int* dn = nullptr) {
  if (dn) n = min(n, *dn);
  __shared__ uint32_t running[256];
  __shared__ uint32_t wcount[kSortThreads / 32][256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  running[threadIdx.x] = offs[threadIdx.x * ntiles + blockIdx.x];
  for (int w = 0; w < kSortThreads / 32; w++) wcount[w][threadIdx.x] = 0;
  __syncthreads();
  const int base = blockIdx.x * kSortTile;
  const uint32_t lt = (1u << lane) - 1u;
  for (int r = 0; r < kSortItems; r++) {
    const int i = base + r * kSortThreads + threadIdx.x;
    const bool valid = i < n;
    Key<KW> k;
    uint32_t pl = 0;
    int dg = -1;
    if (valid) {
      k = kin[i];
      pl = pin[i];
      dg = (int)digit_of(k, pass);
    }
    const uint32_t peers = __match_any_sync(0xffffffffu, dg);
    const uint32_t rank = __popc(peers & lt);
    if (valid && rank == 0) wcount[warp][dg] = __popc(peers);
    __syncthreads();
    if (valid) {
      uint32_t off = running[dg] + rank;
      for (int w = 0; w < warp; w++) off += wcount[w][dg];
      kout[off] = k;
      pout[off] = pl;
    }
    __syncthreads();
    uint32_t tot = 0;
    for (int w = 0; w < kSortThreads / 32; w++) {
      tot += wcount[w][threadIdx.x];
      wcount[w][threadIdx.x] = 0;
    }
    running[threadIdx.x] += tot;
    __syncthreads();
  }
}

// All passes of a stable LSD radix sort in ONE thread block (1024 threads), for
// sorts small enough that launch latency dominates. Warp w owns the w-th
// contiguous chunk; per pass: per-warp digit counts, one scan over (digit,
// warp) in shared memory, then each warp scatters its chunk in order (32 keys
// at a time, ranked with warp match), which keeps the sort stable.
constexpr int kBlockSortThreads = 1024;
constexpr int kBlockSortMax = 32768;

template <int KW>
__global__ void __launch_bounds__(kBlockSortThreads) k_block_radix(Key<KW>* k0, uint32_t* p0, Key<KW>* k1,
                                                                   uint32_t* p1, int n, int passes,
                                                                   const int* dn = nullptr) {
  if (dn) n = max(0, min(n, *dn));
  __shared__ uint32_t cnt[kBlockSortThreads / 32][256];
  __shared__ uint32_t tot[256];
  __shared__ uint32_t orw[KW], andw[KW];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kWarps = kBlockSortThreads / 32;
  constexpr int kB = KW <= 1 ? 8 : KW <= 4 ? 4 : 2;  // records per lane in flight
  const int chunk = ((n + kWarps - 1) / kWarps + 31) & ~31;
  const int lo = min(n, warp * chunk), hi = min(n, lo + chunk);
  const uint32_t lt = (1u << lane) - 1u;
  // Bits that differ between keys: a pass whose digit is the same for every
  // key would leave the (stable) order as it is, so it is skipped.
  if (threadIdx.x < KW) { orw[threadIdx.x] = 0u; andw[threadIdx.x] = ~0u; }
  __syncthreads();
  {
    uint32_t o[KW], a[KW];
#pragma unroll
    for (int w = 0; w < KW; w++) { o[w] = 0u; a[w] = ~0u; }
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const Key<KW> k = k0[i];
#pragma unroll
      for (int w = 0; w < KW; w++) { o[w] |= k.w[w]; a[w] &= k.w[w]; }
    }
#pragma unroll
    for (int w = 0; w < KW; w++) {
      o[w] = __reduce_or_sync(0xffffffffu, o[w]);
      a[w] = __reduce_and_sync(0xffffffffu, a[w]);
      if (lane == 0) { atomicOr(&orw[w], o[w]); atomicAnd(&andw[w], a[w]); }
    }
  }
  __syncthreads();
  int flip = 0;  // executed passes, mod 2: the records are in (k1, p1) when set
  for (int pass = 0; pass < passes; pass++) {
    const int dw = KW - 1 - pass / 4, sh = (pass % 4) * 8;
    if ((((orw[dw] ^ andw[dw]) >> sh) & 0xffu) == 0u) continue;
    const Key<KW>* ki = flip ? k1 : k0;
    const uint32_t* pi = flip ? p1 : p0;
    Key<KW>* ko = flip ? k0 : k1;
    uint32_t* po = flip ? p0 : p1;
    flip ^= 1;
    for (int w = 0; w < kWarps; w++)
      if (threadIdx.x < 256) cnt[w][threadIdx.x] = 0;
    __syncthreads();
    // histogram: each lane loads kB keys of its warp's chunk before counting
    // any, so the loads of a batch are in flight together
    for (int base = lo; base < hi; base += 32 * kB) {
      int dg[kB];
#pragma unroll
      for (int u = 0; u < kB; u++) {
        const int i = base + u * 32 + lane;
        dg[u] = i < hi ? (int)digit_of(ki[i], pass) : -1;
      }
#pragma unroll
      for (int u = 0; u < kB; u++) {
        const uint32_t peers = __match_any_sync(0xffffffffu, dg[u]);
        if (dg[u] >= 0 && (peers & lt) == 0) cnt[warp][dg[u]] += __popc(peers);
        __syncwarp();
      }
    }
    __syncthreads();
    // exclusive offsets: digit-major, warp-minor
    if (threadIdx.x < 256) {
      uint32_t run = 0;
      for (int w = 0; w < kWarps; w++) {
        const uint32_t c = cnt[w][threadIdx.x];
        cnt[w][threadIdx.x] = run;
        run += c;
      }
      tot[threadIdx.x] = run;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      // scan of the 256 digit totals: 8 per lane, then across lanes
      uint32_t v[8], sum = 0;
      for (int q = 0; q < 8; q++) { v[q] = tot[threadIdx.x * 8 + q]; sum += v[q]; }
      uint32_t incl = sum;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      uint32_t run = incl - sum;
      for (int q = 0; q < 8; q++) { tot[threadIdx.x * 8 + q] = run; run += v[q]; }
    }
    __syncthreads();
    if (threadIdx.x < 256)
      for (int w = 0; w < kWarps; w++) cnt[w][threadIdx.x] += tot[threadIdx.x];
    __syncthreads();
    // stable scatter in the same order, kB records per lane loaded at once
    for (int base = lo; base < hi; base += 32 * kB) {
      Key<KW> k[kB];
      uint32_t pl[kB];
#pragma unroll
      for (int u = 0; u < kB; u++) {
        const int i = base + u * 32 + lane;
        if (i < hi) {
          k[u] = ki[i];
          pl[u] = pi[i];
        }
      }
#pragma unroll
      for (int u = 0; u < kB; u++) {
        const int i = base + u * 32 + lane;
        const bool valid = i < hi;
        const int dg = valid ? (int)digit_of(k[u], pass) : -1;
        const uint32_t peers = __match_any_sync(0xffffffffu, dg);
        if (valid) {
          const uint32_t off = cnt[warp][dg] + __popc(peers & lt);
          ko[off] = k[u];
          po[off] = pl[u];
        }
        __syncwarp();
        if (valid && (peers & lt) == 0) cnt[warp][dg] += __popc(peers);
        __syncwarp();
      }
    }
    __syncthreads();
  }
  // The caller expects the records where `passes` executed passes would leave them.
  if (flip != (passes & 1)) {
    const Key<KW>* ks = flip ? k1 : k0;
    const uint32_t* ps = flip ? p1 : p0;
    Key<KW>* kd = flip ? k0 : k1;
    uint32_t* pd = flip ? p0 : p1;
    for (int i = threadIdx.x; i < n; i += blockDim.x) { kd[i] = ks[i]; pd[i] = ps[i]; }
  }
}

// Sorts n records by key over the low `bits` bits of the key (counted from the
// least significant end). Ping-pongs between (k0,p0) and (k1,p1); returns true
// when the result ended in (k1,p1). hist must hold 256 * ceil(n / 2048) + 1 u32.
template <int KW>
bool radix_sort(Key<KW>* k0, uint32_t* p0, Key<KW>* k1, uint32_t* p1, int n, int bits, uint32_t* hist,
                cudaStream_t s, int64_t* launches) {
  if (n <= 1) return false;
  const int ntiles = (n + kSortTile - 1) / kSortTile;
  const int passes = (bits + 7) / 8;
  if (n <= kBlockSortMax) {
    k_block_radix<KW><<<1, kBlockSortThreads, 0, s>>>(k0, p0, k1, p1, n, passes);
    if (launches) *launches += 1;
    return (passes & 1) != 0;
  }
  bool flip = false;
  for (int pass = 0; pass < passes; pass++) {
    const Key<KW>* ki = flip ? k1 : k0;
    const uint32_t* pi = flip ? p1 : p0;
    Key<KW>* ko = flip ? k0 : k1;
    uint32_t* po = flip ? p0 : p1;
    k_radix_hist<KW><<<ntiles, kSortThreads, 0, s>>>(ki, n, pass, hist, ntiles);
    k_scan_exclusive<<<1, 1024, 0, s>>>(hist, 256 * ntiles, nullptr);
    k_radix_scatter<KW><<<ntiles, kSortThreads, 0, s>>>(ki, pi, ko, po, n, pass, hist, ntiles);
    if (launches) *launches += 3;
    flip = !flip;
  }
  return flip;
}

// The same sort with the element count read on the device (*dn, at most cap):
// every launch is sized for cap, so the sequence can be captured in a graph
// before the count exists. The result lands where radix_sort would put it for
// the same `bits` (the returned flag depends on cap and bits only).
template <int KW>
bool radix_sort_dev(Key<KW>* k0, uint32_t* p0, Key<KW>* k1, uint32_t* p1, const int* dn, int cap, int bits,
                    uint32_t* hist, cudaStream_t s, int64_t* launches) {
  const int passes = (bits + 7) / 8;
  if (cap <= kBlockSortMax) {
    k_block_radix<KW><<<1, kBlockSortThreads, 0, s>>>(k0, p0, k1, p1, cap, passes, dn);
    if (launches) *launches += 1;
    return (passes & 1) != 0;
  }
  const int ntiles = (cap + kSortTile - 1) / kSortTile;
  bool flip = false;
  for (int pass = 0; pass < passes; pass++) {
    const Key<KW>* ki = flip ? k1 : k0;
    const uint32_t* pi = flip ? p1 : p0;
    Key<KW>* ko = flip ? k0 : k1;
    uint32_t* po = flip ? p0 : p1;
    k_radix_hist<KW><<<ntiles, kSortThreads, 0, s>>>(ki, cap, pass, hist, ntiles, dn);
    k_scan_exclusive<<<1, 1024, 0, s>>>(hist, 256 * ntiles, nullptr);
    k_radix_scatter<KW><<<ntiles, kSortThreads, 0, s>>>(ki, pi, ko, po, cap, pass, hist, ntiles, dn);
    if (launches) *launches += 3;
    flip = !flip;
  }
  return flip;
}

}  // namespace cs
