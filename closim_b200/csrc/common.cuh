// Shared device helpers for the closim B200 cloth solver.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cs {

namespace cg = cooperative_groups;

// JavaScript Math.max / Math.min semantics (NaN propagates).
template <class T>
__host__ __device__ __forceinline__ T js_max(T a, T b) {
  if (a != a || b != b) return a + b;
  if (a == 0 && b == 0) return signbit(a) ? b : a;
  return a > b ? a : b;
}
template <class T>
__host__ __device__ __forceinline__ T js_min(T a, T b) {
  if (a != a || b != b) return a + b;
  if (a == 0 && b == 0) return signbit(a) ? a : b;
  return a < b ? a : b;
}

// Math.hypot(a, b, c) with V8's algorithm (max-scaled, Kahan-compensated sum of
// squares). Compiled with -fmad=false on the FP64 path so it rounds exactly as V8.
template <class T>
__host__ __device__ __forceinline__ T js_hypot3(T a, T b, T c) {
  if (isinf(a) || isinf(b) || isinf(c)) return (T)INFINITY;
  if (a != a || b != b || c != c) return a + b + c;
  T v0 = fabs(a), v1 = fabs(b), v2 = fabs(c);
  T mx = 0;
  if (v0 > mx) mx = v0;
  if (v1 > mx) mx = v1;
  if (v2 > mx) mx = v2;
  if (mx == 0) return 0;
  T sum = 0, comp = 0;
  T vs[3] = {v0, v1, v2};
#pragma unroll
  for (int i = 0; i < 3; i++) {
    T nn = vs[i] / mx;
    T summand = nn * nn - comp;
    T prelim = sum + summand;
    comp = (prelim - sum) - summand;
    sum = prelim;
  }
  return sqrt(sum) * mx;
}

// Block-wide sum of one value per thread (fixed order: warp shuffle tree, then
// warp 0 sums the warp partials). Deterministic for a fixed block size.
template <class T>
__device__ __forceinline__ T block_sum(T v, T* smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  T r = 0;
  if (warp == 0) {
    r = lane < nw ? smem[lane] : (T)0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  if (threadIdx.x == 0) smem[0] = r;
  __syncthreads();
  r = smem[0];
  __syncthreads();
  return r;
}
template <class T>
__device__ __forceinline__ T block_max(T v, T* smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = js_max(v, __shfl_down_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  T r = 0;
  if (warp == 0) {
    r = lane < nw ? smem[lane] : (T)0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = js_max(r, __shfl_down_sync(0xffffffffu, r, o));
  }
  __syncthreads();
  if (threadIdx.x == 0) smem[0] = r;
  __syncthreads();
  r = smem[0];
  __syncthreads();
  return r;
}

// Block-wide minimum (identity +infinity; inputs must not be NaN).
__device__ __forceinline__ double block_min(double v, double* smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  double r = INFINITY;
  if (warp == 0) {
    r = lane < nw ? smem[lane] : INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = fmin(r, __shfl_down_sync(0xffffffffu, r, o));
  }
  __syncthreads();
  if (threadIdx.x == 0) smem[0] = r;
  __syncthreads();
  r = smem[0];
  __syncthreads();
  return r;
}

// Sum of nparts partials in a fixed order by one warp (every caller gets the
// same bits), used after a grid-wide barrier.
template <class T>
__device__ __forceinline__ T warp_sum_partials(const T* parts, int nparts) {
  const int lane = threadIdx.x & 31;
  T s = 0;
  for (int i = lane; i < nparts; i += 32) s += parts[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}
template <class T>
__device__ __forceinline__ T warp_max_partials(const T* parts, int nparts) {
  const int lane = threadIdx.x & 31;
  T s = 0;
  for (int i = lane; i < nparts; i += 32) s = js_max(s, parts[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s = js_max(s, __shfl_xor_sync(0xffffffffu, s, o));
  return s;
}

}  // namespace cs
