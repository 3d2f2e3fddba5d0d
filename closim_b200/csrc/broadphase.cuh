// LBVH broadphase of the ContactSystem on the device (reference:
// src/backend/webgpu/gpu-broadphase.ts:193-386 for the FP32 mirror pipeline,
// src/collision/bvh.ts + contact-assembly.ts:87-140 for the candidate set).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "radix.cuh"

namespace cs {

// Device buffers of one broadphase (cloth triangles + optional static mesh).
//
// Node numbering follows the Karras build: internal nodes 0..m-2, leaf of
// sorted position s at m-1+s. For traversal every internal node i also owns a
// 64-byte record rec[4i..4i+3] holding both children's boxes and codes:
//   rec[4i+0] = (L.min.xyz, code L)   rec[4i+1] = (L.max.xyz, 0)
//   rec[4i+2] = (R.min.xyz, code R)   rec[4i+3] = (R.max.xyz, 0)
// where code >= 0 is an internal node and code < 0 is the leaf of triangle
// ~code. One popped node costs one 64-byte read; no per-child lookups.
struct BvhBufs {
  int m = 0, ns = 0, ms = 0;
  const uint32_t* idx = nullptr;    // cloth triangles (3m)
  const float* spos = nullptr;      // static vertices (3ns)
  const uint32_t* sidx = nullptr;   // static triangles (3ms)
  double* box64 = nullptr;          // 6m swept box, f64 (exact), by triangle id
  float* boxc = nullptr;            // 6m the same box rounded outward to f32
  float* boxr = nullptr;            // 6m FP32 mirror box (round to nearest)
  float* cent = nullptr;            // 3m FP32 mirror centroid
  float* scene = nullptr;           // 6: centroid bbox
  Key<1>* k0 = nullptr; Key<1>* k1 = nullptr;
  uint32_t* p0 = nullptr; uint32_t* p1 = nullptr;
  uint32_t* hist = nullptr;
  int* left = nullptr; int* right = nullptr; int* parent = nullptr; int* depth = nullptr;
  float* nbox = nullptr;            // 6 (2m-1) node boxes
  float4* rec = nullptr;            // 4 (m-1) traversal records
  uint32_t* visit = nullptr;        // 2m-1 refit arrival counters
  int* root = nullptr;              // 1
  uint32_t* cnt = nullptr;          // per-query pair counts / offsets (two-pass mode), or [0] = total (append mode)
  int2* pairs = nullptr;            // pair capacity
  uint32_t pairCap = 0;             // append mode: pairs beyond this are counted, not written
  int* flags = nullptr;             // [0] stack overflow / malformed tree
};

// Builds boxes (pad), Morton keys, sorts them, builds the Karras hierarchy and
// refits it. mirror = true refits with the FP32 mirror boxes (bit-exact with
// the reference mirror); false refits with outward-rounded boxes of the exact
// f64 boxes (conservative).
void bvh_build(BvhBufs& b, const double* x0, const double* x1, double pad, bool mirror, cudaStream_t s,
               int64_t* launches);
// Recomputes the boxes for a new segment and refits the existing hierarchy
// (topology kept). Valid for the exact pair set, which does not depend on the
// tree's shape.
void bvh_refit(BvhBufs& b, const double* x0, const double* x1, double pad, bool mirror, cudaStream_t s,
               int64_t* launches);
// Two-pass self traversal in the reference's per-leaf stack order: counts per
// sorted leaf, then writes pairs at the scanned offsets.
void bvh_count_self(BvhBufs& b, bool mirror, cudaStream_t s, int64_t* launches);
void bvh_emit_self(BvhBufs& b, bool mirror, cudaStream_t s, int64_t* launches);
// One-pass self traversal: pairs appended in arbitrary order through a global
// counter b.cnt[0] (which must start at 0); the exact set only.
void bvh_append_self(BvhBufs& b, cudaStream_t s, int64_t* launches);
// Static triangles against the cloth hierarchy, appended through cnt[0].
void bvh_append_static(BvhBufs& b, double pad, int2* out, uint32_t cap, uint32_t* cnt, cudaStream_t s,
                       int64_t* launches);
void scan_counts(uint32_t* cnt, int n, uint32_t* total, cudaStream_t s, int64_t* launches);
// Swept boxes of a new segment only (box64 / boxc / boxr / centroids), no refit.
void bvh_boxes(BvhBufs& b, const double* x0, const double* x1, double pad, cudaStream_t s, int64_t* launches);
// Exact query against a superset of pairs: keeps the self pairs whose current
// f64 boxes overlap (adjacency was excluded when the superset was built) and
// the static pairs whose cloth box overlaps the static box padded by `pad`;
// appended through cnt[0] / scnt[0] (order arbitrary).
void filter_pairs(const BvhBufs& b, const int2* sup, int nsup, int2* out, uint32_t cap, uint32_t* cnt,
                  const int2* ssup, int nssup, double pad, int2* sout, uint32_t scap, uint32_t* scnt, cudaStream_t s,
                  int64_t* launches);
void filter_pairs_dev(const BvhBufs& b, const int2* sup, int nsup, int2* out, uint32_t cap, uint32_t* cnt,
                      const int2* ssup, int nssup, double pad, int2* sout, uint32_t scap, uint32_t* scnt,
                      const int* dn, cudaStream_t s, int64_t* launches);

// Sort buffers for the order keys of candidates (15 per self pair, 12 per
// static pair; the records are decoded from the pairs where they are used).
struct CandBufs {
  int cap = 0;
  Key<4>* k0 = nullptr; Key<4>* k1 = nullptr;
  uint32_t* p0 = nullptr; uint32_t* p1 = nullptr;
  uint32_t* hist = nullptr;
};

// Order key of a candidate (contact-assembly.ts:118: kind, p, a, b, c, d),
// packed as a 128-bit integer (w[0] most significant) with `bits` bits per id;
// ids are offset by ns + 2 so static ids -(i+2), -2 and -1 order below cloth
// ids. `tail` extra low bits are appended (zero for sorting).
struct CandKey {
  uint64_t hi, lo;
};
__host__ __device__ inline int cand_id_bits(int n, int ns) {
  const long range = (long)n + ns + 2;
  int b = 1;
  while ((1l << b) < range) b++;
  return b;
}
__device__ __forceinline__ void shl128_or(CandKey& k, int sh, uint64_t v) {
  // k = (k << sh) | v, with v < 2^sh and 0 < sh < 64
  k.hi = (k.hi << sh) | (k.lo >> (64 - sh));
  k.lo = (k.lo << sh) | v;
}
__device__ __forceinline__ CandKey cand_key(const int* r, int ns, int bits, int tail, uint64_t tailVal) {
  const int64_t off = (int64_t)ns + 2;
  CandKey k{0, (uint64_t)r[0]};
  for (int q = 1; q < 6; q++) shl128_or(k, bits, (uint64_t)((int64_t)r[q] + off));
  if (tail > 0) shl128_or(k, tail, tailVal);
  return k;
}
__host__ __device__ inline int cand_key_bits(int bits, int tail) { return 2 + 5 * bits + tail; }

}  // namespace cs
