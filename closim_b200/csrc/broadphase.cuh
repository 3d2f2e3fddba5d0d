// LBVH broadphase of the ContactSystem on the device (reference:
// src/backend/webgpu/gpu-broadphase.ts:193-386 for the FP32 mirror pipeline,
// src/collision/bvh.ts + contact-assembly.ts:87-140 for the candidate set).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "radix.cuh"

namespace cs {

// Device buffers of one broadphase (cloth triangles + optional static mesh).
struct BvhBufs {
  int m = 0, ns = 0, ms = 0;
  const uint32_t* idx = nullptr;    // cloth triangles (3m)
  const float* spos = nullptr;      // static vertices (3ns)
  const uint32_t* sidx = nullptr;   // static triangles (3ms)
  double* box64 = nullptr;          // 6m swept box, f64 (exact)
  float* boxc = nullptr;            // 6m the same box rounded outward to f32
  float* boxr = nullptr;            // 6m FP32 mirror box (round to nearest)
  float* cent = nullptr;            // 3m FP32 mirror centroid
  float* scene = nullptr;           // 6: centroid bbox
  Key<1>* k0 = nullptr; Key<1>* k1 = nullptr;
  uint32_t* p0 = nullptr; uint32_t* p1 = nullptr;
  uint32_t* hist = nullptr;
  int* left = nullptr; int* right = nullptr; int* parent = nullptr; int* depth = nullptr;
  float* nbox = nullptr;            // 6 (2m-1) node boxes
  uint32_t* visit = nullptr;        // 2m-1 refit arrival counters
  int* root = nullptr;              // 1
  uint32_t* cnt = nullptr;          // max(m, ms) + 1 per-query pair counts / offsets
  int2* pairs = nullptr;            // pair capacity
  int* flags = nullptr;             // [0] stack overflow
  const uint32_t* sortedKeys() const;  // unused helper declaration
};

// Builds boxes (pad), Morton keys, sorts them, builds the Karras hierarchy and
// refits it. mirror = true refits with the FP32 mirror boxes (bit-exact with
// the reference mirror); false refits with outward-rounded boxes of the exact
// f64 boxes (conservative).
void bvh_build(BvhBufs& b, const double* x0, const double* x1, double pad, bool mirror, cudaStream_t s,
               int64_t* launches);
// Pass 1 of the self traversal: per sorted leaf, the number of pairs.
void bvh_count_self(BvhBufs& b, bool mirror, cudaStream_t s, int64_t* launches);
// Pass 2: writes pairs at the scanned offsets.
void bvh_emit_self(BvhBufs& b, bool mirror, cudaStream_t s, int64_t* launches);
void bvh_count_static(BvhBufs& b, double pad, cudaStream_t s, int64_t* launches);
void bvh_emit_static(BvhBufs& b, double pad, int2* out, cudaStream_t s, int64_t* launches);
void scan_counts(uint32_t* cnt, int n, uint32_t* total, cudaStream_t s, int64_t* launches);

// Candidates: 15 per self pair (6 VT + 9 EE; void slots get kind 3), 12 per
// static pair (3 VT + 9 EE), sorted by (kind, p, a, b, c, d).
struct CandBufs {
  int cap = 0;
  int* rec = nullptr;       // 6 ints per candidate, unsorted
  int* srt = nullptr;       // 6 ints per candidate, sorted
  Key<4>* k0 = nullptr; Key<4>* k1 = nullptr;
  uint32_t* p0 = nullptr; uint32_t* p1 = nullptr;
  uint32_t* hist = nullptr;
};
void make_candidates(CandBufs& c, const uint32_t* idx, const uint32_t* sidx, int ns, const int2* selfPairs, int nSelf,
                     const int2* staticPairs, int nStatic, cudaStream_t s, int64_t* launches);

}  // namespace cs
