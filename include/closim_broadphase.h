/* C ABI of the stand-alone LBVH broadphase (B200, sm_100a).
 *
 * Replaces the reference's BroadPhase interface (src/collision/broadphase.ts:61-64)
 * as implemented by GpuBroadPhase (src/backend/webgpu/gpu-broadphase.ts:147-386):
 *   new GpuBroadPhase({indices, triCount, pad, pairCapacity})  -> cs_broadphase_create
 *   build(x0, x1): Promise<CandidatePairs>                      -> cs_broadphase_build
 *   CandidatePairs.pairs (sorted by (a, b), a < b)              -> cs_broadphase_pairs
 *   CandidatePairs.diagnostics (broadphase.ts:35-53)            -> cs_broadphase_diagnostics
 *   lastMirror: GpuBroadPhaseMirrorState (gpu-broadphase.ts:39-52) -> cs_broadphase_state
 *
 * Positions are device pointers (the reference's build() takes buffers that are
 * already resident and reads no positions back). Every other pointer is host
 * memory. Calls are synchronous and not thread-safe per handle.
 */
#ifndef CLOSIM_BROADPHASE_H
#define CLOSIM_BROADPHASE_H

#include <stdint.h>

#include "closim_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cs_broadphase cs_broadphase;

/* Pair-set semantics of a handle. */
enum {
  /* The FP32 mirror's set: every box test on FP32 boxes, as GpuBroadPhase
   * (gpu-broadphase.ts:321-357). */
  CS_BROADPHASE_MIRROR = 0,
  /* The CPU TriBvh set (src/collision/bvh.ts:79-124): all non-adjacent pairs
   * whose padded f64 swept boxes overlap, inclusive. */
  CS_BROADPHASE_EXACT = 1
};

/* BroadPhaseDiagnostics (broadphase.ts:35-53) plus the tree's root and depth. */
typedef struct cs_broadphase_diag {
  int64_t scanned_count;     /* pairs found by the traversal */
  int64_t written_count;     /* pairs kept: min(scanned_count, capacity) */
  int64_t capacity;          /* pairCapacity */
  int32_t candidate_overflow; /* 1 when scanned_count > capacity */
  int32_t tree_depth;        /* levels, a leaf counting 1 */
  int32_t root;              /* root node index */
  int32_t reserved;
} cs_broadphase_diag;

/* n vertices, m triangles (indices: 3m, host). pair_capacity is the
 * reference's pairCapacity (default 16384 there). Returns NULL on invalid
 * arguments (an index >= n, m >= 1000003 as the reference's exclusion-key
 * decode requires, an unknown mode) or when device memory runs out. */
cs_broadphase* cs_broadphase_create(int32_t n, int32_t m, const uint32_t* indices, double pad,
                                    int64_t pair_capacity, int32_t mode);
void cs_broadphase_destroy(cs_broadphase* bp);
const char* cs_broadphase_last_error(cs_broadphase* bp);

/* Swept-box broadphase for the segment x0 -> x1 (device f64[3n] each).
 * CS_E_CAPACITY if a traversal needed a stack deeper than 64 entries. */
int cs_broadphase_build(cs_broadphase* bp, const double* x0, const double* x1);
int cs_broadphase_diagnostics(cs_broadphase* bp, cs_broadphase_diag* out);
/* written_count pairs (a, b), a < b, ascending: int32[2 * written_count]. */
int cs_broadphase_pairs(cs_broadphase* bp, int32_t* pairs);
/* The LBVH of the last build, in GpuBroadPhaseMirrorState's layout (any
 * pointer may be NULL): aabb f32[6m] (FP32 swept box), centroid f32[3m],
 * morton u32[m] and payload u32[m] in sorted order, node_min/node_max
 * f32[3(2m-1)], node_left/node_right/node_leaf_tri i32[2m-1] (internal nodes
 * 0..m-2, leaves m-1..2m-2; -1 where absent). In CS_BROADPHASE_EXACT mode the
 * node boxes are the outward-rounded f32 boxes of the f64 swept boxes. */
int cs_broadphase_state(cs_broadphase* bp, float* aabb, float* centroid, uint32_t* morton, uint32_t* payload,
                        float* node_min, float* node_max, int32_t* node_left, int32_t* node_right,
                        int32_t* node_leaf_tri);

#ifdef __cplusplus
}
#endif

#endif /* CLOSIM_BROADPHASE_H */
