// Mixed-precision path: FP32 PCG buffers and launchers (mixed.cu).
#pragma once
#include "plain.cuh"

namespace cs {

struct MixBufs {
  float *r, *z, *p, *Ap, *x;   // 3n each
  float* elem;                 // 9m element HVP terms
  float* tris;                 // 16m per-triangle F, S, Dm^-1, thickness * area
  float* h9;                   // 81m 9x9 blocks (Schwarz assembly)
  float* Linv;                 // D x 576 dense inverses
  // Vertex-major copies of the triangle state for the one-cluster PCG: record q
  // of the membrane incidence (tri << 2 | corner) holds that triangle's 16-float
  // state, its three vertex ids and the corner (5 float4, 80 B), so a vertex
  // reads its incident triangles contiguously with no index indirection.
  float4* vrec;                // 5 x 3m (null when unused)
  const uint32_t* triSlot;     // 3m: incidence record of (triangle, corner)
  float C00, C11, C01, G;
  // Exact-Newton mode: psd = 1 stores the positive part of S (psd_stress) in
  // the triangle records and the Schwarz blocks; hrec (4 float4 per hinge: the
  // 4 vertex ids, then the 12-value Gauss-Newton factor of bend_gn) adds the
  // bending term g (g . p) to the HVP. Both off in the reference mode.
  int psd;
  float4* hrec;
  // Two-level Schwarz (mas2): per domain the coarse diagonal (x, y, z) of
  // R A P; null for the one-level preconditioner.
  float4* dcoarse;
  // Schwarz assembly records per (vertex, incident triangle), in the v2t
  // order: x = the vertex's 3-row block offset in h9 (t * 81 + corner * 27),
  // y = the triangle corners' member indices in the vertex's domain, 4 bits
  // each (15: not a member); asmOff (n+1) indexes them per vertex. Null:
  // the factor derives them from the mesh.
  const uint32_t* asmOff;
  const uint2* asmRec;
};

// Two-level Schwarz share of lane (member l, component c) of a domain warp:
// omega Dc^-1 R r prolongated, = sc (omega / Dc[c]) sc sum_l' r[l', c] with
// sc = 1 / sqrt(|d|) and omega = 0.5 (applyMasTwoLevel, mas.ts:110-145).
__device__ __forceinline__ float coarse_share(const MixBufs& mb, int dom, float rv, int dv) {
  const int lane = threadIdx.x & 31, c = lane % 3;
  float rc = 0.f;
#pragma unroll
  for (int l = 0; l < 8; l++) rc += __shfl_sync(0xffffffffu, rv, l * 3 + c);
  const float dc = reinterpret_cast<const float*>(mb.dcoarse + dom)[c];
  const float sc2 = 1.f / (float)dv;  // sc * sc
  return dc > 1e-12f ? 0.5f * rc * sc2 / dc : 0.f;
}

// Device copy of the one-cluster PCG's per-CTA element lists (cluster_plan.hpp).
// resident = 1: phase A stages p on each CTA's halo in shared memory and runs
// the element HVPs from shared memory; 0: the vertex-major record gathers.
struct ClPlan {
  int resident;
  int smemBytes;  // dynamic shared memory of the launch
  int cCap;       // contact records per CTA kept on chip
  const int *vb, *haloOff, *halo, *triOff, *triId, *hinOff, *hinId, *incOff, *incHin, *ownHalo, *vDst;
  const ushort4 *triLoc, *hinLoc;
  const uint32_t* inc;
};

void mx_prepare(const Dev& d, const MixBufs& mb, bool schwarz, cudaStream_t s, int64_t* lc);
int mx_pcg_grid_blocks(const Dev& d);
int mx_launch_pcg(const Dev& d, const MixBufs& mb, int maxIters, double tol, int blocks, cudaStream_t s);
// One-cluster PCG (mixed_cluster.cu): pA/pB are 3n-float direction buffers,
// coef one double per active contact.
constexpr int kClWarps = 16;  // warps per CTA of the one-cluster PCG (512 threads)
int mx_cluster_size();
// True when a cluster of `clusterSize` CTAs with `smemBytes` of dynamic shared
// memory each can be co-scheduled (sets the kernel's shared-memory limit).
bool mx_cluster_resident_ok(int clusterSize, size_t smemBytes);
int mx_launch_pcg_cluster(const Dev& d, const MixBufs& mb, const ClPlan& plan, float* pA, float* pB, double* coef,
                          int maxIters, double tol, int clusterSize, cudaStream_t s);
void mx_grad_final(const Dev& d, cudaStream_t s, int64_t* lc);
void mx_energy_final(const Dev& d, cudaStream_t s, int64_t* lc);

}  // namespace cs
