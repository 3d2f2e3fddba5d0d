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
};

void mx_prepare(const Dev& d, const MixBufs& mb, bool schwarz, cudaStream_t s, int64_t* lc);
int mx_pcg_grid_blocks(const Dev& d);
int mx_launch_pcg(const Dev& d, const MixBufs& mb, int maxIters, double tol, int blocks, cudaStream_t s);
// One-cluster PCG (mixed_cluster.cu): pA/pB are 3n-float direction buffers,
// coef one double per active contact.
int mx_cluster_size();
int mx_launch_pcg_cluster(const Dev& d, const MixBufs& mb, float* pA, float* pB, double* coef, int maxIters,
                          double tol, int clusterSize, cudaStream_t s);
void mx_grad_final(const Dev& d, cudaStream_t s, int64_t* lc);
void mx_energy_final(const Dev& d, cudaStream_t s, int64_t* lc);

}  // namespace cs
