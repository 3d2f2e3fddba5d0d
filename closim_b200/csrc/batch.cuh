// Batched solver: many independent sheets of uneven size stepped together
// (no reference counterpart; each sheet follows newton.ts:27-303 with floor
// contact, src/collision/contact-assembly.ts restricted to kind 2).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cs {

// Per-sheet material and Newton constants (one row of 8 doubles).
enum BatchMat { BM_C00 = 0, BM_C11, BM_C01, BM_G, BM_THICK, BM_KB, BM_DAMP, BM_BETA, BM_N };
// Per-sheet results of the last step (one row of 8 doubles).
enum BatchOut { BO_NEWTON = 0, BO_PCG, BO_GRADNORM, BO_ENERGY, BO_CONVERGED, BO_TRIALS, BO_FLOOR, BO_REJECTED, BO_N };

struct BatchDev {
  int S;                       // sheets
  const int* vStart;           // S+1 vertex offsets
  const int* tStart;           // S+1 triangle offsets
  const int* hStart;           // S+1 hinge offsets
  const int* order;            // sheets, largest first (work list)
  // packed mesh: global vertex ids
  const uint32_t* idx;         // 3M
  const float4* inv;           // M
  const float* area;           // M
  const float* mass;           // N
  const int4* hinge;           // HG
  const double* hmeta;         // 3HG
  const uint32_t* memOff;      // N+1: vertex -> (tri << 2 | corner)
  const uint32_t* memRec;      // 3M
  const uint32_t* hinOff;      // N+1: vertex -> (hinge << 2 | corner)
  const uint32_t* hinRec;      // 4HG
  const uint8_t* pinned;       // N
  const double* pinPos;        // 3N (valid where pinned)
  const double* mat;           // S x BM_N
  // state and work (FP64, 3N)
  double *x, *v, *x0, *yHat, *g, *dx, *xt, *diag;
  double* elem;                // 9M gradient terms
  double* helem;               // 12HG gradient terms
  // FP32 linear solve
  float *r, *z, *p, *Ap, *xs;  // 3N
  float* dinv;                 // 3N inverse Jacobi diagonal of the current PCG (0 on pinned dofs)
  float* tris;                 // 16M: F (6), S (3), Dm^-1 (4), thickness * area, pad
  // floor contact, per vertex
  uint8_t* act;                // frozen active flag
  double* lagLam;              // lagged normal force
  uint8_t* lagOk;
  int hasFloor;
  double floorY, dHat, kappa, dMin, mu, eps;
  // step constants
  double h, invH2, gravity[3];
  int newtonIters, pcgMaxIters, lsIters;
  double gradTol;
  double* out;                 // S x BO_N
  unsigned int* work;          // work-list counter (reset before each launch)
};

// One launch steps every sheet once: persistent CTAs take sheets from the work
// list; a CTA runs its sheet's whole step with block barriers only.
int batch_launch_step(const BatchDev& b, int threads, int ctas, cudaStream_t s);
int batch_max_ctas(int threads);

}  // namespace cs
