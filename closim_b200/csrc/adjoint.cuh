// Adjoint of the implicit step (adjoint.cu): device buffers and launchers.
#pragma once
#include "elem.cuh"
#include "plain.cuh"

namespace cs {

struct AdjArgs {
  Dev d;                 // x = x1 (the converged state H is evaluated at), contact frozen at x1
  const double* rhs;     // dL/dx1 (3n)
  double* mu;            // solution of H mu = rhs (3n)
  double *r, *z, *p, *Ap;  // PCG work (3n each)
  double* tri9;          // 9m element HVP
  double* hin12;         // 12hg hinge HVP
  double kb;             // bending stiffness (0: no bending term)
  int psd;               // 1: positive part of the membrane stress in the geometric term (forward Newton matrix)
  int maxIters;
  double tol;            // relative residual tolerance
  double* out;           // [iterations, residual, |rhs|]
};

int adj_grid_blocks(const Dev& d);
int adj_launch_pcg(const AdjArgs& a, int blocks, cudaStream_t s);
// acc[0..4) -= mu . dg/d(C00, C11, G, k) at d.x; terms: 4 (m + hg) doubles.
void adj_theta(const Dev& d, const double* mu, double* terms, double* acc, cudaStream_t s);
void adj_propagate(const Dev& d, const double* mu, double* lamX, double* lamV, double damp, cudaStream_t s);
// Forward Newton direction with the full FP64 Hessian (membrane with clamped
// compression, bending, frozen contact): dx = -H^-1 g into d.dx (a.mu must be
// d.dx, a.rhs scratch), then the reference's safeguards. Writes the scalars.
int newton_exact_solve(const AdjArgs& a, int blocks, cudaStream_t s);
void adj_rhs(const Dev& d, const double* lamX, const double* lamV, double damp, double* rhs, cudaStream_t s);

}  // namespace cs
