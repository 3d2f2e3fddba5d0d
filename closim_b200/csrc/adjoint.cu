// Adjoint of the implicit-Euler step through the implicit-function theorem
// (no reference counterpart; it differentiates newton.ts:27-232).
//
// A converged step satisfies g(x1; x0, v0, theta) = 0 with
//   g = M (x1 - yHat) / h^2 + grad E_membrane(x1; C00, C11, C01, G)
//       + grad E_bend(x1; k) + grad E_contact(x1),   yHat = x0 + h v0 + h^2 g_grav,
// so for a loss L(x1): H mu = dL/dx1 (H = dg/dx1, symmetric), and
//   dL/dtheta = -mu . dg/dtheta,  dL/dx0 = M mu / h^2,  dL/dv0 = M mu / h.
// H is applied matrix-free in FP64: M/h^2, the analytic membrane HVP
// (membrane-hvp.ts:18-75), the exact bending HVP (dual numbers over the
// analytic hinge gradient) and the frozen-contact barrier HVP
// (contact-assembly.ts:371-414, active set frozen at x1). Friction and the
// restitution filter are treated as constants, as the forward Newton HVP
// treats friction. Pinned dofs are filtered out of every vector.
//
// dg/dtheta: the membrane gradient is linear in (C00, C11, C01, G), so its
// derivative along C00 is the gradient evaluated with C00 = 1 and the others 0
// (likewise C11, G); the bending gradient is linear in k, so its derivative is
// the analytic hinge gradient at k = 1, the gradient the exact-Newton forward
// takes (the derivative of bending.ts:7-16).
#include <cooperative_groups.h>

#include "adjoint.cuh"
#include "adjoint_math.cuh"
#include "contact.cuh"

namespace cg = cooperative_groups;

namespace cs {

__device__ __forceinline__ void load3(const double* x, int v, double o[3]) {
  o[0] = x[v * 3]; o[1] = x[v * 3 + 1]; o[2] = x[v * 3 + 2];
}

__device__ __forceinline__ double adj_total(const Dev& d, int row, double* bc) {
  if (threadIdx.x < 32) {
    const double s = warp_sum_partials(d.part + row * d.partStride, gridDim.x);
    if (threadIdx.x == 0) bc[0] = s;
  }
  __syncthreads();
  const double r = bc[0];
  __syncthreads();
  return r;
}
__device__ __forceinline__ void adj_put(const Dev& d, int row, double v, double* sm) {
  const double b = block_sum(v, sm);
  if (threadIdx.x == 0) d.part[row * d.partStride + blockIdx.x] = b;
}

// z = M^-1 r on one Schwarz domain with the FP64 factors in d.L (the
// forward's Cholesky factor, or an inverse diagonal where it failed).
__device__ double adj_schwarz(const Dev& d, const double* r, double* z, int dom) {
  const int start = d.domStart[dom], dv = d.domStart[dom + 1] - start, dw = dv * 3;
  const double* L = d.L + (size_t)dom * 576;
  double rhs[24], y[24], sol[24];
  for (int l = 0; l < dv; l++) {
    const int v = d.domVerts[start + l];
    for (int k = 0; k < 3; k++) rhs[l * 3 + k] = r[v * 3 + k];
  }
  if (d.domFlag[dom]) {
    for (int i = 0; i < dw; i++) {
      double s = rhs[i];
      for (int j = 0; j < i; j++) s -= L[i * 24 + j] * y[j];
      y[i] = s / L[i * 24 + i];
    }
    for (int i = dw - 1; i >= 0; i--) {
      double s = y[i];
      for (int j = i + 1; j < dw; j++) s -= L[j * 24 + i] * sol[j];
      sol[i] = s / L[i * 24 + i];
    }
  } else {
    for (int i = 0; i < dw; i++) {
      double s = 0;
      for (int j = 0; j < dw; j++) s += L[i * 24 + j] * rhs[j];
      sol[i] = s;
    }
  }
  double rz = 0;
  for (int l = 0; l < dv; l++) {
    const int v = d.domVerts[start + l];
    const bool pin = d.pinned[v];
    for (int k = 0; k < 3; k++) {
      const double zz = pin ? 0.0 : sol[l * 3 + k];
      z[v * 3 + k] = zz;
      rz += rhs[l * 3 + k] * zz;
    }
  }
  return rz;
}

__device__ __forceinline__ double adj_precond(const Dev& d, const AdjArgs& A, int tid, int nth) {
  double rz = 0;
  if (d.precond >= 1) {  // one-level Schwarz factors (the two-level coarse term is not applied here)
    for (int dom = tid; dom < d.D; dom += nth) rz += adj_schwarz(d, A.r, A.z, dom);
  } else {
    for (int i = tid; i < d.n * 3; i += nth) {
      const double ri = A.r[i];
      double zi = d.diag[i] > 1e-12 ? ri / d.diag[i] : ri;
      if (d.pinned[i / 3]) zi = 0;
      A.z[i] = zi;
      rz += ri * zi;
    }
  }
  return rz;
}

// Membrane HVP in FP64 (membrane-hvp.ts:18-75). With psd set, the second
// Piola stress S in the geometric term dF S is replaced by its positive part
// (negative principal stresses of a compressed triangle clamped to zero), which
// makes every element block positive semi-definite: a Newton matrix for the
// forward solve that leaves its converged solution unchanged.
__device__ __forceinline__ void mem_hvp64(const double* x0, const double* x1, const double* x2, const double* v0,
                                          const double* v1, const double* v2, double a, double b, double c, double d,
                                          double area, const Mat<double>& m, bool psd, double out[9]) {
  double F0[3], F1[3], dF0[3], dF1[3];
  for (int k = 0; k < 3; k++) {
    const double e1 = x1[k] - x0[k], e2 = x2[k] - x0[k];
    const double w1 = v1[k] - v0[k], w2 = v2[k] - v0[k];
    F0[k] = a * e1 + c * e2;
    F1[k] = b * e1 + d * e2;
    dF0[k] = a * w1 + c * w2;
    dF1[k] = b * w1 + d * w2;
  }
  const double E00 = 0.5 * (F0[0] * F0[0] + F0[1] * F0[1] + F0[2] * F0[2] - 1);
  const double E11 = 0.5 * (F1[0] * F1[0] + F1[1] * F1[1] + F1[2] * F1[2] - 1);
  const double E01 = 0.5 * (F0[0] * F1[0] + F0[1] * F1[1] + F0[2] * F1[2]);
  const double dE00 = F0[0] * dF0[0] + F0[1] * dF0[1] + F0[2] * dF0[2];
  const double dE11 = F1[0] * dF1[0] + F1[1] * dF1[1] + F1[2] * dF1[2];
  const double dE01 = 0.5 * (dF0[0] * F1[0] + F0[0] * dF1[0] + dF0[1] * F1[1] + F0[1] * dF1[1] + dF0[2] * F1[2] +
                             F0[2] * dF1[2]);
  double S00 = m.C00 * E00 + m.C01 * E11;
  double S11 = m.C11 * E11 + m.C01 * E00;
  double S01 = 2 * m.G * E01;
  if (psd) psd_stress(S00, S11, S01);
  const double dS00 = m.C00 * dE00 + m.C01 * dE11;
  const double dS11 = m.C11 * dE11 + m.C01 * dE00;
  const double dS01 = 2 * m.G * dE01;
  const double s = m.thickness * area;
  for (int k = 0; k < 3; k++) {
    const double P0 = dF0[k] * S00 + F0[k] * dS00 + dF1[k] * S01 + F1[k] * dS01;
    const double P1 = dF0[k] * S01 + F0[k] * dS01 + dF1[k] * S11 + F1[k] * dS11;
    const double g1 = s * (P0 * a + P1 * b);
    const double g2 = s * (P0 * c + P1 * d);
    out[k] = -(g1 + g2);
    out[3 + k] = g1;
    out[6 + k] = g2;
  }
}

// H p into A.Ap (element pass, grid barrier, gather); returns the partial p.Hp.
__device__ double adj_hvp(cg::grid_group& grid, const Dev& d, const AdjArgs& A, int tid, int nth) {
  for (int t = tid; t < d.m; t += nth) {
    const uint32_t i0 = d.idx[t * 3], i1 = d.idx[t * 3 + 1], i2 = d.idx[t * 3 + 2];
    double x0[3], x1[3], x2[3], v0[3], v1[3], v2[3];
    load3(d.x, i0, x0); load3(d.x, i1, x1); load3(d.x, i2, x2);
    load3(A.p, i0, v0); load3(A.p, i1, v1); load3(A.p, i2, v2);
    const float4 iv = d.inv[t];
    double o[9];
    mem_hvp64(x0, x1, x2, v0, v1, v2, iv.x, iv.y, iv.z, iv.w, d.area[t], d.mat, A.psd != 0, o);
    for (int k = 0; k < 9; k++) A.tri9[(size_t)t * 9 + k] = o[k];
  }
  if (A.kb > 0)
    for (int hh = tid; hh < d.hg; hh += nth) {
      const int4 hv = d.hinge[hh];
      double q[12], v[12], o[12];
      load3(d.x, hv.x, q); load3(d.x, hv.y, q + 3); load3(d.x, hv.z, q + 6); load3(d.x, hv.w, q + 9);
      load3(A.p, hv.x, v); load3(A.p, hv.y, v + 3); load3(A.p, hv.z, v + 6); load3(A.p, hv.w, v + 9);
      bend_hvp(q, v, d.hmeta[hh * 3], d.hmeta[hh * 3 + 1], d.hmeta[hh * 3 + 2], A.kb, o);
      for (int k = 0; k < 12; k++) A.hin12[(size_t)hh * 12 + k] = o[k];
    }
  if (d.hasContact) contact_hvp_coeffs(d, A.p, tid, nth);
  grid.sync();
  double pAp = 0;
  for (int v = tid; v < d.n; v += nth) {
    double s[3] = {0, 0, 0};
    for (uint32_t k = d.memOff[v]; k < d.memOff[v + 1]; k++) {
      const uint32_t rec = d.memRec[k];
      const double* e = A.tri9 + (size_t)(rec >> 2) * 9 + (rec & 3) * 3;
      s[0] += e[0]; s[1] += e[1]; s[2] += e[2];
    }
    if (A.kb > 0)
      for (uint32_t k = d.hinOff[v]; k < d.hinOff[v + 1]; k++) {
        const uint32_t rec = d.hinRec[k];
        const double* e = A.hin12 + (size_t)(rec >> 2) * 12 + (rec & 3) * 3;
        s[0] += e[0]; s[1] += e[1]; s[2] += e[2];
      }
    double ch[3] = {0, 0, 0};
    if (d.hasContact) contact_hvp_gather(d, v, ch);
    const double M = d.mass[v];
    const bool pin = d.pinned[v];
    for (int k = 0; k < 3; k++) {
      const int i = v * 3 + k;
      const double ap = pin ? 0.0 : M * A.p[i] * d.invH2 + s[k] + ch[k];
      A.Ap[i] = ap;
      pAp += A.p[i] * ap;
    }
  }
  return pAp;
}

// PCG on H mu = rhs (pcg.ts's recurrence, FP64 tree reductions), one
// cooperative launch. out: [iterations, final residual, |rhs|].
__global__ void __launch_bounds__(kThreads) k_adj_pcg(AdjArgs A) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double sm[32];
  __shared__ double bc[2];
  const Dev& d = A.d;
  const int n3 = d.n * 3;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  double bb = 0, rr = 0;
  for (int i = tid; i < n3; i += nth) {
    const double ri = d.pinned[i / 3] ? 0.0 : A.rhs[i];
    bb += A.rhs[i] * A.rhs[i];
    A.r[i] = ri;
    A.mu[i] = 0;
    rr += ri * ri;
  }
  grid.sync();
  const double rz0 = adj_precond(d, A, tid, nth);
  adj_put(d, 0, bb, sm);
  adj_put(d, 1, rr, sm);
  adj_put(d, 2, rz0, sm);
  grid.sync();
  for (int i = tid; i < n3; i += nth) A.p[i] = A.z[i];
  const double bNorm = sqrt(adj_total(d, 0, bc));
  double residual = sqrt(adj_total(d, 1, bc));
  double rz = adj_total(d, 2, bc);
  const double absTol = fmax(A.tol * bNorm, 1e-300);
  int k = 0;
  bool done = !(residual > absTol);
  grid.sync();
  for (; !done && k < A.maxIters; k++) {
    const double pAp = adj_hvp(grid, d, A, tid, nth);
    adj_put(d, 3, pAp, sm);
    grid.sync();
    const double pApT = adj_total(d, 3, bc);
    if (!(pApT > 0)) break;  // H not positive along p: stop with the current iterate
    const double alpha = rz / pApT;
    double rrn = 0;
    for (int i = tid; i < n3; i += nth) {
      A.mu[i] += alpha * A.p[i];
      const double ri = A.r[i] - alpha * A.Ap[i];
      A.r[i] = ri;
      rrn += ri * ri;
    }
    grid.sync();
    const double rzn = adj_precond(d, A, tid, nth);
    adj_put(d, 4, rrn, sm);
    adj_put(d, 5, rzn, sm);
    grid.sync();
    residual = sqrt(adj_total(d, 4, bc));
    const double rzNew = adj_total(d, 5, bc);
    if (!(residual > absTol)) { k++; done = true; break; }
    const double beta = rzNew / rz;
    rz = rzNew;
    for (int i = tid; i < n3; i += nth) A.p[i] = A.z[i] + beta * A.p[i];
    grid.sync();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    A.out[0] = k;
    A.out[1] = residual;
    A.out[2] = bNorm;
  }
}

// Per-element terms of mu . dg/dtheta for theta = (C00, C11, G, k): four rows
// of per-triangle / per-hinge values in `terms` (stride m + hg), summed later.
__global__ void __launch_bounds__(kThreads) k_adj_theta_terms(Dev d, const double* mu, double* terms, int stride) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < d.m) {
    const uint32_t ids[3] = {d.idx[e * 3], d.idx[e * 3 + 1], d.idx[e * 3 + 2]};
    double x0[3], x1[3], x2[3];
    load3(d.x, ids[0], x0); load3(d.x, ids[1], x1); load3(d.x, ids[2], x2);
    const float4 iv = d.inv[e];
    double mu9[9];
    for (int c = 0; c < 3; c++) {
      const bool pin = d.pinned[ids[c]];
      for (int k = 0; k < 3; k++) mu9[c * 3 + k] = pin ? 0.0 : mu[ids[c] * 3 + k];
    }
    const double th = d.mat.thickness;
    const Mat<double> unit[3] = {{1, 0, 0, 0, th}, {0, 1, 0, 0, th}, {0, 0, 0, 1, th}};
    for (int j = 0; j < 3; j++) {
      double en, g[9], E[3];
      tri_grad<double>(x0, x1, x2, iv.x, iv.y, iv.z, iv.w, d.area[e], unit[j], en, g, E);
      double s = 0;
      for (int k = 0; k < 9; k++) s += mu9[k] * g[k];
      terms[(size_t)j * stride + e] = s;
    }
    terms[(size_t)3 * stride + e] = 0;
  } else if (e < d.m + d.hg) {
    const int hh = e - d.m;
    const int4 hv = d.hinge[hh];
    const int ids[4] = {hv.x, hv.y, hv.z, hv.w};
    double q[12], g[12];
    for (int c = 0; c < 4; c++) load3(d.x, ids[c], q + c * 3);
    bend_grad<double>(q, d.hmeta[hh * 3], d.hmeta[hh * 3 + 1], d.hmeta[hh * 3 + 2], 1.0, g);
    double s = 0;
    for (int c = 0; c < 4; c++) {
      if (d.pinned[ids[c]]) continue;
      for (int k = 0; k < 3; k++) s += mu[ids[c] * 3 + k] * g[c * 3 + k];
    }
    for (int j = 0; j < 3; j++) terms[(size_t)j * stride + e] = 0;
    terms[(size_t)3 * stride + e] = s;
  }
}

// Fixed-order sums of the four rows (one block per row); acc[j] -= sum.
__global__ void __launch_bounds__(1024) k_adj_theta_sum(const double* terms, int stride, int count, double* acc) {
  __shared__ double sm[32];
  double s = 0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) s += terms[(size_t)blockIdx.x * stride + i];
  const double t = block_sum(s, sm);
  if (threadIdx.x == 0) acc[blockIdx.x] -= t;
}

// lambda_x0 = M mu / h^2 - (damp / h) lambda_v,  lambda_v0 = M mu / h (pins filtered);
// then the next step's total lambda_x1 = lambda_x0 + (damp / h) lambda_v0 is formed
// by the caller through adj_rhs.
__global__ void k_adj_propagate(Dev d, const double* mu, double* lamX, double* lamV, double damp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n * 3) return;
  const int v = i / 3;
  if (d.pinned[v]) { lamX[i] = 0; lamV[i] = 0; return; }
  const double M = d.mass[v];
  const double lv = lamV[i];
  lamX[i] = M * mu[i] * d.invH2 - damp * lv / d.h;
  lamV[i] = M * mu[i] / d.h;
}

// rhs = lambda_x1 + (damp / h) lambda_v1 (v1 = damp (x1 - x0) / h).
__global__ void k_adj_rhs(Dev d, const double* lamX, const double* lamV, double damp, double* rhs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n * 3) return;
  rhs[i] = d.pinned[i / 3] ? 0.0 : lamX[i] + damp * lamV[i] / d.h;
}

// Newton epilogue after the full-Hessian solve (newton.ts:152-179): descent
// safeguard (Jacobi-scaled steepest descent when g.dx >= 0) and the 2 mm trust
// region. One block; tree reductions. Writes the step's scalars.
__global__ void __launch_bounds__(1024) k_newton_epilogue(Dev d, const double* out3) {
  __shared__ double sm[32];
  const int n3 = d.n * 3;
  double gt = 0;
  for (int i = threadIdx.x; i < n3; i += blockDim.x) gt += d.g[i] * d.dx[i];
  double gtdx = block_sum(gt, sm);
  bool fallback = false;
  if (!isfinite(gtdx) || gtdx >= 0) {
    fallback = true;
    gt = 0;
    for (int i = threadIdx.x; i < n3; i += blockDim.x) {
      const double di = -d.g[i] / d.diag[i];
      d.dx[i] = di;
      gt += d.g[i] * di;
    }
    gtdx = block_sum(gt, sm);
  }
  double mx = 0;
  for (int i = threadIdx.x; i < n3; i += blockDim.x) mx = fmax(mx, fabs(d.dx[i]));
  const double maxDx = block_max(mx, sm);
  if (maxDx > 0.002) {
    const double sc = 0.002 / maxDx;
    for (int i = threadIdx.x; i < n3; i += blockDim.x) d.dx[i] *= sc;
    gtdx *= sc;
  }
  if (threadIdx.x == 0) {
    d.scal[S_PCG_ITERS] = out3[0];
    d.scal[S_PCG_RES] = out3[1];
    d.scal[S_GTDX] = gtdx;
    d.scal[S_FALLBACK] = fallback ? 1 : 0;
    d.scal[S_MAXDX] = maxDx;
  }
}

__global__ void k_neg_grad(Dev d, double* rhs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < d.n * 3) rhs[i] = -d.g[i];
}

int newton_exact_solve(const AdjArgs& a, int blocks, cudaStream_t s) {
  k_neg_grad<<<(a.d.n * 3 + kThreads - 1) / kThreads, kThreads, 0, s>>>(a.d, const_cast<double*>(a.rhs));
  const int rc = adj_launch_pcg(a, blocks, s);
  if (rc != 0) return rc;
  k_newton_epilogue<<<1, 1024, 0, s>>>(a.d, a.out);
  return (int)cudaGetLastError();
}

static inline int ablk(long n) { return (int)((n + kThreads - 1) / kThreads); }

int adj_grid_blocks(const Dev& d) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_adj_pcg, kThreads, 0);
  const int want = ablk(std::max(std::max(d.n * 3, d.m), std::max(d.hg, d.D)));
  int cap = per * sms;
  if (cap < 1) cap = 1;
  return std::max(1, std::min(want, std::min(cap, d.partStride)));
}

int adj_launch_pcg(const AdjArgs& a, int blocks, cudaStream_t s) {
  AdjArgs c = a;
  void* args[] = {&c};
  return (int)cudaLaunchCooperativeKernel((void*)k_adj_pcg, dim3(blocks), dim3(kThreads), args, 0, s);
}

void adj_theta(const Dev& d, const double* mu, double* terms, double* acc, cudaStream_t s) {
  const int stride = d.m + d.hg;
  k_adj_theta_terms<<<ablk(stride), kThreads, 0, s>>>(d, mu, terms, stride);
  k_adj_theta_sum<<<4, 1024, 0, s>>>(terms, stride, d.kb > 0 ? stride : d.m, acc);
}

void adj_propagate(const Dev& d, const double* mu, double* lamX, double* lamV, double damp, cudaStream_t s) {
  k_adj_propagate<<<ablk(d.n * 3), kThreads, 0, s>>>(d, mu, lamX, lamV, damp);
}

void adj_rhs(const Dev& d, const double* lamX, const double* lamV, double damp, double* rhs, cudaStream_t s) {
  k_adj_rhs<<<ablk(d.n * 3), kThreads, 0, s>>>(d, lamX, lamV, damp, rhs);
}

}  // namespace cs
