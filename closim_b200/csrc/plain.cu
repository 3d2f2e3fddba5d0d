// FP64 path of the implicit-Euler Newton step (compiled with -fmad=false).
//
// One thread per element over SoA mesh constants writes element-local results;
// one thread per vertex gathers them through the element-ordered CSR
// incidence, so each vertex sum adds the same terms in the same order as the
// reference's scatter (src/mesh/incidence.ts:1-7). The PCG solve runs as one
// cooperative persistent kernel: grid-wide barriers separate its phases and
// every reduction is a fixed-order two-level sum that all blocks evaluate
// identically, so control decisions agree across the grid and runs repeat
// bit for bit.
#include <cstdio>

#include "adjoint_math.cuh"
#include "contact.cuh"
#include "plain.cuh"

namespace cs {

static inline int nblk(int n) { return (n + kThreads - 1) / kThreads; }

__device__ __forceinline__ void load3(const double* x, int v, double o[3]) {
  o[0] = x[v * 3]; o[1] = x[v * 3 + 1]; o[2] = x[v * 3 + 2];
}

// s0 + t[0] + t[1] + ... evaluated left to right by one thread: the
// reference's `for (i...) s += t[i]` accumulation, rounding for rounding.
__device__ __forceinline__ double seq_chain(const double* t, int n, double s = 0.0) {
  int i = 0;
  for (; i + 4 <= n; i += 4) {
    const double a0 = t[i], a1 = t[i + 1], a2 = t[i + 2], a3 = t[i + 3];
    s = s + a0;
    s = s + a1;
    s = s + a2;
    s = s + a3;
  }
  for (; i < n; i++) s = s + t[i];
  return s;
}

// The same left-to-right chain, run by a whole block: warps 1.. stream the
// terms through a double-buffered shared-memory stage while thread 0 adds the
// previous stage in order. Every thread of the block must call it; the sum is
// valid in thread 0.
constexpr int kChunk = 2048;
__device__ __forceinline__ double block_chain(const double* t, int n, double* buf) {
  double s = 0.0;
  const int first = n < kChunk ? n : kChunk;
  for (int j = threadIdx.x; j < first; j += blockDim.x) buf[j] = t[j];
  __syncthreads();
  const int nchunks = (n + kChunk - 1) / kChunk;
  for (int c = 0; c < nchunks; c++) {
    const int base = c * kChunk;
    const int len = n - base < kChunk ? n - base : kChunk;
    const double* cur = buf + (c & 1) * kChunk;
    if (threadIdx.x >= 32) {
      const int nbase = base + kChunk;
      if (nbase < n) {
        double* nxt = buf + ((c + 1) & 1) * kChunk;
        const int nlen = n - nbase < kChunk ? n - nbase : kChunk;
        for (int j = threadIdx.x - 32; j < nlen; j += blockDim.x - 32) nxt[j] = t[nbase + j];
      }
    } else if (threadIdx.x == 0) {
      int j = 0;
      for (; j + 16 <= len; j += 16) {
        double a[16];
#pragma unroll
        for (int q = 0; q < 16; q++) a[q] = cur[j + q];
#pragma unroll
        for (int q = 0; q < 16; q++) s = s + a[q];
      }
      for (; j < len; j++) s = s + cur[j];
    }
    __syncthreads();
  }
  return s;
}

// ---- predictor (newton.ts:41-50) -------------------------------------------
// yHat = x0 + h v + h^2 g is the inertial target and, in the reference, the
// first Newton iterate. Exact-Newton mode starts from x0 + h v instead: for a
// sheet resting on a barrier, the gravity term pushes every contact vertex
// into the barrier and Newton spends its first iterations damping back out
// (on the floor drape, 10 iterations per step against 3 in free fall). The
// converged step does not depend on the first iterate.
__global__ void k_predict(Dev d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const double h = d.h;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const double x0 = d.x[i * 3 + k];
    d.x0[i * 3 + k] = x0;
    const double drift = x0 + h * d.v[i * 3 + k];
    const double y = drift + h * h * d.gravity[k];
    d.yHat[i * 3 + k] = y;
    d.x[i * 3 + k] = d.driftGuess ? drift : y;
  }
}

__global__ void k_pins(Dev d, double* x) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.npins) return;
  const int id = d.pinIds[k];
  x[id * 3] = d.pinPos[k * 3];
  x[id * 3 + 1] = d.pinPos[k * 3 + 1];
  x[id * 3 + 2] = d.pinPos[k * 3 + 2];
}

// ---- gradient (fem.ts:15-54, newton.ts:113-130) -------------------------------
__global__ void __launch_bounds__(kThreads) k_tri_grad(Dev d) {
  __shared__ double sm[32];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double strain = 0;
  if (t < d.m) {
    const uint32_t i0 = d.idx[t * 3], i1 = d.idx[t * 3 + 1], i2 = d.idx[t * 3 + 2];
    double p0[3], p1[3], p2[3];
    load3(d.x, i0, p0); load3(d.x, i1, p1); load3(d.x, i2, p2);
    const float4 iv = d.inv[t];
    double e, g[9], E[3];
    tri_grad<double>(p0, p1, p2, iv.x, iv.y, iv.z, iv.w, d.area[t], d.mat, e, g, E);
#pragma unroll
    for (int k = 0; k < 9; k++) d.elem[(size_t)t * 9 + k] = g[k];
    strain = js_max(js_max(fabs(E[0]), fabs(E[1])), fabs(E[2]));
  }
  const double bm = block_max(strain, sm);
  if (threadIdx.x == 0) d.part[0 * d.partStride + blockIdx.x] = bm;
}

__global__ void __launch_bounds__(kThreads) k_hinge_grad(Dev d) {
  const int hh = blockIdx.x * blockDim.x + threadIdx.x;
  if (hh >= d.hg) return;
  const int4 hv = d.hinge[hh];
  double q[12];
  load3(d.x, hv.x, q); load3(d.x, hv.y, q + 3); load3(d.x, hv.z, q + 6); load3(d.x, hv.w, q + 9);
  double out[12];
  hinge_fd_grad(q, d.hmeta[hh * 3], d.hmeta[hh * 3 + 1], d.hmeta[hh * 3 + 2], d.kb, out);
#pragma unroll
  for (int k = 0; k < 12; k++) d.helem[(size_t)hh * 12 + k] = out[k];
}

// Mixed path: the analytic gradient of the same hinge energy (bend_grad, the
// derivative of bending.ts:7-16) in place of the reference's central
// differences, which cost 24 energy evaluations per hinge.
__global__ void __launch_bounds__(kThreads) k_hinge_grad_analytic(Dev d) {
  const int hh = blockIdx.x * blockDim.x + threadIdx.x;
  if (hh >= d.hg) return;
  const int4 hv = d.hinge[hh];
  double q[12];
  load3(d.x, hv.x, q); load3(d.x, hv.y, q + 3); load3(d.x, hv.z, q + 6); load3(d.x, hv.w, q + 9);
  double out[12];
  bend_grad<double>(q, d.hmeta[hh * 3], d.hmeta[hh * 3 + 1], d.hmeta[hh * 3 + 2], d.kb, out);
#pragma unroll
  for (int k = 0; k < 12; k++) d.helem[(size_t)hh * 12 + k] = out[k];
}

// g = M (x - yHat) / h^2 + gradE (+ contact grad), pin filter, partial |g|^2.
__global__ void __launch_bounds__(kThreads) k_gather_grad(Dev d) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < d.n) {
    double s[3] = {0, 0, 0};
    for (uint32_t k = d.memOff[v]; k < d.memOff[v + 1]; k++) {
      const uint32_t rec = d.memRec[k];
      const double* e = d.elem + (size_t)(rec >> 2) * 9 + (rec & 3) * 3;
      s[0] += e[0]; s[1] += e[1]; s[2] += e[2];
    }
    if (d.kb > 0)
      for (uint32_t k = d.hinOff[v]; k < d.hinOff[v + 1]; k++) {
        const uint32_t rec = d.hinRec[k];
        const double* e = d.helem + (size_t)(rec >> 2) * 12 + (rec & 3) * 3;
        s[0] += e[0]; s[1] += e[1]; s[2] += e[2];
      }
    const double M = d.mass[v];
    const bool pin = d.pinned[v];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const int i = v * 3 + k;
      double gi = M * (d.x[i] - d.yHat[i]) * d.invH2 + s[k];
      if (d.hasContact) gi += d.cgrad[i];
      if (pin) gi = 0;
      d.g[i] = gi;
      d.T0[i] = gi * gi;
    }
  }
}

// Final reduction of the gradient pass: sqrt(sum g^2) in index order
// (newton.ts:128), max strain (order-free).
__global__ void __launch_bounds__(kThreads) k_grad_final(Dev d, int nbT) {
  __shared__ double cbuf[2 * kChunk];
  const double gs = block_chain(d.T0, d.n * 3, cbuf);
  if (threadIdx.x >= 32) return;
  const double ms = warp_max_partials(d.part + 0 * d.partStride, nbT);
  if (threadIdx.x == 0) {
    d.scal[S_GRADNORM] = sqrt(gs);
    d.scal[S_MAXSTRAIN] = ms;
  }
}

// ---- total energy (newton.ts:76-88; fem.ts:56-75) ------------------------------
// Per-element energy terms: inertia 0.5 m d^2 / h^2 per dof into T0, triangle
// energies then hinge energies into T1 (the order internalEnergyOnly adds them).
__global__ void __launch_bounds__(kThreads) k_energy(Dev d, const double* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < d.n) {
    const double m = d.mass[i];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double dd = x[i * 3 + k] - d.yHat[i * 3 + k];
      d.T0[i * 3 + k] = 0.5 * m * dd * dd / (d.h * d.h);
    }
  }
  if (i < d.m) {
    double p0[3], p1[3], p2[3];
    load3(x, d.idx[i * 3], p0); load3(x, d.idx[i * 3 + 1], p1); load3(x, d.idx[i * 3 + 2], p2);
    const float4 iv = d.inv[i];
    d.T1[i] = tri_energy<double>(p0, p1, p2, iv.x, iv.y, iv.z, iv.w, d.area[i], d.mat);
  }
  if (i < d.hg && d.kb > 0) {
    const int4 hv = d.hinge[i];
    double q[12];
    load3(x, hv.x, q); load3(x, hv.y, q + 3); load3(x, hv.z, q + 6); load3(x, hv.w, q + 9);
    d.T1[d.m + i] = hinge_energy4(q, d.hmeta[i * 3], d.hmeta[i * 3 + 1], d.hmeta[i * 3 + 2], d.kb);
  }
}

// totalEnergy (newton.ts:76-88): ((sum inertia) + internal) + merit, each sum a
// left-to-right chain; block 0 inertia, block 1 internal, block 2 merit.
__global__ void __launch_bounds__(kThreads) k_energy_chains(Dev d, int nMerit) {
  __shared__ double cbuf[2 * kChunk];
  double v = 0.0;
  if (blockIdx.x == 0) v = block_chain(d.T0, d.n * 3, cbuf);
  if (blockIdx.x == 1) v = block_chain(d.T1, d.m + (d.kb > 0 ? d.hg : 0), cbuf);
  if (blockIdx.x == 2) v = d.hasContact ? block_chain(d.Tc, nMerit, cbuf) : 0.0;
  if (threadIdx.x == 0) d.scal[S_E_INERTIA + blockIdx.x] = v;
}
__global__ void k_energy_final(Dev d) {
  double e = d.scal[S_E_INERTIA] + d.scal[S_E_TRI];
  if (d.hasContact) e += d.scal[S_E_MERIT];
  d.scal[S_ENERGY_TRIAL] = e;
}

__global__ void k_diag_init(Dev d, double beta) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n * 3) return;
  d.diag[i] = (double)d.mass[i / 3] * d.invH2 + beta;
}

// ---- one-level additive Schwarz (schwarz.ts:154-309) ---------------------------
// Factor: one warp per domain. Lane l owns the rows of member l and adds its
// incident triangles' 9x9 rows in ascending triangle order (the reference's
// per-entry accumulation order); the Cholesky is row-parallel with each entry
// computed by one lane in the reference's sequential inner order.
constexpr int kSchwarzWarps = 4;
__global__ void __launch_bounds__(kSchwarzWarps * 32) k_schwarz_factor(Dev d) {
  __shared__ double A[kSchwarzWarps][24 * 24];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int dom = blockIdx.x * kSchwarzWarps + wib;
  if (dom >= d.D) return;
  double* a = A[wib];
  const int start = d.domStart[dom], dv = d.domStart[dom + 1] - start, dw = dv * 3;
  for (int i = lane; i < 24 * 24; i += 32) a[i] = 0;
  __syncwarp();
  if (lane < dv) {
    const int v = d.domVerts[start + lane];
    for (int k = d.v2tOff[v]; k < d.v2tOff[v + 1]; k++) {
      const int t = d.v2t[k];
      const int cvs[3] = {(int)d.idx[t * 3], (int)d.idx[t * 3 + 1], (int)d.idx[t * 3 + 2]};
      const int ci = cvs[0] == v ? 0 : cvs[1] == v ? 1 : 2;
      double p0[3], p1[3], p2[3];
      load3(d.x, cvs[0], p0); load3(d.x, cvs[1], p1); load3(d.x, cvs[2], p2);
      const float4 iv = d.inv[t];
      double h27[27];
      tri_hessian9_rows<double>(p0, p1, p2, iv.x, iv.y, iv.z, iv.w, d.area[t], d.mat, ci * 3, ci * 3 + 3, h27);
      for (int cj = 0; cj < 3; cj++) {
        int lw = -1;
        for (int q = 0; q < dv; q++)
          if (d.domVerts[start + q] == cvs[cj]) { lw = q; break; }
        if (lw < 0) continue;
        for (int aa = 0; aa < 3; aa++)
          for (int bb = 0; bb < 3; bb++) a[(lane * 3 + aa) * dw + (lw * 3 + bb)] += h27[aa * 9 + cj * 3 + bb];
      }
    }
  }
  __syncwarp();
  if (lane < dw) {
    const int v = d.domVerts[start + lane / 3];
    a[lane * dw + lane] += d.diag[v * 3 + lane % 3];
  }
  __syncwarp();
  for (int i = lane; i < dw; i += 32)
    for (int j = i + 1; j < dw; j++) {
      const double s = 0.5 * (a[i * dw + j] + a[j * dw + i]);
      a[i * dw + j] = s;
      a[j * dw + i] = s;
    }
  __syncwarp();
  double scale = 0;
  for (int i = 0; i < dw; i++) scale = js_max(scale, fabs(a[i * dw + i]));
  const double tiny = 1e-20 * (1 + scale);
  bool ok = true;
  for (int k = 0; k < dw; k++) {
    double diagk = 0;
    if (lane == 0) {
      double sum = a[k * dw + k];
      for (int s = 0; s < k; s++) sum -= a[k * dw + s] * a[k * dw + s];
      ok = sum > tiny;
      if (ok) a[k * dw + k] = sqrt(sum);
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    __syncwarp();
    if (!ok) break;
    diagk = a[k * dw + k];
    if (lane > k && lane < dw) {
      double s2 = a[lane * dw + k];
      for (int s = 0; s < k; s++) s2 -= a[lane * dw + s] * a[k * dw + s];
      a[lane * dw + k] = s2 / diagk;
    }
    __syncwarp();
  }
  double* L = d.L + (size_t)dom * 576;
  if (ok) {
    for (int i = lane; i < dw; i += 32)
      for (int j = 0; j < 24; j++) L[i * 24 + j] = j <= i && j < dw ? a[i * dw + j] : 0.0;
  } else {
    for (int i = lane; i < dw; i += 32) {
      const int v = d.domVerts[start + i / 3];
      const double dd = d.diag[v * 3 + i % 3];
      for (int j = 0; j < 24; j++) L[i * 24 + j] = j == i ? (dd > 1e-12 ? 1 / dd : 0.0) : 0.0;
    }
  }
  if (lane == 0) d.domFlag[dom] = ok ? 1 : 0;
}

// Two-level Schwarz (src/solver/mas.ts buildCoarseDiag, mas.ts:57-101): the
// coarse diagonal of each domain, one thread per domain, in the reference's
// accumulation order: the domain's triangles in ascending order, their
// within-domain (ci, cj) pairs, then the Jacobi diagonal over the members.
constexpr int kCoarseTris = 96;  // triangles touching a domain of <= 8 vertices
__global__ void __launch_bounds__(kThreads) k_coarse_diag(Dev d) {
  const int dom = blockIdx.x * blockDim.x + threadIdx.x;
  if (dom >= d.D) return;
  const int start = d.domStart[dom], dv = d.domStart[dom + 1] - start;
  int tris[kCoarseTris];
  int nt = 0;
  for (int l = 0; l < dv; l++) {
    const int v = d.domVerts[start + l];
    for (int k = d.v2tOff[v]; k < d.v2tOff[v + 1]; k++) {
      const int t = d.v2t[k];
      int pos = nt;  // insertion into the sorted list, duplicates skipped
      bool dup = false;
      for (int q = 0; q < nt; q++) {
        if (tris[q] == t) { dup = true; break; }
        if (tris[q] > t) { pos = q; break; }
      }
      if (dup || nt >= kCoarseTris) continue;
      for (int q = nt; q > pos; q--) tris[q] = tris[q - 1];
      tris[pos] = t;
      nt++;
    }
  }
  auto inDom = [&](int v) {
    for (int l = 0; l < dv; l++)
      if (d.domVerts[start + l] == v) return true;
    return false;
  };
  double dc[3] = {0, 0, 0};
  for (int q = 0; q < nt; q++) {
    const int t = tris[q];
    const int cvs[3] = {(int)d.idx[t * 3], (int)d.idx[t * 3 + 1], (int)d.idx[t * 3 + 2]};
    const bool in[3] = {inDom(cvs[0]), inDom(cvs[1]), inDom(cvs[2])};
    double p0[3], p1[3], p2[3];
    load3(d.x, cvs[0], p0); load3(d.x, cvs[1], p1); load3(d.x, cvs[2], p2);
    const float4 iv = d.inv[t];
    for (int ci = 0; ci < 3; ci++) {
      if (!in[ci]) continue;
      double h27[27];  // rows ci*3 .. ci*3+2 of the 9x9 block
      tri_hessian9_rows<double>(p0, p1, p2, iv.x, iv.y, iv.z, iv.w, d.area[t], d.mat, ci * 3, ci * 3 + 3, h27);
      for (int cj = 0; cj < 3; cj++) {
        if (!in[cj]) continue;
        const double s = 1.0 / (double)dv;
        for (int a = 0; a < 3; a++) dc[a] += s * h27[a * 9 + cj * 3 + a];
      }
    }
  }
  for (int l = 0; l < dv; l++) {
    const int v = d.domVerts[start + l];
    const double s = 1.0 / (double)dv;
    for (int a = 0; a < 3; a++) dc[a] += s * d.diag[v * 3 + a];
  }
  for (int a = 0; a < 3; a++) d.dcoarse[dom * 3 + a] = dc[a];
}

// z = M^-1 r on one domain; returns sum r.z over its (pin-filtered) dofs.
__device__ double schwarz_apply_domain(const Dev& d, int dom) {
  const int start = d.domStart[dom], dv = d.domStart[dom + 1] - start, dw = dv * 3;
  const double* L = d.L + (size_t)dom * 576;
  double rhs[24], y[24], sol[24];
  for (int l = 0; l < dv; l++) {
    const int v = d.domVerts[start + l];
    rhs[l * 3] = d.r[v * 3]; rhs[l * 3 + 1] = d.r[v * 3 + 1]; rhs[l * 3 + 2] = d.r[v * 3 + 2];
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
  // two-level: + P (omega Dc^-1) R r on this domain (applyMasTwoLevel,
  // mas.ts:110-145, omega = 0.5; the coarse vector of a domain is constant per
  // component over its members, scaled by 1/sqrt(|d|) both ways)
  double cz[3] = {0, 0, 0};
  const double sc = 1 / sqrt((double)dv);
  if (d.precond == 2) {
    double rc[3] = {0, 0, 0};
    for (int l = 0; l < dv; l++)
      for (int k = 0; k < 3; k++) rc[k] += rhs[l * 3 + k] * sc;
    for (int k = 0; k < 3; k++) {
      const double dd = d.dcoarse[dom * 3 + k];
      cz[k] = dd > 1e-12 ? (0.5 * rc[k]) / dd : 0.0;
    }
  }
  for (int l = 0; l < dv; l++) {
    const int v = d.domVerts[start + l];
    const bool pin = d.pinned[v];
    for (int k = 0; k < 3; k++) {
      double zz = 0.0 + sol[l * 3 + k];
      if (d.precond == 2) zz += cz[k] * sc;
      if (pin) zz = 0.0;
      d.z[v * 3 + k] = zz;
      d.T2[v * 3 + k] = d.r[v * 3 + k] * zz;
    }
  }
  return 0.0;
}

// ---- PCG as one cooperative kernel (pcg.ts:11-95 + newton.ts:148-179) ----------
struct PcgArgs {
  Dev d;
  int maxIters;
  double tol;
};

// Block partial -> row slot; after grid.sync every block reads the same total.
__device__ __forceinline__ void put_partial(const Dev& d, int row, double v, double* sm) {
  const double b = block_sum(v, sm);
  if (threadIdx.x == 0) d.part[row * d.partStride + blockIdx.x] = b;
}
__device__ __forceinline__ double get_total(const Dev& d, int row, double* bc) {
  if (threadIdx.x < 32) {
    const double s = warp_sum_partials(d.part + row * d.partStride, gridDim.x);
    if (threadIdx.x == 0) bc[0] = s;
  }
  __syncthreads();
  const double r = bc[0];
  __syncthreads();
  return r;
}
__device__ __forceinline__ double get_max_nonan(const Dev& d, int row, double* bc) {
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    double s = 0;
    for (int i = lane; i < (int)gridDim.x; i += 32) {
      const double v = d.part[row * d.partStride + i];
      if (v > s) s = v;
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double w = __shfl_xor_sync(0xffffffffu, s, o);
      if (w > s) s = w;
    }
    if (lane == 0) bc[0] = s;
  }
  __syncthreads();
  const double r = bc[0];
  __syncthreads();
  return r;
}
__device__ __forceinline__ double block_max_nonan(double v, double* sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_down_sync(0xffffffffu, v, o);
    if (w > v) v = w;
  }
  __syncthreads();
  if (lane == 0) sm[warp] = v;
  __syncthreads();
  double r = 0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < (int)(blockDim.x >> 5); i++)
      if (sm[i] > r) r = sm[i];
    sm[0] = r;
  }
  __syncthreads();
  r = sm[0];
  __syncthreads();
  return r;
}

// Chained sums after a grid barrier: chain w (w < nch) runs on block w as a
// block_chain; results land in scal[S_CH0 + w]. With fewer blocks than chains,
// block 0 runs them one after another.
__device__ __forceinline__ void run_chains(const Dev& d, int nch, const double* a0, const double* a1,
                                           const double* a2, int n, double* cbuf) {
  const double* arr[3] = {a0, a1, a2};
  if ((int)gridDim.x >= nch) {
    if ((int)blockIdx.x < nch) {
      const double v = block_chain(arr[blockIdx.x], n, cbuf);
      if (threadIdx.x == 0) d.scal[S_CH0 + blockIdx.x] = v;
    }
  } else if (blockIdx.x == 0) {
    for (int w = 0; w < nch; w++) {
      const double v = block_chain(arr[w], n, cbuf);
      if (threadIdx.x == 0) d.scal[S_CH0 + w] = v;
    }
  }
}
// One chain into scal[slot], on block 0.
__device__ __forceinline__ void run_chain1(const Dev& d, const double* a, int n, int slot, double* cbuf) {
  if (blockIdx.x == 0) {
    const double v = block_chain(a, n, cbuf);
    if (threadIdx.x == 0) d.scal[slot] = v;
  }
}

__global__ void __launch_bounds__(kThreads) k_pcg(PcgArgs A) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double sm[32];
  __shared__ double bc[2];
  __shared__ double cbuf[2 * kChunk];
  const Dev& d = A.d;
  const int n3 = d.n * 3;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const bool jacobi = d.precond == 0;
  // ---- init: r = filter(b), z = M^-1 r, p = z (pcg.ts:27-55) ----
  for (int i = tid; i < n3; i += nth) {
    const double bi = -d.g[i];
    d.T0[i] = bi * bi;
    const double ri = d.pinned[i / 3] ? 0.0 : bi;
    d.r[i] = ri;
    d.dx[i] = 0;
    d.T1[i] = ri * ri;
    if (jacobi) {
      double zi = d.diag[i] > 1e-12 ? ri / d.diag[i] : ri;
      if (d.pinned[i / 3]) zi = 0;
      d.z[i] = zi;
      d.p[i] = zi;
      d.T2[i] = ri * zi;
    }
  }
  grid.sync();
  if (!jacobi) {
    for (int dom = tid; dom < d.D; dom += nth) schwarz_apply_domain(d, dom);
    grid.sync();
    for (int i = tid; i < n3; i += nth) d.p[i] = d.z[i];
  }
  // chains: rz (T2), |b|^2 (T0), |r|^2 (T1)
  run_chains(d, 3, d.T2, d.T0, d.T1, n3, cbuf);
  grid.sync();
  double rz = d.scal[S_CH0];
  const double bNorm = sqrt(d.scal[S_CH1]);
  const double absTol = js_max(A.tol * js_max(bNorm, 1e-12), 1e-12);
  double residual = sqrt(d.scal[S_CH2]);
  int iters = 0;
  bool done = residual < absTol;
  if (!done) {
    for (int i = tid; i < n3; i += nth) d.T3[i] = d.p[i] * d.p[i];
    grid.sync();
    run_chain1(d, d.T3, n3, S_CH3, cbuf);
    grid.sync();
  }
  int k = 0;
  for (; !done && k < A.maxIters; k++) {
    // ---- Ap = M/h^2 p + membraneHvp (fem.ts:108-130) + contact HVP ----
    const double pNorm = sqrt(d.scal[S_CH3]);
    const double h = 1e-8 * (1 + pNorm);
    for (int t = tid; t < d.m; t += nth) {
      const uint32_t vi[3] = {d.idx[t * 3], d.idx[t * 3 + 1], d.idx[t * 3 + 2]};
      double xp[9], xm[9];
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int q = 0; q < 3; q++) {
          const double xx = d.x[vi[c] * 3 + q], pq = d.p[vi[c] * 3 + q];
          xp[c * 3 + q] = xx + h * pq;
          xm[c * 3 + q] = xx - h * pq;
        }
      const float4 iv = d.inv[t];
      const double ar = d.area[t];
      double e, gp[9], gm[9], E[3];
      tri_grad<double>(xp, xp + 3, xp + 6, iv.x, iv.y, iv.z, iv.w, ar, d.mat, e, gp, E);
      tri_grad<double>(xm, xm + 3, xm + 6, iv.x, iv.y, iv.z, iv.w, ar, d.mat, e, gm, E);
      double* o = d.elem + (size_t)t * 18;
#pragma unroll
      for (int q = 0; q < 9; q++) { o[q] = gp[q]; o[9 + q] = gm[q]; }
    }
    if (d.hasContact) contact_hvp_coeffs(d, d.p, tid, nth);
    grid.sync();
    for (int v = tid; v < d.n; v += nth) {
      double sp[3] = {0, 0, 0}, sn[3] = {0, 0, 0};
      for (uint32_t q = d.memOff[v]; q < d.memOff[v + 1]; q++) {
        const uint32_t rec = d.memRec[q];
        const double* e = d.elem + (size_t)(rec >> 2) * 18 + (rec & 3) * 3;
        sp[0] += e[0]; sp[1] += e[1]; sp[2] += e[2];
        sn[0] += e[9]; sn[1] += e[10]; sn[2] += e[11];
      }
      double ch[3] = {0, 0, 0};
      if (d.hasContact) contact_hvp_gather(d, v, ch);
      const double M = d.mass[v];
      const bool pin = d.pinned[v];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const int i = v * 3 + c;
        const double Hp = (sp[c] - sn[c]) / (2 * h);
        double ap = M * d.p[i] * d.invH2 + Hp;
        if (d.hasContact) ap += ch[c];
        if (pin) ap = 0;
        d.Ap[i] = ap;
        d.T0[i] = d.p[i] * ap;
      }
    }
    grid.sync();
    run_chain1(d, d.T0, n3, S_CH1, cbuf);
    grid.sync();
    const double pAp = d.scal[S_CH1];
    if (!(pAp > 1e-30)) { iters = k; done = true; break; }
    const double alpha = rz / pAp;
    for (int i = tid; i < n3; i += nth) {
      const bool pin = d.pinned[i / 3];
      double xi = d.dx[i] + alpha * d.p[i];
      double ri = d.r[i] - alpha * d.Ap[i];
      if (pin) { xi = 0; ri = 0; }
      d.dx[i] = xi;
      d.r[i] = ri;
      d.T1[i] = ri * ri;
      if (jacobi) {
        double zi = d.diag[i] > 1e-12 ? ri / d.diag[i] : ri;
        if (pin) zi = 0;
        d.z[i] = zi;
        d.T2[i] = ri * zi;
      }
    }
    grid.sync();
    run_chains(d, jacobi ? 2 : 1, d.T1, d.T2, d.T2, n3, cbuf);  // |r|^2 -> CH0, r.z -> CH1
    grid.sync();
    residual = sqrt(d.scal[S_CH0]);
    if (residual < absTol) { iters = k + 1; done = true; break; }
    if (!jacobi) {
      for (int dom = tid; dom < d.D; dom += nth) schwarz_apply_domain(d, dom);
      grid.sync();
      run_chain1(d, d.T2, n3, S_CH1, cbuf);
      grid.sync();
    }
    const double rzNew = d.scal[S_CH1];
    const double beta = rzNew / rz;
    for (int i = tid; i < n3; i += nth) {
      const double pi = d.z[i] + beta * d.p[i];
      d.p[i] = pi;
      d.T3[i] = pi * pi;
    }
    rz = rzNew;
    grid.sync();
    run_chain1(d, d.T3, n3, S_CH3, cbuf);
    grid.sync();
  }
  if (!done) iters = A.maxIters;
  // ---- descent safeguard + trust region (newton.ts:152-179) ----
  grid.sync();
  for (int i = tid; i < n3; i += nth) d.T0[i] = d.g[i] * d.dx[i];
  grid.sync();
  run_chain1(d, d.T0, n3, S_CH2, cbuf);
  grid.sync();
  double gtdx = d.scal[S_CH2];
  bool fallback = false;
  if (!isfinite(gtdx) || gtdx >= 0) {
    fallback = true;
    for (int i = tid; i < n3; i += nth) {
      const double di = -d.g[i] / d.diag[i];
      d.dx[i] = di;
      d.T1[i] = d.g[i] * di;
    }
    grid.sync();
    run_chain1(d, d.T1, n3, S_CH3, cbuf);
    grid.sync();
    gtdx = d.scal[S_CH3];
  }
  double mx = 0;
  for (int i = tid; i < n3; i += nth) {
    const double a = fabs(d.dx[i]);
    if (a > mx) mx = a;
  }
  const double bmx = block_max_nonan(mx, sm);
  if (threadIdx.x == 0) d.part[6 * d.partStride + blockIdx.x] = bmx;
  grid.sync();
  const double maxDx = get_max_nonan(d, 6, bc);
  const double TRUST = 0.002;
  if (maxDx > TRUST) {
    const double s = TRUST / maxDx;
    for (int i = tid; i < n3; i += nth) d.dx[i] *= s;
    gtdx *= s;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    d.scal[S_PCG_ITERS] = iters;
    d.scal[S_PCG_RES] = residual;
    d.scal[S_GTDX] = gtdx;
    d.scal[S_FALLBACK] = fallback ? 1 : 0;
    d.scal[S_MAXDX] = maxDx;
  }
}

// ---- standalone FD membrane HVP (fem.ts:108-130) -----------------------------------
// out = (gradM(x + h p) - gradM(x - h p)) / (2h), h = 1e-8 (1 + |p|): the same
// element and gather arithmetic as the PCG kernel's HVP phase, as plain kernels.
__global__ void k_hvp_terms(const double* p, int n3, double* T) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) T[i] = p[i] * p[i];
}
__global__ void __launch_bounds__(kThreads) k_hvp_h(const double* T, int n3, double* h) {
  __shared__ double cbuf[2 * kChunk];
  const double pp = block_chain(T, n3, cbuf);
  if (threadIdx.x == 0) *h = 1e-8 * (1 + sqrt(pp));
}
__device__ __forceinline__ void hvp_elem_tri(int t, const uint32_t* idx, const float4* inv, const float* area,
                                             const Mat<double>& mat, const double* x, const double* p, double h,
                                             double* elem) {
  const uint32_t vi[3] = {idx[t * 3], idx[t * 3 + 1], idx[t * 3 + 2]};
  double xp[9], xm[9];
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const double xx = x[vi[c] * 3 + q], pq = p[vi[c] * 3 + q];
      xp[c * 3 + q] = xx + h * pq;
      xm[c * 3 + q] = xx - h * pq;
    }
  const float4 iv = inv[t];
  double e, gp[9], gm[9], E[3];
  tri_grad<double>(xp, xp + 3, xp + 6, iv.x, iv.y, iv.z, iv.w, area[t], mat, e, gp, E);
  tri_grad<double>(xm, xm + 3, xm + 6, iv.x, iv.y, iv.z, iv.w, area[t], mat, e, gm, E);
  double* o = elem + (size_t)t * 18;
#pragma unroll
  for (int q = 0; q < 9; q++) { o[q] = gp[q]; o[9 + q] = gm[q]; }
}
__global__ void __launch_bounds__(kThreads) k_hvp_elem(const uint32_t* idx, const float4* inv, const float* area,
                                                       Mat<double> mat, int m, const double* x, const double* p,
                                                       const double* h, double* elem) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < m) hvp_elem_tri(t, idx, inv, area, mat, x, p, *h, elem);
}
__global__ void __launch_bounds__(kThreads) k_hvp_gather(const uint32_t* memOff, const uint32_t* memRec, int n,
                                                         const double* elem, const double* h, double* out) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  double sp[3] = {0, 0, 0}, sn[3] = {0, 0, 0};
  for (uint32_t q = memOff[v]; q < memOff[v + 1]; q++) {
    const uint32_t rec = memRec[q];
    const double* e = elem + (size_t)(rec >> 2) * 18 + (rec & 3) * 3;
    sp[0] += e[0]; sp[1] += e[1]; sp[2] += e[2];
    sn[0] += e[9]; sn[1] += e[10]; sn[2] += e[11];
  }
  const double hh = *h;
#pragma unroll
  for (int c = 0; c < 3; c++) out[v * 3 + c] = (sp[c] - sn[c]) / (2 * hh);
}

void launch_membrane_hvp(const uint32_t* idx, const float4* inv, const float* area, const Mat<double>& mat, int n,
                         int m, const uint32_t* memOff, const uint32_t* memRec, const double* x, const double* p,
                         double* out, double* T, double* h, double* elem, cudaStream_t s) {
  k_hvp_terms<<<nblk(n * 3), kThreads, 0, s>>>(p, n * 3, T);
  k_hvp_h<<<1, kThreads, 0, s>>>(T, n * 3, h);
  k_hvp_elem<<<nblk(m), kThreads, 0, s>>>(idx, inv, area, mat, m, x, p, h, elem);
  k_hvp_gather<<<nblk(n), kThreads, 0, s>>>(memOff, memRec, n, elem, h, out);
}

// ---- material-model evaluation (material-model.ts:278-288) -------------------------
// internalEnergyOnly (fem.ts:56-75) terms: triangle energies, then hinge
// energies when kb > 0, into T1 in the order the reference adds them.
__global__ void __launch_bounds__(kThreads) k_internal_energy_terms(Dev d, const double* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < d.m) {
    double p0[3], p1[3], p2[3];
    load3(x, d.idx[i * 3], p0); load3(x, d.idx[i * 3 + 1], p1); load3(x, d.idx[i * 3 + 2], p2);
    const float4 iv = d.inv[i];
    d.T1[i] = tri_energy<double>(p0, p1, p2, iv.x, iv.y, iv.z, iv.w, d.area[i], d.mat);
  }
  if (i < d.hg && d.kb > 0) {
    const int4 hv = d.hinge[i];
    double q[12];
    load3(x, hv.x, q); load3(x, hv.y, q + 3); load3(x, hv.z, q + 6); load3(x, hv.w, q + 9);
    d.T1[d.m + i] = hinge_energy4(q, d.hmeta[i * 3], d.hmeta[i * 3 + 1], d.hmeta[i * 3 + 2], d.kb);
  }
}
// evalInternal's gradient (fem.ts:15-54): per vertex, its triangle terms in
// ascending triangle order, then its hinge terms in hinge order (the
// reference's scatter order); no inertia, pins or contact.
__global__ void __launch_bounds__(kThreads) k_gather_internal(Dev d, double* grad) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= d.n) return;
  double s[3] = {0, 0, 0};
  for (uint32_t k = d.memOff[v]; k < d.memOff[v + 1]; k++) {
    const uint32_t rec = d.memRec[k];
    const double* e = d.elem + (size_t)(rec >> 2) * 9 + (rec & 3) * 3;
    s[0] += e[0]; s[1] += e[1]; s[2] += e[2];
  }
  if (d.kb > 0)
    for (uint32_t k = d.hinOff[v]; k < d.hinOff[v + 1]; k++) {
      const uint32_t rec = d.hinRec[k];
      const double* e = d.helem + (size_t)(rec >> 2) * 12 + (rec & 3) * 3;
      s[0] += e[0]; s[1] += e[1]; s[2] += e[2];
    }
  grad[v * 3] = s[0];
  grad[v * 3 + 1] = s[1];
  grad[v * 3 + 2] = s[2];
}
// out[0] = the internal energy chain, out[1] = max strain over the triangle
// partials (nbT of them; 0 when none were computed).
__global__ void __launch_bounds__(kThreads) k_internal_final(Dev d, int nbT, double* out) {
  __shared__ double cbuf[2 * kChunk];
  const double e = block_chain(d.T1, d.m + (d.kb > 0 ? d.hg : 0), cbuf);
  if (threadIdx.x >= 32) return;
  const double ms = nbT > 0 ? warp_max_partials(d.part + 0 * d.partStride, nbT) : 0.0;
  if (threadIdx.x == 0) {
    out[0] = e;
    out[1] = ms;
  }
}
// evalMembraneHvp (membrane-hvp.ts:80-108): the analytic per-triangle HVP
// (triangleHvp, membrane-hvp.ts:18-75) and the same vertex gather order.
__global__ void __launch_bounds__(kThreads) k_tri_hvp_elem(Dev d, const double* x, const double* p) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.m) return;
  const uint32_t i0 = d.idx[t * 3], i1 = d.idx[t * 3 + 1], i2 = d.idx[t * 3 + 2];
  double p0[3], p1[3], p2[3], v0[3], v1[3], v2[3];
  load3(x, i0, p0); load3(x, i1, p1); load3(x, i2, p2);
  load3(p, i0, v0); load3(p, i1, v1); load3(p, i2, v2);
  const float4 iv = d.inv[t];
  double o[9];
  tri_hvp<double>(p0, p1, p2, v0, v1, v2, iv.x, iv.y, iv.z, iv.w, d.area[t], d.mat, o);
#pragma unroll
  for (int k = 0; k < 9; k++) d.elem[(size_t)t * 9 + k] = o[k];
}
__global__ void __launch_bounds__(kThreads) k_gather_elem9(Dev d, double* out) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= d.n) return;
  double s[3] = {0, 0, 0};
  for (uint32_t k = d.memOff[v]; k < d.memOff[v + 1]; k++) {
    const uint32_t rec = d.memRec[k];
    const double* e = d.elem + (size_t)(rec >> 2) * 9 + (rec & 3) * 3;
    s[0] += e[0]; s[1] += e[1]; s[2] += e[2];
  }
  out[v * 3] = s[0];
  out[v * 3 + 1] = s[1];
  out[v * 3 + 2] = s[2];
}

void launch_internal_eval(const Dev& d0, const double* x, double* grad, double* out2, cudaStream_t s) {
  Dev d = d0;
  d.x = const_cast<double*>(x);
  int nbT = 0;
  if (grad) {
    k_tri_grad<<<nblk(d.m), kThreads, 0, s>>>(d);
    nbT = nblk(d.m);
    if (d.kb > 0 && d.hg > 0) k_hinge_grad<<<nblk(d.hg), kThreads, 0, s>>>(d);
    k_gather_internal<<<nblk(d.n), kThreads, 0, s>>>(d, grad);
  }
  k_internal_energy_terms<<<nblk(std::max(d.m, d.hg)), kThreads, 0, s>>>(d, x);
  k_internal_final<<<1, kThreads, 0, s>>>(d, nbT, out2);
}

void launch_membrane_hvp_analytic(const Dev& d, const double* x, const double* p, double* out, cudaStream_t s) {
  k_tri_hvp_elem<<<nblk(d.m), kThreads, 0, s>>>(d, x, p);
  k_gather_elem9<<<nblk(d.n), kThreads, 0, s>>>(d, out);
}

// ---- Armijo trial + velocity ----------------------------------------------------
__global__ void k_trial(Dev d, double alpha) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n * 3) return;
  d.xt[i] = d.x[i] + alpha * d.dx[i];
}

__global__ void k_velocity(Dev d, double damp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n * 3) return;
  d.v[i] = ((d.x[i] - d.x0[i]) / d.h) * damp;
}

// ---- simulation-session hand-off -------------------------------------------------
// flag = 1 when any coordinate of x is non-finite.
__global__ void k_nonfinite(const double* x, int n3, int* flag) {
  int bad = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x)
    if (!isfinite(x[i])) bad = 1;
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}
// stable <- x when the flag is clear (the last NaN-free state stays on the device).
__global__ void k_keep_if_finite(const double* x, double* stable, int n3, const int* flag) {
  if (*flag) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) stable[i] = x[i];
}

void launch_session_check(const double* x, double* stable, int n3, int* flag, cudaStream_t s) {
  cudaMemsetAsync(flag, 0, sizeof(int), s);
  const int blocks = std::min(1184, std::max(1, (n3 + kThreads - 1) / kThreads));
  k_nonfinite<<<blocks, kThreads, 0, s>>>(x, n3, flag);
  k_keep_if_finite<<<blocks, kThreads, 0, s>>>(x, stable, n3, flag);
}

// ---- launchers ------------------------------------------------------------------

void launch_predict(const Dev& d, cudaStream_t s) {
  k_predict<<<nblk(d.n), kThreads, 0, s>>>(d);
  launch_pins(d, d.x, s);
}
void launch_pins(const Dev& d, double* x, cudaStream_t s) {
  if (d.npins > 0) k_pins<<<nblk(d.npins), kThreads, 0, s>>>(d, x);
}
void launch_grad_terms(const Dev& d, cudaStream_t s, bool analyticBend) {
  k_tri_grad<<<nblk(d.m), kThreads, 0, s>>>(d);
  if (d.kb > 0 && d.hg > 0) {
    if (analyticBend) k_hinge_grad_analytic<<<nblk(d.hg), kThreads, 0, s>>>(d);
    else k_hinge_grad<<<nblk(d.hg), kThreads, 0, s>>>(d);
  }
  k_gather_grad<<<nblk(d.n), kThreads, 0, s>>>(d);
}
void launch_grad(const Dev& d, cudaStream_t s, bool analyticBend) {
  launch_grad_terms(d, s, analyticBend);
  k_grad_final<<<1, kThreads, 0, s>>>(d, nblk(d.m));
}
void launch_energy_terms(const Dev& d, const double* x, cudaStream_t s) {
  const int nb = nblk(std::max(std::max(d.n, d.m), d.hg));
  k_energy<<<nb, kThreads, 0, s>>>(d, x);
}
void launch_energy(const Dev& d, const double* x, cudaStream_t s) {
  launch_energy_terms(d, x, s);
  k_energy_chains<<<3, kThreads, 0, s>>>(d, d.hasContact ? d.c.nActive : 0);
  k_energy_final<<<1, 1, 0, s>>>(d);
}
void launch_diag_init(const Dev& d, double beta, cudaStream_t s) {
  k_diag_init<<<nblk(d.n * 3), kThreads, 0, s>>>(d, beta);
}
void launch_schwarz_factor(const Dev& d, cudaStream_t s) {
  k_schwarz_factor<<<(d.D + kSchwarzWarps - 1) / kSchwarzWarps, kSchwarzWarps * 32, 0, s>>>(d);
  if (d.precond == 2) k_coarse_diag<<<nblk(d.D), kThreads, 0, s>>>(d);
}
int pcg_grid_blocks(const Dev& d) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg, kThreads, 0);
  const int want = nblk(std::max(d.n * 3, d.m));
  int cap = per * sms;
  if (cap < 1) cap = 1;
  return std::max(1, std::min(want, std::min(cap, d.partStride)));
}
int launch_pcg(const Dev& d, int maxIters, double tol, int gridBlocks, cudaStream_t s) {
  PcgArgs a{d, maxIters, tol};
  void* args[] = {&a};
  return (int)cudaLaunchCooperativeKernel((void*)k_pcg, dim3(gridBlocks), dim3(kThreads), args, 0, s);
}
void launch_trial(const Dev& d, double alpha, cudaStream_t s) {
  k_trial<<<nblk(d.n * 3), kThreads, 0, s>>>(d, alpha);
  launch_pins(d, d.xt, s);
}
void launch_velocity(const Dev& d, double damp, cudaStream_t s) {
  k_velocity<<<nblk(d.n * 3), kThreads, 0, s>>>(d, damp);
}

}  // namespace cs
