// Mixed-precision path of the Newton step (FP32 linear solve, FP64 where it
// matters). Compiled with FMA contraction on.
//
// Per Newton iteration the membrane state of every triangle is evaluated once
// in FP64 (deformation gradient F, 2nd Piola stress S) and stored as FP32, so
// the PCG's matrix-free HVP is the exact directional derivative of the
// gradient (src/physics/membrane-hvp.ts:18-75) at ~60 FP32 flops and 64 bytes
// per triangle. PCG vectors are FP32; every dot product and norm accumulates
// in FP64 through a fixed-order two-level tree (deterministic). The one-level
// Schwarz preconditioner (src/solver/schwarz.ts) is assembled and factored in
// FP64 and applied as an FP32 dense inverse per domain, one warp per domain.
// Gradient, energies, contact and CCD stay on the FP64 kernels.
#include "adjoint_math.cuh"
#include "contact.cuh"
#include "mixed.cuh"

namespace cs {

static inline int mblk(long n) { return (int)((n + kThreads - 1) / kThreads); }

__device__ __forceinline__ void ld3(const double* x, int v, double o[3]) {
  o[0] = x[v * 3]; o[1] = x[v * 3 + 1]; o[2] = x[v * 3 + 2];
}

// ---- per-triangle membrane state (F, S) and the 9x9 block -------------------------
// tris: 16 floats per triangle: F00 F10 F20 F01 F11 F21, S00 S11 S01, a b c d, s, pad x2
__global__ void __launch_bounds__(kThreads) k_mx_tristate(Dev d, MixBufs mb) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.m) return;
  double x0[3], x1[3], x2[3];
  ld3(d.x, d.idx[t * 3], x0); ld3(d.x, d.idx[t * 3 + 1], x1); ld3(d.x, d.idx[t * 3 + 2], x2);
  const float4 iv = d.inv[t];
  const double a = iv.x, b = iv.y, c = iv.z, dd = iv.w;
  const double e1[3] = {x1[0] - x0[0], x1[1] - x0[1], x1[2] - x0[2]};
  const double e2[3] = {x2[0] - x0[0], x2[1] - x0[1], x2[2] - x0[2]};
  double F0[3], F1[3];
  for (int i = 0; i < 3; i++) { F0[i] = a * e1[i] + c * e2[i]; F1[i] = b * e1[i] + dd * e2[i]; }
  const double E00 = 0.5 * (F0[0] * F0[0] + F0[1] * F0[1] + F0[2] * F0[2] - 1);
  const double E11 = 0.5 * (F1[0] * F1[0] + F1[1] * F1[1] + F1[2] * F1[2] - 1);
  const double E01 = 0.5 * (F0[0] * F1[0] + F0[1] * F1[1] + F0[2] * F1[2]);
  const Mat<double>& m = d.mat;
  float* o = mb.tris + (size_t)t * 16;
  for (int i = 0; i < 3; i++) { o[i] = (float)F0[i]; o[3 + i] = (float)F1[i]; }
  double S00 = m.C00 * E00 + m.C01 * E11, S11 = m.C11 * E11 + m.C01 * E00, S01 = 2 * m.G * E01;
  if (mb.psd) psd_stress(S00, S11, S01);
  o[6] = (float)S00;
  o[7] = (float)S11;
  o[8] = (float)S01;
  o[9] = iv.x; o[10] = iv.y; o[11] = iv.z; o[12] = iv.w;
  o[13] = (float)(m.thickness * (double)d.area[t]);
  o[14] = 0.f; o[15] = 0.f;
  if (mb.vrec) {
    const float4 r0 = make_float4(o[0], o[1], o[2], o[3]), r1 = make_float4(o[4], o[5], o[6], o[7]),
                 r2 = make_float4(o[8], o[9], o[10], o[11]), r3 = make_float4(o[12], o[13], 0.f, 0.f);
    for (int c = 0; c < 3; c++) {
      float4* q = mb.vrec + (size_t)mb.triSlot[t * 3 + c] * 5;
      q[0] = r0; q[1] = r1; q[2] = r2; q[3] = r3;
      q[4] = make_float4(__int_as_float((int)d.idx[t * 3]), __int_as_float((int)d.idx[t * 3 + 1]),
                         __int_as_float((int)d.idx[t * 3 + 2]), __int_as_float(c));
    }
  }
}

// Full 9x9 membrane block per triangle (FP64 closed form), stored FP32.
__global__ void __launch_bounds__(kThreads) k_mx_h9(Dev d, MixBufs mb) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.m) return;
  double x0[3], x1[3], x2[3];
  ld3(d.x, d.idx[t * 3], x0); ld3(d.x, d.idx[t * 3 + 1], x1); ld3(d.x, d.idx[t * 3 + 2], x2);
  const float4 iv = d.inv[t];
  membrane_block9<float>(x0, x1, x2, iv.x, iv.y, iv.z, iv.w, d.mat.thickness * (double)d.area[t], d.mat.C00,
                         d.mat.C11, d.mat.C01, d.mat.G, mb.h9 + (size_t)t * 81, mb.psd != 0);
}

// Exact-Newton mode: per hinge its vertex ids and the Gauss-Newton factor
// g = sqrt(k w) d phi / dx (bend_gn) in FP32, for the HVP term g (g . p).
__global__ void __launch_bounds__(kThreads) k_mx_hinge_gn(Dev d, MixBufs mb) {
  const int hh = blockIdx.x * blockDim.x + threadIdx.x;
  if (hh >= d.hg) return;
  const int4 hv = d.hinge[hh];
  double q[12], g[12];
  ld3(d.x, hv.x, q); ld3(d.x, hv.y, q + 3); ld3(d.x, hv.z, q + 6); ld3(d.x, hv.w, q + 9);
  bend_gn(q, d.hmeta[hh * 3 + 1], d.hmeta[hh * 3 + 2], d.kb, g);
  float4* o = mb.hrec + (size_t)hh * 4;
  o[0] = make_float4(__int_as_float(hv.x), __int_as_float(hv.y), __int_as_float(hv.z), __int_as_float(hv.w));
  o[1] = make_float4((float)g[0], (float)g[1], (float)g[2], (float)g[3]);
  o[2] = make_float4((float)g[4], (float)g[5], (float)g[6], (float)g[7]);
  o[3] = make_float4((float)g[8], (float)g[9], (float)g[10], (float)g[11]);
}

// Schwarz factor: assemble (FP64 sums of the stored blocks + Jacobi diagonal),
// symmetrize, Cholesky; store A^-1 = L^-T L^-1 as FP32 (Jacobi inverse on failure).
// One warp per domain, lane = local dof:
// - assembly: lane (vertex, component) owns one row and adds its incident
//   triangles' block rows in incidence order;
// - right-looking Cholesky: per pivot, every row below scales its entry and
//   updates its own part of the trailing lower triangle, in parallel;
// - L^-1 column by column (lane = column) by forward substitution in registers;
// - A^-1 row by row (lane = row).
// Rows are padded to 25 doubles so a column read by the warp spreads over banks.
constexpr int kMxWarps = 4;
constexpr int kFS = 25;
__global__ void __launch_bounds__(kMxWarps * 32) k_mx_schwarz_factor(Dev d, MixBufs mb) {
  __shared__ double A[kMxWarps][24 * kFS];
  __shared__ int dvs[kMxWarps][8];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int dom = blockIdx.x * kMxWarps + wib;
  if (dom >= d.D) return;
  double* a = A[wib];
  const int start = d.domStart[dom], dv = d.domStart[dom + 1] - start, dw = dv * 3;
  for (int i = lane; i < 24 * kFS; i += 32) a[i] = 0;
  if (lane < dv) dvs[wib][lane] = d.domVerts[start + lane];
  __syncwarp();
  if (lane < dw) {
    const int lv = lane / 3, aa = lane % 3;
    const int v = dvs[wib][lv];
    double* row = a + lane * kFS;
    if (mb.asmRec) {
      // precomputed per (vertex, incident triangle) in the v2t order: the row
      // block's offset in h9 and the corners' local members (15: outside the
      // domain); four triangles' loads in flight at once
      const uint32_t k1 = mb.asmOff[v + 1];
      for (uint32_t k0 = mb.asmOff[v]; k0 < k1; k0 += 4) {
        uint2 r[4];
#pragma unroll
        for (int u = 0; u < 4; u++) r[u] = k0 + u < k1 ? mb.asmRec[k0 + u] : make_uint2(0u, 0xfffu);
        float hv[4][9];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const float* h = mb.h9 + (size_t)r[u].x + aa * 9;
#pragma unroll
          for (int e = 0; e < 9; e++) hv[u][e] = (r[u].y & 0xfffu) != 0xfffu ? h[e] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
          for (int cj = 0; cj < 3; cj++) {
            const int lw = (int)((r[u].y >> (4 * cj)) & 15u);
            if (lw < 15)
              for (int bb = 0; bb < 3; bb++) row[lw * 3 + bb] += hv[u][cj * 3 + bb];
          }
      }
    } else {
      for (int k = d.v2tOff[v]; k < d.v2tOff[v + 1]; k++) {
        const int t = d.v2t[k];
        const int cvs[3] = {(int)d.idx[t * 3], (int)d.idx[t * 3 + 1], (int)d.idx[t * 3 + 2]};
        const int ci = cvs[0] == v ? 0 : cvs[1] == v ? 1 : 2;
        const float* h = mb.h9 + (size_t)t * 81 + (ci * 3 + aa) * 9;
        for (int cj = 0; cj < 3; cj++) {
          int lw = -1;
          for (int q = 0; q < dv; q++)
            if (dvs[wib][q] == cvs[cj]) { lw = q; break; }
          if (lw < 0) continue;
          for (int bb = 0; bb < 3; bb++) row[lw * 3 + bb] += h[cj * 3 + bb];
        }
      }
    }
    row[lane] += d.diag[v * 3 + aa];
  }
  __syncwarp();
  // two-level: the coarse diagonal diag(R A P) of this domain, the sum of its
  // component-c entries over member pairs divided by |d| (mas.ts:57-101)
  if (mb.dcoarse && lane < 3) {
    double c = 0;
    for (int i = 0; i < dv; i++)
      for (int j = 0; j < dv; j++) c += a[(i * 3 + lane) * kFS + j * 3 + lane];
    reinterpret_cast<float*>(mb.dcoarse + dom)[lane] = (float)(c / dv);
  }
  for (int i = lane; i < dw; i += 32)
    for (int j = i + 1; j < dw; j++) {
      const double sv = 0.5 * (a[i * kFS + j] + a[j * kFS + i]);
      a[i * kFS + j] = sv;
      a[j * kFS + i] = sv;
    }
  __syncwarp();
  double scale = 0;
  for (int i = 0; i < dw; i++) scale = fmax(scale, fabs(a[i * kFS + i]));
  const double tiny = 1e-20 * (1 + scale);
  bool ok = true;
  for (int k = 0; k < dw; k++) {
    const double piv = a[k * kFS + k];  // the same value in every lane
    ok = piv > tiny;
    if (!ok) break;
    const double lkk = sqrt(piv);
    __syncwarp();
    if (lane == k) a[k * kFS + k] = lkk;
    if (lane > k && lane < dw) a[lane * kFS + k] /= lkk;
    __syncwarp();
    if (lane > k && lane < dw) {
      const double lik = a[lane * kFS + k];
      for (int j = k + 1; j <= lane; j++) a[lane * kFS + j] -= lik * a[j * kFS + k];
    }
    __syncwarp();
  }
  float* Li = mb.Linv + (size_t)dom * 576;
  if (!ok) {
    for (int i = lane; i < 24; i += 32)
      for (int j = 0; j < 24; j++) {
        double v = 0;
        if (i == j && i < dw) {
          const double dd = d.diag[dvs[wib][i / 3] * 3 + i % 3];
          v = dd > 1e-12 ? 1 / dd : 0.0;
        }
        Li[i * 24 + j] = (float)v;
      }
    return;
  }
  // column `lane` of L^-1: forward substitution with the right-hand side e_lane,
  // eliminating column by column (rows past dw hold zeros)
  double col[24];
#pragma unroll
  for (int i = 0; i < 24; i++) col[i] = i == lane ? 1.0 : 0.0;
#pragma unroll
  for (int i = 0; i < 24; i++) {
    if (i < dw) {
      const double xi = col[i] / a[i * kFS + i];
      col[i] = xi;
#pragma unroll
      for (int r = i + 1; r < 24; r++) col[r] -= a[r * kFS + i] * xi;
    }
  }
  __syncwarp();
  // a = L^-1 (row-major), written once every lane has finished reading L
#pragma unroll
  for (int i = 0; i < 24; i++)
    if (i < dw && lane < dw) a[i * kFS + lane] = col[i];
  __syncwarp();
  // A^-1[i][j] = sum_k L^-1[k][i] L^-1[k][j]; lane i writes row i
  if (lane < 24) {
    for (int j = 0; j < 24; j++) {
      double sv = 0;
      if (lane < dw && j < dw)
        for (int k = 0; k < dw; k++) sv += a[k * kFS + lane] * a[k * kFS + j];
      Li[lane * 24 + j] = (float)sv;
    }
  }
}

// ---- PCG (pcg.ts:11-95) in FP32 with FP64 reductions, + newton.ts:152-179 --------------
struct MxArgs {
  Dev d;
  MixBufs mb;
  int maxIters;
  double tol;
};

__device__ __forceinline__ double mx_total(const Dev& d, int row, double* bc) {
  if (threadIdx.x < 32) {
    const double s = warp_sum_partials(d.part + row * d.partStride, gridDim.x);
    if (threadIdx.x == 0) bc[0] = s;
  }
  __syncthreads();
  const double r = bc[0];
  __syncthreads();
  return r;
}
__device__ __forceinline__ void mx_put(const Dev& d, int row, double v, double* sm) {
  const double b = block_sum(v, sm);
  if (threadIdx.x == 0) d.part[row * d.partStride + blockIdx.x] = b;
}

// z = A_d^-1 r on every domain, one warp per domain, lane = local dof.
__device__ __forceinline__ double mx_schwarz(const Dev& d, const MixBufs& mb, int gwarp, int nwarps) {
  const int lane = threadIdx.x & 31;
  double rz = 0;
  for (int dom = gwarp; dom < d.D; dom += nwarps) {
    const int start = d.domStart[dom], dv = d.domStart[dom + 1] - start, dw = dv * 3;
    float rv = 0.f;
    int gi = -1;
    if (lane < dw) {
      gi = d.domVerts[start + lane / 3] * 3 + lane % 3;
      rv = mb.r[gi];
    }
    const float* Li = mb.Linv + (size_t)dom * 576 + lane * 24;
    float z = 0.f;
    for (int j = 0; j < 24; j++) {
      const float rj = __shfl_sync(0xffffffffu, rv, j);
      if (lane < dw) z = fmaf(Li[j], rj, z);
    }
    if (mb.dcoarse) z += coarse_share(mb, dom, rv, dv);
    if (lane < dw) {
      if (d.pinned[gi / 3]) z = 0.f;
      mb.z[gi] = z;
      rz += (double)rv * (double)z;
    }
  }
  return rz;
}

__global__ void __launch_bounds__(kThreads) k_mx_pcg(MxArgs A) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double sm[32];
  __shared__ double bc[2];
  const Dev& d = A.d;
  const MixBufs& mb = A.mb;
  const int n3 = d.n * 3;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const int gwarp = tid >> 5, nwarps = nth >> 5;
  const bool jacobi = d.precond == 0;
  const float invH2 = (float)d.invH2;
  double bb = 0, rr = 0, rz0 = 0;
  for (int i = tid; i < n3; i += nth) {
    const double bi = -d.g[i];
    bb += bi * bi;
    const float ri = d.pinned[i / 3] ? 0.f : (float)bi;
    mb.r[i] = ri;
    mb.x[i] = 0.f;
    rr += (double)ri * ri;
    if (jacobi) {
      float zi = d.diag[i] > 1e-12 ? (float)((double)ri / d.diag[i]) : ri;
      if (d.pinned[i / 3]) zi = 0.f;
      mb.z[i] = zi;
      mb.p[i] = zi;
      rz0 += (double)ri * zi;
    }
  }
  mx_put(d, 0, bb, sm);
  mx_put(d, 1, rr, sm);
  if (jacobi) mx_put(d, 2, rz0, sm);
  grid.sync();
  if (!jacobi) {
    const double rzp = mx_schwarz(d, mb, gwarp, nwarps);
    mx_put(d, 2, rzp, sm);
    grid.sync();
    for (int i = tid; i < n3; i += nth) mb.p[i] = mb.z[i];
  }
  double rz = mx_total(d, 2, bc);
  const double bNorm = sqrt(mx_total(d, 0, bc));
  const double absTol = fmax(A.tol * fmax(bNorm, 1e-12), 1e-12);
  double residual = sqrt(mx_total(d, 1, bc));
  int iters = 0;
  bool done = residual < absTol;
  if (!done) grid.sync();
  int k = 0;
  for (; !done && k < A.maxIters; k++) {
    // element HVP from the stored (F, S): dF = Ds(p) Dm^-1, dE, dS, dP = dF S + F dS
    for (int t = tid; t < d.m; t += nth) {
      const float* T = mb.tris + (size_t)t * 16;
      const float4 t0 = *(const float4*)T, t1 = *(const float4*)(T + 4), t2 = *(const float4*)(T + 8),
                   t3 = *(const float4*)(T + 12);
      const float F0[3] = {t0.x, t0.y, t0.z}, F1[3] = {t0.w, t1.x, t1.y};
      const float S00 = t1.z, S11 = t1.w, S01 = t2.x;
      const float a = t2.y, b = t2.z, c = t2.w, dd = t3.x, s = t3.y;
      const uint32_t i0 = d.idx[t * 3], i1 = d.idx[t * 3 + 1], i2 = d.idx[t * 3 + 2];
      float w1[3], w2[3];
      for (int q = 0; q < 3; q++) {
        const float p0 = mb.p[i0 * 3 + q];
        w1[q] = mb.p[i1 * 3 + q] - p0;
        w2[q] = mb.p[i2 * 3 + q] - p0;
      }
      float dF0[3], dF1[3];
      for (int q = 0; q < 3; q++) { dF0[q] = a * w1[q] + c * w2[q]; dF1[q] = b * w1[q] + dd * w2[q]; }
      const float dE00 = F0[0] * dF0[0] + F0[1] * dF0[1] + F0[2] * dF0[2];
      const float dE11 = F1[0] * dF1[0] + F1[1] * dF1[1] + F1[2] * dF1[2];
      const float dE01 = 0.5f * (dF0[0] * F1[0] + F0[0] * dF1[0] + dF0[1] * F1[1] + F0[1] * dF1[1] +
                                 dF0[2] * F1[2] + F0[2] * dF1[2]);
      const float dS00 = mb.C00 * dE00 + mb.C01 * dE11;
      const float dS11 = mb.C11 * dE11 + mb.C01 * dE00;
      const float dS01 = 2.f * mb.G * dE01;
      float* o = mb.elem + (size_t)t * 9;
      for (int q = 0; q < 3; q++) {
        const float P0 = dF0[q] * S00 + F0[q] * dS00 + dF1[q] * S01 + F1[q] * dS01;
        const float P1 = dF0[q] * S01 + F0[q] * dS01 + dF1[q] * S11 + F1[q] * dS11;
        const float g1 = s * (P0 * a + P1 * b);
        const float g2 = s * (P0 * c + P1 * dd);
        o[q] = -(g1 + g2);
        o[3 + q] = g1;
        o[6 + q] = g2;
      }
    }
    if (d.hasContact) {
      // frozen-barrier coefficients in FP64 (contact-assembly.ts:371-387)
      const Contact& c = d.c;
      for (int i = tid, na = n_active(c); i < na; i += nth) {
        const Frozen f = c.active[i];
        const double dist = js_max(frozen_dist(c, d.x, f), 1e-12);
        double jv;
        if (f.kind == 2) jv = mb.p[f.p * 3 + 1];
        else {
          double v[4][3] = {};
          const int ids[4] = {f.kind == 0 ? f.p : f.a, f.kind == 0 ? f.a : f.b, f.kind == 0 ? f.b : f.c,
                              f.kind == 0 ? f.c : f.d};
          for (int q = 0; q < 4; q++)
            if (ids[q] >= 0)
              for (int e = 0; e < 3; e++) v[q][e] = mb.p[ids[q] * 3 + e];
          const double nv[4] = {f.nx * v[0][0] + f.ny * v[0][1] + f.nz * v[0][2],
                                f.nx * v[1][0] + f.ny * v[1][1] + f.nz * v[1][2],
                                f.nx * v[2][0] + f.ny * v[2][1] + f.nz * v[2][2],
                                f.nx * v[3][0] + f.ny * v[3][1] + f.nz * v[3][2]};
          if (f.kind == 0) jv = nv[0] - f.w0 * nv[1] - f.w1 * nv[2] - f.w2 * nv[3];
          else jv = f.w0 * nv[0] + f.w1 * nv[1] + f.w2 * nv[2] + f.w3 * nv[3];
        }
        c.dd[i] = dist < c.dHat ? barrier_curvature(dist, c.dHat, c.kappa) * jv : 0.0;
      }
    }
    grid.sync();
    double pAp = 0;
    for (int v = tid; v < d.n; v += nth) {
      float sp[3] = {0.f, 0.f, 0.f};
      for (uint32_t q = d.memOff[v]; q < d.memOff[v + 1]; q++) {
        const uint32_t rec = d.memRec[q];
        const float* e = mb.elem + (size_t)(rec >> 2) * 9 + (rec & 3) * 3;
        sp[0] += e[0]; sp[1] += e[1]; sp[2] += e[2];
      }
      double ch[3] = {0, 0, 0};
      if (d.hasContact) contact_hvp_gather(d, v, ch);
      const float M = d.mass[v];
      const bool pin = d.pinned[v];
      for (int q = 0; q < 3; q++) {
        const int i = v * 3 + q;
        float ap = M * mb.p[i] * invH2 + sp[q] + (float)ch[q];
        if (pin) ap = 0.f;
        mb.Ap[i] = ap;
        pAp += (double)mb.p[i] * ap;
      }
    }
    mx_put(d, 3, pAp, sm);
    grid.sync();
    const double pApT = mx_total(d, 3, bc);
    if (!(pApT > 1e-30)) { iters = k; done = true; break; }
    const float alpha = (float)(rz / pApT);
    double rrn = 0, rzn = 0;
    for (int i = tid; i < n3; i += nth) {
      const bool pin = d.pinned[i / 3];
      float xi = mb.x[i] + alpha * mb.p[i];
      float ri = mb.r[i] - alpha * mb.Ap[i];
      if (pin) { xi = 0.f; ri = 0.f; }
      mb.x[i] = xi;
      mb.r[i] = ri;
      rrn += (double)ri * ri;
      if (jacobi) {
        float zi = d.diag[i] > 1e-12 ? (float)((double)ri / d.diag[i]) : ri;
        if (pin) zi = 0.f;
        mb.z[i] = zi;
        rzn += (double)ri * zi;
      }
    }
    mx_put(d, 4, rrn, sm);
    if (jacobi) mx_put(d, 5, rzn, sm);
    grid.sync();
    residual = sqrt(mx_total(d, 4, bc));
    if (residual < absTol) { iters = k + 1; done = true; break; }
    if (!jacobi) {
      const double rzp = mx_schwarz(d, mb, gwarp, nwarps);
      mx_put(d, 5, rzp, sm);
      grid.sync();
    }
    const double rzNew = mx_total(d, 5, bc);
    const float beta = (float)(rzNew / rz);
    for (int i = tid; i < n3; i += nth) mb.p[i] = mb.z[i] + beta * mb.p[i];
    rz = rzNew;
    grid.sync();
  }
  if (!done) iters = A.maxIters;
  grid.sync();
  // descent safeguard + trust region in FP64 (dx kept in d.dx)
  double gt = 0;
  for (int i = tid; i < n3; i += nth) {
    const double di = mb.x[i];
    d.dx[i] = di;
    gt += d.g[i] * di;
  }
  mx_put(d, 6, gt, sm);
  grid.sync();
  double gtdx = mx_total(d, 6, bc);
  bool fallback = false;
  if (!isfinite(gtdx) || gtdx >= 0) {
    fallback = true;
    gt = 0;
    for (int i = tid; i < n3; i += nth) {
      const double di = -d.g[i] / d.diag[i];
      d.dx[i] = di;
      gt += d.g[i] * di;
    }
    mx_put(d, 7, gt, sm);
    grid.sync();
    gtdx = mx_total(d, 7, bc);
  }
  double mxd = 0;
  for (int i = tid; i < n3; i += nth) {
    const double a = fabs(d.dx[i]);
    if (a > mxd) mxd = a;
  }
  // max over the grid (exact in any order)
  {
    double v = mxd;
    for (int o = 16; o > 0; o >>= 1) {
      const double w = __shfl_down_sync(0xffffffffu, v, o);
      if (w > v) v = w;
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double r = 0;
      for (int i = 0; i < (int)(blockDim.x >> 5); i++) if (sm[i] > r) r = sm[i];
      d.part[0 * d.partStride + blockIdx.x] = r;
    }
  }
  grid.sync();
  if (threadIdx.x == 0) {
    double r = 0;
    for (int i = 0; i < (int)gridDim.x; i++) {
      const double v = d.part[i];
      if (v > r) r = v;
    }
    bc[0] = r;
  }
  __syncthreads();
  const double maxDx = bc[0];
  if (maxDx > 0.002) {
    const double s = 0.002 / maxDx;
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

// ---- FP64 reductions as trees (the gradient norm and the Armijo energy) ----------------
__global__ void __launch_bounds__(kThreads) k_mx_sum_terms(const double* t, int n, double* part) {
  __shared__ double sm[32];
  double s = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += t[i];
  const double b = block_sum(s, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = b;
}
// The three energy term arrays in one launch: blockIdx.y picks the array; each
// is summed over the same block partition as a k_mx_sum_terms launch of gridDim.x.
__global__ void __launch_bounds__(kThreads) k_mx_sum_terms3(const double* t0, int n0, const double* t1, int n1,
                                                           const double* t2, int n2, double* p0, double* p1,
                                                           double* p2, const int* dn2) {
  __shared__ double sm[32];
  const double* t = blockIdx.y == 0 ? t0 : blockIdx.y == 1 ? t1 : t2;
  const int n = blockIdx.y == 0 ? n0 : blockIdx.y == 1 ? n1 : (dn2 ? min(n2, *dn2) : n2);
  double* part = blockIdx.y == 0 ? p0 : blockIdx.y == 1 ? p1 : p2;
  double s = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += t[i];
  const double b = block_sum(s, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = b;
}
__global__ void k_mx_grad_final(Dev d, int nbT, int nbG) {
  if (threadIdx.x >= 32) return;
  const double ms = warp_max_partials(d.part + 0 * d.partStride, nbT);
  const double gs = warp_sum_partials(d.part + 1 * d.partStride, nbG);
  if (threadIdx.x == 0) {
    d.scal[S_GRADNORM] = sqrt(gs);
    d.scal[S_MAXSTRAIN] = ms;
  }
}
__global__ void k_mx_energy_final(Dev d, int nb) {
  if (threadIdx.x >= 32) return;
  const double ei = warp_sum_partials(d.part + 2 * d.partStride, nb);
  const double et = warp_sum_partials(d.part + 3 * d.partStride, nb);
  const double em = warp_sum_partials(d.part + 4 * d.partStride, nb);
  if (threadIdx.x == 0) {
    d.scal[S_E_INERTIA] = ei;
    d.scal[S_E_TRI] = et;
    d.scal[S_E_MERIT] = em;
    double e = ei + et;
    if (d.hasContact) e += em;
    d.scal[S_ENERGY_TRIAL] = e;
  }
}

// ---- launchers ---------------------------------------------------------------------------
void mx_prepare(const Dev& d, const MixBufs& mb, bool schwarz, cudaStream_t s, int64_t* lc) {
  k_mx_tristate<<<mblk(d.m), kThreads, 0, s>>>(d, mb);
  *lc += 1;
  if (mb.hrec && d.hg > 0) {
    k_mx_hinge_gn<<<mblk(d.hg), kThreads, 0, s>>>(d, mb);
    *lc += 1;
  }
  if (schwarz) {
    k_mx_h9<<<mblk(d.m), kThreads, 0, s>>>(d, mb);
    k_mx_schwarz_factor<<<(d.D + kMxWarps - 1) / kMxWarps, kMxWarps * 32, 0, s>>>(d, mb);
    *lc += 2;
  }
}
int mx_pcg_grid_blocks(const Dev& d) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_mx_pcg, kThreads, 0);
  const int want = mblk(std::max(d.n * 3, d.m));
  int cap = per * sms;
  if (cap < 1) cap = 1;
  return std::max(1, std::min(want, std::min(cap, d.partStride)));
}
int mx_launch_pcg(const Dev& d, const MixBufs& mb, int maxIters, double tol, int blocks, cudaStream_t s) {
  MxArgs a{d, mb, maxIters, tol};
  void* args[] = {&a};
  return (int)cudaLaunchCooperativeKernel((void*)k_mx_pcg, dim3(blocks), dim3(kThreads), args, 0, s);
}
// Gradient norm from the T0 terms the gather wrote (tree instead of chain).
void mx_grad_final(const Dev& d, cudaStream_t s, int64_t* lc) {
  const int nbG = std::min(mblk(d.n * 3), d.partStride);
  k_mx_sum_terms<<<nbG, kThreads, 0, s>>>(d.T0, d.n * 3, d.part + 1 * d.partStride);
  k_mx_grad_final<<<1, 32, 0, s>>>(d, mblk(d.m), nbG);
  *lc += 2;
}
// Armijo energy from the T0 / T1 / Tc terms (tree sums).
void mx_energy_final(const Dev& d, cudaStream_t s, int64_t* lc) {
  const int nb = std::min(mblk(std::max(std::max(d.n * 3, d.m + d.hg), d.hasContact ? d.c.nActive : 0)),
                          d.partStride);
  k_mx_sum_terms3<<<dim3(nb, 3), kThreads, 0, s>>>(d.T0, d.n * 3, d.T1, d.m + (d.kb > 0 ? d.hg : 0), d.Tc,
                                                   d.hasContact ? d.c.nActive : 0, d.part + 2 * d.partStride,
                                                   d.part + 3 * d.partStride, d.part + 4 * d.partStride,
                                                   d.hasContact ? d.c.nActiveD : nullptr);
  k_mx_energy_final<<<1, 32, 0, s>>>(d, nb);
  *lc += 2;
}

}  // namespace cs
