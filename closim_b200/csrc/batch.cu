// Batched implicit step: one launch steps every sheet of a packed work list.
//
// Each sheet is an independent scene (no coupling), so a sheet maps to ONE
// thread block that runs its whole step -- predictor and floor-CCD bisection,
// up to newtonIters Newton iterations (gradient, FP32 Jacobi-PCG with FP64 dot
// products, descent safeguard, 2 mm trust region, CCD-gated Armijo search,
// lagged-friction commit), velocity update and restitution -- with block
// barriers only: no grid-wide synchronization and no host round trip. The
// launch is persistent: blocks take sheets from a work list ordered largest
// first. The algorithm per sheet is newton.ts:27-303 with the floor-contact
// subset of contact-assembly.ts (kind 2: per-vertex barrier, lagged friction,
// floor CCD, restitution); the bending gradient is the analytic gradient of
// the hinge energy instead of its central difference (bending.ts:19-42).
// Every reduction is a fixed-order block tree, so a sheet's result does not
// depend on which block or how many blocks run it.
#include "adjoint_math.cuh"
#include "batch.cuh"
#include "contact_math.cuh"
#include "elem.cuh"
#include "hvp32.cuh"

namespace cs {

namespace {

struct Range {
  int v0, v1, t0, t1, h0, h1;
};

__device__ __forceinline__ void ld3b(const double* x, int v, double o[3]) {
  o[0] = x[v * 3]; o[1] = x[v * 3 + 1]; o[2] = x[v * 3 + 2];
}

__device__ __forceinline__ void enforce_pins(const BatchDev& b, const Range& R, double* x) {
  for (int v = R.v0 + threadIdx.x; v < R.v1; v += blockDim.x)
    if (b.pinned[v])
      for (int k = 0; k < 3; k++) x[v * 3 + k] = b.pinPos[v * 3 + k];
}

// checkTrial restricted to the floor (contact-assembly.ts:489-553): the
// smallest floor distance must exceed dMin and no vertex may cross the dMin
// level during x0 -> xT.
__device__ bool floor_trial_ok(const BatchDev& b, const Range& R, const double* xT, double* sm) {
  if (!b.hasFloor) return true;
  double mn = INFINITY;
  int bad = 0;
  for (int v = R.v0 + threadIdx.x; v < R.v1; v += blockDim.x) {
    const double yT = xT[v * 3 + 1] - b.floorY;
    if (yT < mn || yT != yT) mn = yT != yT ? -INFINITY : yT;
    const double y0 = b.x0[v * 3 + 1] - b.floorY;
    if (y0 - fabs(yT - y0) > b.dMin) continue;
    if (y0 > b.dMin && yT <= b.dMin && y0 > yT) {
      const double toi = (y0 - b.dMin) / (y0 - yT);
      if (toi < 1 - 1e-9) bad = 1;
    }
  }
  const double m = block_min(mn, sm);
  const double anyBad = block_max((double)bad, sm);
  return !(m <= b.dMin) && anyBad == 0;
}

__device__ __forceinline__ void update_active(const BatchDev& b, const Range& R, const double* x) {
  for (int v = R.v0 + threadIdx.x; v < R.v1; v += blockDim.x)
    b.act[v] = b.hasFloor && (x[v * 3 + 1] - b.floorY < b.dHat) ? 1 : 0;
}

// totalEnergy (newton.ts:76-88): inertia + membrane + bending + barrier merit.
__device__ double sheet_energy(const BatchDev& b, const Range& R, const double* x, const Mat<double>& mt, double kb,
                               double* sm) {
  double e = 0;
  for (int v = R.v0 + threadIdx.x; v < R.v1; v += blockDim.x) {
    const double M = b.mass[v];
    for (int k = 0; k < 3; k++) {
      const double d = x[v * 3 + k] - b.yHat[v * 3 + k];
      e += 0.5 * M * d * d * b.invH2;
    }
    if (b.act[v]) {
      const double d = fmax(x[v * 3 + 1] - b.floorY, 1e-12);
      if (d < b.dHat) e += b.kappa * barrier_value(d, b.dHat);
    }
  }
  for (int t = R.t0 + threadIdx.x; t < R.t1; t += blockDim.x) {
    double p0[3], p1[3], p2[3];
    ld3b(x, b.idx[t * 3], p0); ld3b(x, b.idx[t * 3 + 1], p1); ld3b(x, b.idx[t * 3 + 2], p2);
    const float4 iv = b.inv[t];
    e += tri_energy<double>(p0, p1, p2, iv.x, iv.y, iv.z, iv.w, b.area[t], mt);
  }
  if (kb > 0)
    for (int hh = R.h0 + threadIdx.x; hh < R.h1; hh += blockDim.x) {
      const int4 hv = b.hinge[hh];
      double q[12], gdum[12];
      ld3b(x, hv.x, q); ld3b(x, hv.y, q + 3); ld3b(x, hv.z, q + 6); ld3b(x, hv.w, q + 9);
      e += bend_grad<double>(q, b.hmeta[hh * 3], b.hmeta[hh * 3 + 1], b.hmeta[hh * 3 + 2], kb, gdum);
    }
  return block_sum(e, sm);
}

// Newton gradient at b.x into b.g (filtered), the barrier curvature added to
// the diagonal estimate; returns |g|.
__device__ double sheet_gradient(const BatchDev& b, const Range& R, const Mat<double>& mt, double kb, double* sm) {
  for (int t = R.t0 + threadIdx.x; t < R.t1; t += blockDim.x) {
    double p0[3], p1[3], p2[3];
    ld3b(b.x, b.idx[t * 3], p0); ld3b(b.x, b.idx[t * 3 + 1], p1); ld3b(b.x, b.idx[t * 3 + 2], p2);
    const float4 iv = b.inv[t];
    double en, gg[9], E[3];
    tri_grad<double>(p0, p1, p2, iv.x, iv.y, iv.z, iv.w, b.area[t], mt, en, gg, E);
    for (int k = 0; k < 9; k++) b.elem[(size_t)t * 9 + k] = gg[k];
  }
  if (kb > 0)
    for (int hh = R.h0 + threadIdx.x; hh < R.h1; hh += blockDim.x) {
      const int4 hv = b.hinge[hh];
      double q[12], gg[12];
      ld3b(b.x, hv.x, q); ld3b(b.x, hv.y, q + 3); ld3b(b.x, hv.z, q + 6); ld3b(b.x, hv.w, q + 9);
      bend_grad<double>(q, b.hmeta[hh * 3], b.hmeta[hh * 3 + 1], b.hmeta[hh * 3 + 2], kb, gg);
      for (int k = 0; k < 12; k++) b.helem[(size_t)hh * 12 + k] = gg[k];
    }
  __syncthreads();
  double gn = 0;
  for (int v = R.v0 + threadIdx.x; v < R.v1; v += blockDim.x) {
    double s[3] = {0, 0, 0};
    for (uint32_t q = b.memOff[v]; q < b.memOff[v + 1]; q++) {
      const uint32_t rec = b.memRec[q];
      const double* e = b.elem + (size_t)(rec >> 2) * 9 + (rec & 3) * 3;
      s[0] += e[0]; s[1] += e[1]; s[2] += e[2];
    }
    if (kb > 0)
      for (uint32_t q = b.hinOff[v]; q < b.hinOff[v + 1]; q++) {
        const uint32_t rec = b.hinRec[q];
        const double* e = b.helem + (size_t)(rec >> 2) * 12 + (rec & 3) * 3;
        s[0] += e[0]; s[1] += e[1]; s[2] += e[2];
      }
    if (b.act[v]) {
      // barrier (addDistGrad) and lagged friction (addFrictionForce) of the floor contact
      const double d = fmax(b.x[v * 3 + 1] - b.floorY, 1e-12);
      if (d < b.dHat) {
        s[1] += barrier_grad_scalar(d, b.dHat, b.kappa, 1);
        const double lam = b.lagOk[v] ? b.lagLam[v] : barrier_normal_force(d, b.dHat, b.kappa, 1);
        double u[3], fr[3];
        for (int k = 0; k < 3; k++) u[k] = b.x[v * 3 + k] - b.x0[v * 3 + k];
        coulomb_force(u, 0.0, 1.0, 0.0, lam, b.mu, b.eps, fr);
        for (int k = 0; k < 3; k++) s[k] -= fr[k];
        b.diag[v * 3 + 1] += barrier_curvature(d, b.dHat, b.kappa);  // addDiagEstimate (accumulates)
      }
    }
    const double M = b.mass[v];
    const bool pin = b.pinned[v];
    for (int k = 0; k < 3; k++) {
      const int i = v * 3 + k;
      double gi = M * (b.x[i] - b.yHat[i]) * b.invH2 + s[k];
      if (pin) gi = 0;
      b.g[i] = gi;
      gn += gi * gi;
    }
  }
  return sqrt(block_sum(gn, sm));
}

// FP32 state of every triangle for the matrix-free HVP (F, S, Dm^-1, s).
__device__ void sheet_tristate(const BatchDev& b, const Range& R, const Mat<double>& m) {
  for (int t = R.t0 + threadIdx.x; t < R.t1; t += blockDim.x) {
    double x0[3], x1[3], x2[3];
    ld3b(b.x, b.idx[t * 3], x0); ld3b(b.x, b.idx[t * 3 + 1], x1); ld3b(b.x, b.idx[t * 3 + 2], x2);
    const float4 iv = b.inv[t];
    double F0[3], F1[3];
    for (int k = 0; k < 3; k++) {
      const double e1 = x1[k] - x0[k], e2 = x2[k] - x0[k];
      F0[k] = iv.x * e1 + iv.z * e2;
      F1[k] = iv.y * e1 + iv.w * e2;
    }
    const double E00 = 0.5 * (F0[0] * F0[0] + F0[1] * F0[1] + F0[2] * F0[2] - 1);
    const double E11 = 0.5 * (F1[0] * F1[0] + F1[1] * F1[1] + F1[2] * F1[2] - 1);
    const double E01 = 0.5 * (F0[0] * F1[0] + F0[1] * F1[1] + F0[2] * F1[2]);
    float* o = b.tris + (size_t)t * 16;
    for (int k = 0; k < 3; k++) { o[k] = (float)F0[k]; o[3 + k] = (float)F1[k]; }
    o[6] = (float)(m.C00 * E00 + m.C01 * E11);
    o[7] = (float)(m.C11 * E11 + m.C01 * E00);
    o[8] = (float)(2 * m.G * E01);
    o[9] = iv.x; o[10] = iv.y; o[11] = iv.z; o[12] = iv.w;
    o[13] = (float)(m.thickness * (double)b.area[t]);
    o[14] = 0.f; o[15] = 0.f;
  }
}

// Ap = (M/h^2 + H_membrane + H_floor) p in FP32; returns p.Ap (FP64). Each
// vertex adds the corner share of its incident triangles' HVP directly
// (recomputed per corner from the stored FP32 state), so no per-triangle
// result is written and read back and no barrier splits the product.
__device__ double sheet_hvp(const BatchDev& b, const Range& R, float C00, float C11, float C01, float G,
                            double* sm) {
  double pAp = 0;
  const float invH2 = (float)b.invH2;
  for (int v = R.v0 + threadIdx.x; v < R.v1; v += blockDim.x) {
    float sp[3] = {0.f, 0.f, 0.f};
    for (uint32_t q = b.memOff[v]; q < b.memOff[v + 1]; q++) {
      const uint32_t rec = __ldg(b.memRec + q);
      const uint32_t t = rec >> 2;
      const int i0 = (int)__ldg(b.idx + t * 3), i1 = (int)__ldg(b.idx + t * 3 + 1), i2 = (int)__ldg(b.idx + t * 3 + 2);
      const float3 p0 = make_float3(b.p[i0 * 3], b.p[i0 * 3 + 1], b.p[i0 * 3 + 2]);
      const float3 p1 = make_float3(b.p[i1 * 3], b.p[i1 * 3 + 1], b.p[i1 * 3 + 2]);
      const float3 p2 = make_float3(b.p[i2 * 3], b.p[i2 * 3 + 1], b.p[i2 * 3 + 2]);
      float o[3];
      tri_hvp_corner(b.tris + (size_t)t * 16, p0, p1, p2, (int)(rec & 3), C00, C11, C01, G, o);
      sp[0] += o[0]; sp[1] += o[1]; sp[2] += o[2];
    }
    float cy = 0.f;
    if (b.act[v]) {
      const double d = fmax(b.x[v * 3 + 1] - b.floorY, 1e-12);
      if (d < b.dHat) cy = (float)(barrier_curvature(d, b.dHat, b.kappa) * (double)b.p[v * 3 + 1]);
    }
    const float M = b.mass[v];
    const bool pin = b.pinned[v];
    for (int q = 0; q < 3; q++) {
      const int i = v * 3 + q;
      float ap = M * b.p[i] * invH2 + sp[q] + (q == 1 ? cy : 0.f);
      if (pin) ap = 0.f;
      b.Ap[i] = ap;
      pAp += (double)b.p[i] * ap;
    }
  }
  return block_sum(pAp, sm);
}

// pcg.ts:11-95 (Jacobi, tolerance 1e-3) and the newton.ts:152-179 epilogue;
// the direction lands in b.dx. Returns the PCG iteration count.
__device__ int sheet_pcg(const BatchDev& b, const Range& R, float C00, float C11, float C01, float G, double* sm,
                         double& gtdxOut) {
  double bb = 0, rr = 0, rz = 0;
  for (int i = 3 * R.v0 + threadIdx.x; i < 3 * R.v1; i += blockDim.x) {
    const double bi = -b.g[i];
    bb += bi * bi;
    const bool pin = b.pinned[i / 3];
    const float ri = pin ? 0.f : (float)bi;
    b.r[i] = ri;
    b.xs[i] = 0.f;
    rr += (double)ri * ri;
    const float di = pin ? 0.f : b.diag[i] > 1e-12 ? (float)(1.0 / b.diag[i]) : 1.f;
    b.dinv[i] = di;
    const float zi = ri * di;
    b.z[i] = zi;
    b.p[i] = zi;
    rz += (double)ri * zi;
  }
  const double bNorm = sqrt(block_sum(bb, sm));
  double residual = sqrt(block_sum(rr, sm));
  rz = block_sum(rz, sm);
  const double absTol = fmax(1e-3 * fmax(bNorm, 1e-12), 1e-12);
  int iters = 0;
  bool done = residual < absTol;
  int k = 0;
  for (; !done && k < b.pcgMaxIters; k++) {
    const double pAp = sheet_hvp(b, R, C00, C11, C01, G, sm);
    if (!(pAp > 1e-30)) { iters = k; done = true; break; }
    const float alpha = (float)(rz / pAp);
    double rrn = 0, rzn = 0;
    for (int i = 3 * R.v0 + threadIdx.x; i < 3 * R.v1; i += blockDim.x) {
      const bool pin = b.pinned[i / 3];
      float xi = b.xs[i] + alpha * b.p[i];
      float ri = b.r[i] - alpha * b.Ap[i];
      if (pin) { xi = 0.f; ri = 0.f; }
      b.xs[i] = xi;
      b.r[i] = ri;
      rrn += (double)ri * ri;
      const float zi = ri * b.dinv[i];
      b.z[i] = zi;
      rzn += (double)ri * zi;
    }
    residual = sqrt(block_sum(rrn, sm));
    rzn = block_sum(rzn, sm);
    if (residual < absTol) { iters = k + 1; done = true; break; }
    const float beta = (float)(rzn / rz);
    rz = rzn;
    for (int i = 3 * R.v0 + threadIdx.x; i < 3 * R.v1; i += blockDim.x) b.p[i] = b.z[i] + beta * b.p[i];
    __syncthreads();
  }
  if (!done) iters = b.pcgMaxIters;
  double gt = 0;
  for (int i = 3 * R.v0 + threadIdx.x; i < 3 * R.v1; i += blockDim.x) {
    const double di = b.xs[i];
    b.dx[i] = di;
    gt += b.g[i] * di;
  }
  double gtdx = block_sum(gt, sm);
  if (!isfinite(gtdx) || gtdx >= 0) {
    gt = 0;
    for (int i = 3 * R.v0 + threadIdx.x; i < 3 * R.v1; i += blockDim.x) {
      const double di = -b.g[i] / b.diag[i];
      b.dx[i] = di;
      gt += b.g[i] * di;
    }
    gtdx = block_sum(gt, sm);
  }
  double mx = 0;
  for (int i = 3 * R.v0 + threadIdx.x; i < 3 * R.v1; i += blockDim.x) mx = fmax(mx, fabs(b.dx[i]));
  const double maxDx = block_max(mx, sm);
  if (maxDx > 0.002) {
    const double sc = 0.002 / maxDx;
    for (int i = 3 * R.v0 + threadIdx.x; i < 3 * R.v1; i += blockDim.x) b.dx[i] *= sc;
    gtdx *= sc;
    __syncthreads();
  }
  gtdxOut = gtdx;
  return iters;
}

__device__ void step_sheet(const BatchDev& b, int s, double* sm) {
  const Range R{b.vStart[s], b.vStart[s + 1], b.tStart[s], b.tStart[s + 1], b.hStart[s], b.hStart[s + 1]};
  const double* mr = b.mat + (size_t)s * BM_N;
  const Mat<double> mt{mr[BM_C00], mr[BM_C11], mr[BM_C01], mr[BM_G], mr[BM_THICK]};
  const double kb = mr[BM_KB], damp = mr[BM_DAMP], beta = mr[BM_BETA];
  const float C00 = (float)mr[BM_C00], C11 = (float)mr[BM_C11], C01 = (float)mr[BM_C01], G = (float)mr[BM_G];
  const double h = b.h;
  // predictor y_hat = x + h v + h^2 g, initial guess y_hat with pins (newton.ts:40-51)
  for (int v = R.v0 + threadIdx.x; v < R.v1; v += blockDim.x)
    for (int k = 0; k < 3; k++) {
      const int i = v * 3 + k;
      const double xv = b.x[i];
      b.x0[i] = xv;
      const double y = xv + h * b.v[i] + h * h * b.gravity[k];
      b.yHat[i] = y;
      b.x[i] = y;
    }
  __syncthreads();
  enforce_pins(b, R, b.x);
  __syncthreads();
  int rejected = 0;
  if (b.hasFloor && !floor_trial_ok(b, R, b.x, sm)) {
    // bisect back along x0 -> y_hat to the largest CCD-valid fraction (newton.ts:53-72)
    double lo = 0, hi = 1;
    for (int it = 0; it < 8; it++) {
      const double mid = 0.5 * (lo + hi);
      for (int i = 3 * R.v0 + threadIdx.x; i < 3 * R.v1; i += blockDim.x) b.xt[i] = b.x0[i] + mid * (b.x[i] - b.x0[i]);
      __syncthreads();
      enforce_pins(b, R, b.xt);
      __syncthreads();
      if (floor_trial_ok(b, R, b.xt, sm)) lo = mid;
      else hi = mid;
      if (hi - lo < 1e-4) break;
    }
    for (int i = 3 * R.v0 + threadIdx.x; i < 3 * R.v1; i += blockDim.x) b.x[i] = b.x0[i] + lo * (b.x[i] - b.x0[i]);
    __syncthreads();
    enforce_pins(b, R, b.x);
    __syncthreads();
  }
  update_active(b, R, b.x);
  __syncthreads();
  double energy = sheet_energy(b, R, b.x, mt, kb, sm);
  for (int v = R.v0 + threadIdx.x; v < R.v1; v += blockDim.x) {
    const double d0 = b.mass[v] * b.invH2 + beta;
    b.diag[v * 3] = d0; b.diag[v * 3 + 1] = d0; b.diag[v * 3 + 2] = d0;
  }
  __syncthreads();
  double gradNorm = INFINITY;
  int used = 0, pcgTotal = 0, trials = 0, converged = 0;
  for (int ni = 0; ni < b.newtonIters; ni++) {
    used = ni + 1;
    update_active(b, R, b.x);
    __syncthreads();
    gradNorm = sheet_gradient(b, R, mt, kb, sm);
    if (!isfinite(gradNorm)) { converged = -1; break; }
    if (gradNorm < b.gradTol) { converged = 1; break; }
    sheet_tristate(b, R, mt);
    __syncthreads();
    double gtdx;
    pcgTotal += sheet_pcg(b, R, C00, C11, C01, G, sm, gtdx);
    double alpha = 1;
    bool accepted = false;
    for (int li = 0; li < b.lsIters; li++) {
      trials++;
      for (int i = 3 * R.v0 + threadIdx.x; i < 3 * R.v1; i += blockDim.x) b.xt[i] = b.x[i] + alpha * b.dx[i];
      __syncthreads();
      enforce_pins(b, R, b.xt);
      __syncthreads();
      if (!floor_trial_ok(b, R, b.xt, sm)) { rejected++; alpha *= 0.5; continue; }
      const double eNew = sheet_energy(b, R, b.xt, mt, kb, sm);
      if (!isfinite(eNew)) { rejected++; alpha *= 0.5; continue; }
      if (eNew <= energy + 1e-4 * alpha * gtdx) {
        for (int i = 3 * R.v0 + threadIdx.x; i < 3 * R.v1; i += blockDim.x) b.x[i] = b.xt[i];
        energy = eNew;
        accepted = true;
        __syncthreads();
        // commit: lagged normal force of every active floor contact (contact-assembly.ts:475-485)
        for (int v = R.v0 + threadIdx.x; v < R.v1; v += blockDim.x)
          if (b.act[v]) {
            const double d = fmax(b.x[v * 3 + 1] - b.floorY, 1e-12);
            if (d < b.dHat) { b.lagLam[v] = barrier_normal_force(d, b.dHat, b.kappa, 1); b.lagOk[v] = 1; }
          }
        __syncthreads();
        break;
      }
      rejected++;
      alpha *= 0.5;
    }
    if (!accepted || alpha < 1e-6) break;
  }
  // velocity update, restitution-0 on floor contacts (newton.ts:222-245)
  for (int i = 3 * R.v0 + threadIdx.x; i < 3 * R.v1; i += blockDim.x) b.v[i] = ((b.x[i] - b.x0[i]) / h) * damp;
  __syncthreads();
  update_active(b, R, b.x);
  __syncthreads();
  int nfloor = 0;
  for (int v = R.v0 + threadIdx.x; v < R.v1; v += blockDim.x)
    if (b.act[v]) {
      nfloor++;
      if (b.v[v * 3 + 1] < 0) b.v[v * 3 + 1] = 0;
    }
  enforce_pins(b, R, b.x);
  const double nf = block_sum((double)nfloor, sm);
  if (threadIdx.x == 0) {
    double* o = b.out + (size_t)s * BO_N;
    o[BO_NEWTON] = used;
    o[BO_PCG] = pcgTotal;
    o[BO_GRADNORM] = gradNorm;
    o[BO_ENERGY] = energy;
    o[BO_CONVERGED] = converged;
    o[BO_TRIALS] = trials;
    o[BO_FLOOR] = nf;
    o[BO_REJECTED] = rejected;
  }
  __syncthreads();
}

template <int T>
__global__ void __launch_bounds__(T, 1) k_batch_step(BatchDev b) {
  __shared__ double sm[32];
  __shared__ int sheetSh;
  for (int guard = 0; guard <= b.S; guard++) {
    if (threadIdx.x == 0) {
      const unsigned k = atomicAdd(b.work, 1u);
      sheetSh = k < (unsigned)b.S ? b.order[k] : -1;
    }
    __syncthreads();
    const int sheet = sheetSh;
    __syncthreads();
    if (sheet < 0) return;
    step_sheet(b, sheet, sm);
  }
}

}  // namespace

int batch_max_ctas(int threads) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e = cudaSuccess;
  if (threads == 128) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_step<128>, 128, 0);
  else if (threads == 256) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_step<256>, 256, 0);
  else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_step<512>, 512, 0);
  if (e != cudaSuccess || per < 1) per = 1;
  return per * sms;
}

int batch_launch_step(const BatchDev& b, int threads, int ctas, cudaStream_t s) {
  cudaMemsetAsync(b.work, 0, sizeof(unsigned int), s);
  if (threads == 128) k_batch_step<128><<<ctas, 128, 0, s>>>(b);
  else if (threads == 256) k_batch_step<256><<<ctas, 256, 0, s>>>(b);
  else k_batch_step<512><<<ctas, 512, 0, s>>>(b);
  return (int)cudaGetLastError();
}

}  // namespace cs
