// Device functions of the frozen-contact model used inside the FP64 kernels
// (reference src/collision/contact-assembly.ts:222-414).
#pragma once
#include "contact_math.cuh"
#include "plain.cuh"

namespace cs {

__device__ __forceinline__ void cpos(const Contact& c, const double* x, int v, double o[3]) {
  if (v >= 0) { o[0] = x[v * 3]; o[1] = x[v * 3 + 1]; o[2] = x[v * 3 + 2]; return; }
  const int i = -v - 2;
  o[0] = c.spos[i * 3]; o[1] = c.spos[i * 3 + 1]; o[2] = c.spos[i * 3 + 2];
}

// frozenDist (contact-assembly.ts:222-258): n . r(x) with lagged weights.
__device__ __forceinline__ double frozen_dist(const Contact& c, const double* x, const Frozen& f) {
  if (f.kind == 2) return x[f.p * 3 + 1] - c.floorY;
  if (f.kind == 0) {
    double A[3], B[3], C[3];
    cpos(c, x, f.a, A); cpos(c, x, f.b, B); cpos(c, x, f.c, C);
    const double qx = f.w0 * A[0] + f.w1 * B[0] + f.w2 * C[0];
    const double qy = f.w0 * A[1] + f.w1 * B[1] + f.w2 * C[1];
    const double qz = f.w0 * A[2] + f.w1 * B[2] + f.w2 * C[2];
    const double ddx = x[f.p * 3] - qx, ddy = x[f.p * 3 + 1] - qy, ddz = x[f.p * 3 + 2] - qz;
    return f.nx * ddx + f.ny * ddy + f.nz * ddz;
  }
  double A[3], B[3], C[3], D[3];
  cpos(c, x, f.a, A); cpos(c, x, f.b, B); cpos(c, x, f.c, C); cpos(c, x, f.d, D);
  const double rx = f.w0 * A[0] + f.w1 * B[0] + f.w2 * C[0] + f.w3 * D[0];
  const double ry = f.w0 * A[1] + f.w1 * B[1] + f.w2 * C[1] + f.w3 * D[1];
  const double rz = f.w0 * A[2] + f.w1 * B[2] + f.w2 * C[2] + f.w3 * D[2];
  return f.nx * rx + f.ny * ry + f.nz * rz;
}

// distJvp (contact-assembly.ts:394-414).
__device__ __forceinline__ double dist_jvp(const Frozen& f, const double* v) {
  if (f.kind == 2) return v[f.p * 3 + 1];
  if (f.kind == 0) {
    double j = f.nx * v[f.p * 3] + f.ny * v[f.p * 3 + 1] + f.nz * v[f.p * 3 + 2];
    const double ws[3] = {f.w0, f.w1, f.w2};
    const int vs[3] = {f.a, f.b, f.c};
    for (int k = 0; k < 3; k++) {
      if (vs[k] < 0) continue;
      j -= ws[k] * (f.nx * v[vs[k] * 3] + f.ny * v[vs[k] * 3 + 1] + f.nz * v[vs[k] * 3 + 2]);
    }
    return j;
  }
  const double ws[4] = {f.w0, f.w1, f.w2, f.w3};
  const int vs[4] = {f.a, f.b, f.c, f.d};
  double j = 0;
  for (int k = 0; k < 4; k++) {
    if (vs[k] < 0) continue;
    j += ws[k] * (f.nx * v[vs[k] * 3] + f.ny * v[vs[k] * 3 + 1] + f.nz * v[vs[k] * 3 + 2]);
  }
  return j;
}

// addDistGrad contribution of one stencil slot (contact-assembly.ts:288-315).
__device__ __forceinline__ void dist_grad_slot(const Frozen& f, int slot, double g, double o[3]) {
  if (f.kind == 2) { o[1] += g; return; }
  if (f.kind == 0) {
    if (slot == 0) { o[0] += g * f.nx; o[1] += g * f.ny; o[2] += g * f.nz; return; }
    const double w = slot == 1 ? f.w0 : slot == 2 ? f.w1 : f.w2;
    o[0] += -g * w * f.nx; o[1] += -g * w * f.ny; o[2] += -g * w * f.nz;
    return;
  }
  const double w = slot == 0 ? f.w0 : slot == 1 ? f.w1 : slot == 2 ? f.w2 : f.w3;
  o[0] += g * w * f.nx; o[1] += g * w * f.ny; o[2] += g * w * f.nz;
}

// addFrictionForce contribution of one slot (contact-assembly.ts:318-341).
__device__ __forceinline__ void friction_slot(const Frozen& f, int slot, const double* ff, double o[3]) {
  if (f.kind == 2 || (f.kind == 0 && slot == 0)) { o[0] += ff[0]; o[1] += ff[1]; o[2] += ff[2]; return; }
  if (f.kind == 0) {
    const double w = slot == 1 ? f.w0 : slot == 2 ? f.w1 : f.w2;
    o[0] += -ff[0] * w; o[1] += -ff[1] * w; o[2] += -ff[2] * w;
    return;
  }
  const double w = slot == 0 ? f.w0 : slot == 1 ? f.w1 : slot == 2 ? -f.w2 : -f.w3;
  o[0] += ff[0] * w; o[1] += ff[1] * w; o[2] += ff[2] * w;
}

// Relative-slip Jacobian along v (the derivative of relativeSlip,
// contact-assembly.ts:344-367, including its D(c.d) reading for the third
// triangle vertex of a VT contact, which makes that vertex drop out).
__device__ __forceinline__ void slip_jvp(const Frozen& f, const double* v, double o[3]) {
  auto V = [&](int q, double s, double* acc) {
    if (q < 0) return;
    acc[0] += s * v[q * 3]; acc[1] += s * v[q * 3 + 1]; acc[2] += s * v[q * 3 + 2];
  };
  o[0] = o[1] = o[2] = 0;
  if (f.kind == 2) { V(f.p, 1.0, o); return; }
  if (f.kind == 0) { V(f.p, 1.0, o); V(f.a, -f.w0, o); V(f.b, -f.w1, o); return; }
  V(f.a, f.w0, o); V(f.b, f.w1, o); V(f.c, f.w2, o); V(f.d, f.w3, o);
}

// Transpose of slip_jvp for one stencil slot: adds the slot's share of F.
__device__ __forceinline__ void slip_jt_slot(const Frozen& f, int slot, const double F[3], double o[3]) {
  double w;
  if (f.kind == 2) w = slot == 0 ? 1.0 : 0.0;
  else if (f.kind == 0) w = slot == 0 ? 1.0 : slot == 1 ? -f.w0 : slot == 2 ? -f.w1 : 0.0;
  else w = slot == 0 ? f.w0 : slot == 1 ? f.w1 : slot == 2 ? f.w2 : f.w3;
  o[0] += w * F[0]; o[1] += w * F[1]; o[2] += w * F[2];
}

// Friction Hessian applied to a slip increment du: s (P du - t (t . du)),
// P = I - n n^T (exact-Newton mode; fh as in Contact).
__device__ __forceinline__ void fric_hess_apply(const double* fh, const double du[3], double F[3]) {
  const double s = fh[1];
  const double nd = fh[5] * du[0] + fh[6] * du[1] + fh[7] * du[2];
  const double pu[3] = {du[0] - nd * fh[5], du[1] - nd * fh[6], du[2] - nd * fh[7]};
  const double td = fh[2] * pu[0] + fh[3] * pu[1] + fh[4] * pu[2];
  F[0] = s * (pu[0] - td * fh[2]);
  F[1] = s * (pu[1] - td * fh[3]);
  F[2] = s * (pu[2] - td * fh[4]);
}

// Per-contact HVP coefficient dd = kappa max(b'', 0) * (J v) (contact-assembly.ts:371-387).
__device__ __forceinline__ void contact_hvp_coeffs(const Dev& d, const double* v, int tid, int nth) {
  const Contact& c = d.c;
  for (int i = tid, na = n_active(c); i < na; i += nth) {
    const Frozen f = c.active[i];
    const double dist = js_max(frozen_dist(c, d.x, f), 1e-12);
    double dd = 0;
    if (dist < c.dHat) dd = barrier_curvature(dist, c.dHat, c.kappa) * dist_jvp(f, v);
    c.dd[i] = dd;
    if (c.fric) {
      double F[3] = {0, 0, 0};
      if (c.fh[i * 8 + 1] != 0) {
        double du[3];
        slip_jvp(f, v, du);
        fric_hess_apply(c.fh + i * 8, du, F);
      }
      c.fdd[i * 3] = F[0]; c.fdd[i * 3 + 1] = F[1]; c.fdd[i * 3 + 2] = F[2];
    }
  }
}

// Per-vertex sum of the contact HVP, contacts in order (contact-assembly.ts:388-391).
__device__ __forceinline__ void contact_hvp_gather(const Dev& d, int vtx, double out[3]) {
  const Contact& c = d.c;
  out[0] = out[1] = out[2] = 0;
  for (uint32_t k = c.cOff[vtx]; k < c.cOff[vtx + 1]; k++) {
    const uint32_t rec = c.cRec[k];
    const double g = c.dd[rec >> 2];
    if (c.fric) slip_jt_slot(c.active[rec >> 2], rec & 3, c.fdd + (rec >> 2) * 3, out);
    if (g == 0) continue;
    dist_grad_slot(c.active[rec >> 2], rec & 3, g, out);
  }
}

}  // namespace cs
