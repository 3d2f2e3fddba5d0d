// Per-primitive contact math (host + device). Same operation order as the
// reference so that each primitive's result matches it bit for bit when the
// same libm is used (the FP64 path is compiled with -fmad=false):
//   closest points  src/collision/closest-point.ts:14-108 (Ericson 5.1.5 / 5.1.9)
//   cubic roots     src/collision/cubic.ts:4-66
//   VT / EE CCD     src/collision/ccd-vt.ts:20-115, ccd-ee.ts:24-101
//   barrier         src/collision/barrier.ts:4-24
//   friction        src/collision/friction.ts:14-23
#pragma once
#include <math.h>

#include "common.cuh"
#include "jsmath.cuh"

namespace cs {

#define CSHD __host__ __device__ __forceinline__

struct Closest {
  double s, t, dist, rx, ry, rz;
};

CSHD Closest pack_cp(double s, double t, double rx, double ry, double rz) {
  Closest c;
  c.s = s; c.t = t; c.dist = js_hypot3(rx, ry, rz); c.rx = rx; c.ry = ry; c.rz = rz;
  return c;
}

// Vertex p vs triangle (a, b, c); s weights b, t weights c.
CSHD Closest closest_vt(const double* P, const double* A, const double* B, const double* Cc) {
  const double px = P[0], py = P[1], pz = P[2], ax = A[0], ay = A[1], az = A[2];
  const double bx = B[0], by = B[1], bz = B[2], cx = Cc[0], cy = Cc[1], cz = Cc[2];
  const double abx = bx - ax, aby = by - ay, abz = bz - az;
  const double acx = cx - ax, acy = cy - ay, acz = cz - az;
  const double apx = px - ax, apy = py - ay, apz = pz - az;
  const double d1 = abx * apx + aby * apy + abz * apz;
  const double d2 = acx * apx + acy * apy + acz * apz;
  if (d1 <= 0 && d2 <= 0) return pack_cp(0, 0, px - ax, py - ay, pz - az);
  const double bpx = px - bx, bpy = py - by, bpz = pz - bz;
  const double d3 = abx * bpx + aby * bpy + abz * bpz;
  const double d4 = acx * bpx + acy * bpy + acz * bpz;
  if (d3 >= 0 && d4 <= d3) return pack_cp(1, 0, px - bx, py - by, pz - bz);
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) {
    const double v = d1 / (d1 - d3);
    return pack_cp(v, 0, px - (ax + v * abx), py - (ay + v * aby), pz - (az + v * abz));
  }
  const double cpx = px - cx, cpy = py - cy, cpz = pz - cz;
  const double d5 = abx * cpx + aby * cpy + abz * cpz;
  const double d6 = acx * cpx + acy * cpy + acz * cpz;
  if (d6 >= 0 && d5 <= d6) return pack_cp(0, 1, px - cx, py - cy, pz - cz);
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    const double w = d2 / (d2 - d6);
    return pack_cp(0, w, px - (ax + w * acx), py - (ay + w * acy), pz - (az + w * acz));
  }
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0 && d4 - d3 >= 0 && d5 - d6 >= 0) {
    const double w = (d4 - d3) / (d4 - d3 + (d5 - d6));
    const double qx = bx + w * (cx - bx), qy = by + w * (cy - by), qz = bz + w * (cz - bz);
    return pack_cp(1 - w, w, px - qx, py - qy, pz - qz);
  }
  const double denom = 1 / (va + vb + vc);
  const double v = vb * denom;
  const double w = vc * denom;
  const double qx = ax + abx * v + acx * w;
  const double qy = ay + aby * v + acy * w;
  const double qz = az + abz * v + acz * w;
  return pack_cp(v, w, px - qx, py - qy, pz - qz);
}

CSHD double clamp_lh(double v, double lo, double hi) { return v < lo ? lo : v > hi ? hi : v; }

// Segment ab vs segment cd; s on ab, t on cd.
CSHD Closest closest_ee(const double* A, const double* B, const double* Cc, const double* D) {
  const double ax = A[0], ay = A[1], az = A[2], bx = B[0], by = B[1], bz = B[2];
  const double cx = Cc[0], cy = Cc[1], cz = Cc[2], dx = D[0], dy = D[1], dz = D[2];
  const double d1x = bx - ax, d1y = by - ay, d1z = bz - az;
  const double d2x = dx - cx, d2y = dy - cy, d2z = dz - cz;
  const double rx = ax - cx, ry = ay - cy, rz = az - cz;
  const double a = d1x * d1x + d1y * d1y + d1z * d1z;
  const double e = d2x * d2x + d2y * d2y + d2z * d2z;
  const double f = d2x * rx + d2y * ry + d2z * rz;
  double s, t;
  if (a <= 1e-30 && e <= 1e-30) {
    s = 0; t = 0;
  } else if (a <= 1e-30) {
    s = 0; t = clamp_lh(f / e, 0, 1);
  } else {
    const double c = d1x * rx + d1y * ry + d1z * rz;
    if (e <= 1e-30) {
      t = 0; s = clamp_lh(-c / a, 0, 1);
    } else {
      const double b = d1x * d2x + d1y * d2y + d1z * d2z;
      const double denom = a * e - b * b;
      s = denom > 1e-30 ? clamp_lh((b * f - c * e) / denom, 0, 1) : 0;
      t = (b * s + f) / e;
      if (t < 0) { t = 0; s = clamp_lh(-c / a, 0, 1); }
      else if (t > 1) { t = 1; s = clamp_lh((b - c) / a, 0, 1); }
    }
  }
  const double axp = ax + d1x * s, ayp = ay + d1y * s, azp = az + d1z * s;
  const double cxp = cx + d2x * t, cyp = cy + d2y * t, czp = cz + d2z * t;
  return pack_cp(s, t, axp - cxp, ayp - cyp, azp - czp);
}

// Roots of a3 t^3 + a2 t^2 + a1 t + a0 in [0, 1], sorted, deduplicated (at most 3).
CSHD int solve_quadratic01(double a2, double a1, double a0, double* out) {
  const double eps = 1e-12;
  if (fabs(a2) < eps) {
    if (fabs(a1) < eps) return 0;
    const double r = -a0 / a1;
    if (r >= 0 && r <= 1) { out[0] = r; return 1; }
    return 0;
  }
  const double disc = a1 * a1 - 4 * a2 * a0;
  if (disc < 0) return 0;
  const double sd = sqrt(disc);
  const double r0 = (-a1 - sd) / (2 * a2), r1 = (-a1 + sd) / (2 * a2);
  int k = 0;
  if (r0 >= 0 && r0 <= 1) out[k++] = r0;
  if (r1 >= 0 && r1 <= 1) out[k++] = r1;
  if (k == 2 && out[1] < out[0]) { const double t = out[0]; out[0] = out[1]; out[1] = t; }
  return k;
}

CSHD int solve_cubic01(double a3, double a2, double a1, double a0, double* out) {
  const double eps = 1e-12;
  if (fabs(a3) < eps) return solve_quadratic01(a2, a1, a0, out);
  const double A = a2 / a3, B = a1 / a3, C = a0 / a3;
  const double sqA = A * A;
  const double p = (3 * B - sqA) / 3;
  const double q = (2 * sqA * A - 9 * A * B + 27 * C) / 27;
  double roots[3];
  int nr = 0;
  const double disc = (q * q) / 4 + (p * p * p) / 27;
  const double shift = A / 3;
  if (disc > eps) {
    const double sd = sqrt(disc);
    const double u = js_cbrt(-q / 2 + sd);
    const double v = js_cbrt(-q / 2 - sd);
    roots[nr++] = u + v - shift;
  } else if (fabs(disc) <= eps) {
    const double u = js_cbrt(-q / 2);
    roots[nr++] = 2 * u - shift;
    roots[nr++] = -u - shift;
  } else {
    const double r = sqrt(-(p * p * p) / 27);
    const double phi = js_acos(js_min(1.0, js_max(-1.0, -q / (2 * r))));
    const double s = 2 * js_cbrt(r);
    const double PI = 3.141592653589793;
    roots[nr++] = s * cos(phi / 3) - shift;
    roots[nr++] = s * cos((phi + 2 * PI) / 3) - shift;
    roots[nr++] = s * cos((phi + 4 * PI) / 3) - shift;
  }
  double kept[3];
  int nk = 0;
  for (int i = 0; i < nr; i++) {
    double r = roots[i];
    if (!isfinite(r)) continue;
    for (int k = 0; k < 4; k++) {
      const double f = ((a3 * r + a2) * r + a1) * r + a0;
      const double df = (3 * a3 * r + 2 * a2) * r + a1;
      if (fabs(df) < 1e-18) break;
      r -= f / df;
    }
    if (r >= -1e-9 && r <= 1 + 1e-9) kept[nk++] = js_min(1.0, js_max(0.0, r));
  }
  // insertion sort (<= 3 values), then drop values within 1e-9 of their sorted predecessor
  for (int i = 1; i < nk; i++)
    for (int j = i; j > 0 && kept[j] < kept[j - 1]; j--) {
      const double t = kept[j]; kept[j] = kept[j - 1]; kept[j - 1] = t;
    }
  int no = 0;
  for (int i = 0; i < nk; i++)
    if (i == 0 || kept[i] - kept[i - 1] > 1e-9) out[no++] = kept[i];
  return no;
}

CSHD void cross3(double* o, const double* u, const double* v) {
  o[0] = u[1] * v[2] - u[2] * v[1];
  o[1] = u[2] * v[0] - u[0] * v[2];
  o[2] = u[0] * v[1] - u[1] * v[0];
}
CSHD double dot3(const double* u, const double* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; }

// Largest per-axis deviation of the stencil's motion from its mean motion.
CSHD double stencil_dev(const double* P0, const double* P1) {
  double mx = 0, my = 0, mz = 0;
  for (int v = 0; v < 4; v++) {
    mx += P1[v * 3] - P0[v * 3];
    my += P1[v * 3 + 1] - P0[v * 3 + 1];
    mz += P1[v * 3 + 2] - P0[v * 3 + 2];
  }
  mx /= 4; my /= 4; mz /= 4;
  double dev = 0;
  for (int v = 0; v < 4; v++) {
    const double dx = P1[v * 3] - P0[v * 3] - mx;
    const double dy = P1[v * 3 + 1] - P0[v * 3 + 1] - my;
    const double dz = P1[v * 3 + 2] - P0[v * 3 + 2] - mz;
    const double m = js_max(js_max(fabs(dx), fabs(dy)), fabs(dz));
    if (m > dev) dev = m;
  }
  return dev;
}

// Largest Euclidean motion of a stencil vertex relative to the stencil's mean
// motion. Every point of either primitive (VT or EE) is a convex combination of
// its vertices, so the gap vector between two such points changes by at most
// twice this between P0 and P1: the distance at P0 is at least the distance at
// P1 minus twice this.
CSHD double stencil_rel_motion(const double* P0, const double* P1) {
  double mx = 0, my = 0, mz = 0;
  for (int v = 0; v < 4; v++) {
    mx += P1[v * 3] - P0[v * 3];
    my += P1[v * 3 + 1] - P0[v * 3 + 1];
    mz += P1[v * 3 + 2] - P0[v * 3 + 2];
  }
  mx /= 4; my /= 4; mz /= 4;
  double e = 0;
  for (int v = 0; v < 4; v++) {
    const double dx = P1[v * 3] - P0[v * 3] - mx;
    const double dy = P1[v * 3 + 1] - P0[v * 3 + 1] - my;
    const double dz = P1[v * 3 + 2] - P0[v * 3 + 2] - mz;
    e = js_max(e, sqrt(dx * dx + dy * dy + dz * dz));
  }
  return e;
}

// Sweep bound for the CCD: with d0, d1 the distances at the ends of the
// segment and E = stencil_rel_motion, the distance at time t is at least
// max(d0 - 2 E t, d1 - 2 E (1 - t)) >= (d0 + d1) / 2 - E. When that exceeds the
// thickness, no root and no sample of the CCD below can come within it, so the
// CCD returns +inf; the 1e-6 relative margin covers the rounding of the
// computed distances and sample positions. d1 = NaN disables the test.
CSHD bool sweep_clear(double d0, double d1, double E, double thickness) {
  return (d0 + d1) / 2 - E > thickness * (1 + 1e-6);
}

// Earliest time of impact in [0,1] of vertex p against triangle abc moving
// linearly P0 -> P1 (stencil order p, a, b, c), or +inf when safe. d1 and E
// (the distance at P1 and stencil_rel_motion) feed sweep_clear, which returns
// the same +inf sooner.
CSHD double vt_ccd(const double* P0, const double* P1, double thickness, double d1 = NAN, double E = 0) {
  const double* p0 = P0; const double* a0 = P0 + 3; const double* b0 = P0 + 6; const double* c0 = P0 + 9;
  const double d0 = closest_vt(p0, a0, b0, c0).dist;
  if (d0 <= thickness) return 0;
  const double dev = stencil_dev(P0, P1);
  if (d0 - 4 * dev > thickness) return INFINITY;
  if (sweep_clear(d0, d1, E, thickness)) return INFINITY;
  double dp[3], da[3], db[3], dc[3];
  for (int i = 0; i < 3; i++) {
    dp[i] = P1[i] - P0[i]; da[i] = P1[3 + i] - P0[3 + i];
    db[i] = P1[6 + i] - P0[6 + i]; dc[i] = P1[9 + i] - P0[9 + i];
  }
  double u0[3], du[3], v0[3], dv[3], w0[3], dw[3];
  for (int i = 0; i < 3; i++) {
    u0[i] = p0[i] - a0[i]; du[i] = dp[i] - da[i];
    v0[i] = b0[i] - a0[i]; dv[i] = db[i] - da[i];
    w0[i] = c0[i] - a0[i]; dw[i] = dc[i] - da[i];
  }
  double n0[3], n1[3], n2[3], t1[3], t2[3];
  cross3(n0, v0, w0);
  cross3(t1, v0, dw); cross3(t2, dv, w0);
  for (int i = 0; i < 3; i++) n1[i] = t1[i] + t2[i];
  cross3(n2, dv, dw);
  const double c0c = dot3(u0, n0);
  const double c1c = dot3(u0, n1) + dot3(du, n0);
  const double c2c = dot3(u0, n2) + dot3(du, n1);
  const double c3c = dot3(du, n2);
  double roots[3];
  const int nr = solve_cubic01(c3c, c2c, c1c, c0c, roots);
  double pp[3], aa[3], bb[3], cc[3];
  for (int k = 0; k < nr; k++) {
    const double t = roots[k];
    for (int i = 0; i < 3; i++) {
      pp[i] = p0[i] + dp[i] * t; aa[i] = a0[i] + da[i] * t;
      bb[i] = b0[i] + db[i] * t; cc[i] = c0[i] + dc[i] * t;
    }
    if (closest_vt(pp, aa, bb, cc).dist <= thickness) return t;
  }
  double minD = INFINITY, minT = 0;
  for (int k = 0; k <= 16; k++) {
    const double t = (double)k / 16;
    for (int i = 0; i < 3; i++) {
      pp[i] = p0[i] + dp[i] * t; aa[i] = a0[i] + da[i] * t;
      bb[i] = b0[i] + db[i] * t; cc[i] = c0[i] + dc[i] * t;
    }
    const double d = closest_vt(pp, aa, bb, cc).dist;
    if (d < minD) { minD = d; minT = t; }
  }
  if (minD <= thickness) return minT;
  return INFINITY;
}

CSHD Closest ee_at(const double* a0, const double* da, const double* b0, const double* db, const double* c0,
                   const double* dc, const double* d0, const double* dd, double t) {
  double A[3], B[3], C[3], D[3];
  for (int i = 0; i < 3; i++) {
    A[i] = a0[i] + da[i] * t; B[i] = b0[i] + db[i] * t;
    C[i] = c0[i] + dc[i] * t; D[i] = d0[i] + dd[i] * t;
  }
  return closest_ee(A, B, C, D);
}

// Edge ab vs edge cd (stencil order a, b, c, d); d1, E as for vt_ccd.
CSHD double ee_ccd(const double* P0, const double* P1, double thickness, double d1 = NAN, double E = 0) {
  const double* a0 = P0; const double* b0 = P0 + 3; const double* c0 = P0 + 6; const double* d0 = P0 + 9;
  double da[3], db[3], dc[3], dd[3];
  for (int i = 0; i < 3; i++) {
    da[i] = P1[i] - P0[i]; db[i] = P1[3 + i] - P0[3 + i];
    dc[i] = P1[6 + i] - P0[6 + i]; dd[i] = P1[9 + i] - P0[9 + i];
  }
  const double q0 = ee_at(a0, da, b0, db, c0, dc, d0, dd, 0).dist;
  if (q0 <= thickness) return 0;
  const double dev = stencil_dev(P0, P1);
  if (q0 - 4 * dev > thickness) return INFINITY;
  if (sweep_clear(q0, d1, E, thickness)) return INFINITY;
  double e10[3], de1[3], e20[3], de2[3], r0[3], dr[3];
  for (int i = 0; i < 3; i++) {
    e10[i] = b0[i] - a0[i]; de1[i] = db[i] - da[i];
    e20[i] = d0[i] - c0[i]; de2[i] = dd[i] - dc[i];
    r0[i] = c0[i] - a0[i]; dr[i] = dc[i] - da[i];
  }
  double n0[3], n1[3], n2[3], t1[3], t2[3];
  cross3(n0, e10, e20);
  cross3(t1, e10, de2); cross3(t2, de1, e20);
  for (int i = 0; i < 3; i++) n1[i] = t1[i] + t2[i];
  cross3(n2, de1, de2);
  const double c0c = dot3(r0, n0);
  const double c1c = dot3(r0, n1) + dot3(dr, n0);
  const double c2c = dot3(r0, n2) + dot3(dr, n1);
  const double c3c = dot3(dr, n2);
  double roots[3];
  const int nr = solve_cubic01(c3c, c2c, c1c, c0c, roots);
  for (int k = 0; k < nr; k++) {
    const Closest cp = ee_at(a0, da, b0, db, c0, dc, d0, dd, roots[k]);
    if (cp.dist <= thickness && cp.s >= -1e-6 && cp.s <= 1 + 1e-6 && cp.t >= -1e-6 && cp.t <= 1 + 1e-6)
      return roots[k];
  }
  double minD = INFINITY, minT = 0;
  for (int k = 0; k <= 16; k++) {
    const double t = (double)k / 16;
    const double d = ee_at(a0, da, b0, db, c0, dc, d0, dd, t).dist;
    if (d < minD) { minD = d; minT = t; }
  }
  if (minD <= thickness) return minT;
  return INFINITY;
}

// CCD of a trial candidate (kind 0 VT, 1 EE) whose distance at P1 is dT: equal
// to vt_ccd / ee_ccd. The step-start distance d0 >= dT - 2E, so the sweep bound
// (d0 + dT) / 2 - E is at least dT - 2E: when that clears the thickness, the
// CCD's +inf is known without its closest-point query at P0.
CSHD double trial_ccd(int kind, const double* P0, const double* P1, double dT, double thickness) {
  const double E = stencil_rel_motion(P0, P1);
  if (sweep_clear(dT - 2 * E, dT, E, thickness)) return INFINITY;
  return kind == 0 ? vt_ccd(P0, P1, thickness, dT, E) : ee_ccd(P0, P1, thickness, dT, E);
}

CSHD double barrier_value(double d, double dHat) {
  if (d >= dHat) return 0;
  const double dc = js_max(d, 1e-12);
  const double t = dc - dHat;
  return -t * t * js_log(dc / dHat);
}
CSHD double barrier_grad_scalar(double d, double dHat, double kappa, double w) {
  if (d >= dHat) return 0;
  const double dc = js_max(d, 1e-12);
  const double t = dc - dHat;
  const double db = -2 * t * js_log(dc / dHat) - (t * t) / dc;
  return kappa * w * db;
}
CSHD double barrier_normal_force(double d, double dHat, double kappa, double w) {
  return js_max(0.0, -barrier_grad_scalar(d, dHat, kappa, w));
}
// kappa * max(b''(d), 0) with b'' = -(2L + 4u/d - u^2/d^2), L = js_log(d/dHat), u = d - dHat.
CSHD double barrier_curvature(double d, double dHat, double kappa) {
  const double L = js_log(d / dHat);
  const double u = d - dHat;
  const double b2 = -(2 * L + (4 * u) / d - (u * u) / (d * d));
  return kappa * js_max(b2, 0.0);
}
CSHD void coulomb_force(const double* u, double nx, double ny, double nz, double lambdaN, double mu, double eps,
                        double* f) {
  const double vn = u[0] * nx + u[1] * ny + u[2] * nz;
  const double tx = u[0] - vn * nx, ty = u[1] - vn * ny, tz = u[2] - vn * nz;
  const double mag = sqrt(tx * tx + ty * ty + tz * tz + eps * eps);
  const double s = (mu * js_max(0.0, lambdaN)) / mag;
  f[0] = -s * tx; f[1] = -s * ty; f[2] = -s * tz;
}

}  // namespace cs
