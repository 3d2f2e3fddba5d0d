// Element derivatives for the adjoint of the implicit step (no reference
// counterpart): the analytic gradient of the hinge bending energy and its
// exact directional derivative through dual numbers. Host and device.
//
// Bending energy (src/physics/bending.ts:7-16): W = 0.5 k (theta - theta0)^2 w,
// w = edgeLen^2 / max(areaSum, 1e-12), theta the angle between the normals
// n1 = e0 x e1 and n2 = e0 x e2 of the two triangles (v0, v1, v2), (v0, v1, v3)
// sharing edge e0 = x1 - x0 (src/mesh/mesh.ts:129-140). With the normals
// nA = e0 x e1 and nB = e2 x e0 = -n2, which agree on a flat hinge, the signed
// bend angle phi = atan2((nA x nB) . e0/|e0|, nA . nB) gives theta = pi - |phi|
// and W = 0.5 k w (pi - |phi| - theta0)^2. A flat rest hinge (theta0 = pi) makes
// W = 0.5 k w phi^2, smooth at phi = 0 where acos is not differentiable.
//
// d phi / dx follows the standard dihedral-angle gradient: with unit normals
// nA, nB, heights hA = |nA|/|e0|, hB = |nB|/|e0| of the wing vertices over the
// edge and their projections tA = e1.e0/|e0|^2, tB = e2.e0/|e0|^2,
//   d phi/dx2 = -nA / hA,   d phi/dx3 = -nB / hB,
//   d phi/dx0 = (1 - tA) nA/hA + (1 - tB) nB/hB,   d phi/dx1 = tA nA/hA + tB nB/hB
// (the four sum to zero: the angle is translation invariant).
#pragma once
#include <math.h>

#ifndef CSHD
#define CSHD __host__ __device__ __forceinline__
#endif

namespace cs {

// Forward-mode dual number: v + d eps, eps^2 = 0.
struct Dual {
  double v, d;
  CSHD Dual() : v(0), d(0) {}
  CSHD Dual(double a) : v(a), d(0) {}
  CSHD Dual(double a, double b) : v(a), d(b) {}
};
CSHD Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
CSHD Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
CSHD Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
CSHD Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
CSHD Dual operator/(Dual a, Dual b) { return Dual(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)); }
CSHD Dual dsqrt(Dual a) {
  const double s = sqrt(a.v);
  return Dual(s, s > 0 ? a.d / (2 * s) : 0.0);
}
CSHD Dual datan2(Dual y, Dual x) {
  const double r2 = x.v * x.v + y.v * y.v;
  return Dual(atan2(y.v, x.v), r2 > 0 ? (x.v * y.d - y.v * x.d) / r2 : 0.0);
}
CSHD double dval(double a) { return a; }
CSHD double dval(Dual a) { return a.v; }
CSHD double dsqrt(double a) { return sqrt(a); }
CSHD double datan2(double y, double x) { return atan2(y, x); }

template <class T>
CSHD void dcross(const T* a, const T* b, T* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
template <class T>
CSHD T ddot(const T* a, const T* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

constexpr double kPi = 3.14159265358979323846;

// Signed bend angle and its gradient over the 12 coordinates of (v0, v1, v2, v3).
template <class T>
CSHD T bend_angle_grad(const T* q, T* dphi) {
  T e0[3], e1[3], e2[3];
  for (int k = 0; k < 3; k++) {
    e0[k] = q[3 + k] - q[k];
    e1[k] = q[6 + k] - q[k];
    e2[k] = q[9 + k] - q[k];
  }
  T nA[3], nB[3], c[3];
  dcross(e0, e1, nA);
  dcross(e2, e0, nB);
  const T l2 = ddot(e0, e0);
  const T len = dsqrt(l2);
  dcross(nA, nB, c);
  const T phi = datan2(ddot(c, e0) / len, ddot(nA, nB));
  const T aA = ddot(nA, nA), aB = ddot(nB, nB);
  const T tA = ddot(e1, e0) / l2, tB = ddot(e2, e0) / l2;
  // n/h = (n/|n|) / (|n|/|e0|) = n |e0| / |n|^2
  for (int k = 0; k < 3; k++) {
    const T gA = nA[k] * len / aA, gB = nB[k] * len / aB;
    dphi[6 + k] = -gA;
    dphi[9 + k] = -gB;
    dphi[k] = (T(1.0) - tA) * gA + (T(1.0) - tB) * gB;
    dphi[3 + k] = tA * gA + tB * gB;
  }
  return phi;
}

// Analytic gradient of the hinge energy (12 values); returns the energy.
template <class T>
CSHD T bend_grad(const T* q, double restAngle, double edgeLen, double areaSum, double k, T* g) {
  T dphi[12];
  const T phi = bend_angle_grad(q, dphi);
  const double w = edgeLen * edgeLen / (areaSum > 1e-12 ? areaSum : 1e-12);
  const double flatOff = kPi - restAngle;  // bend angle of the rest shape
  // W = 0.5 k w (|phi| - flatOff)^2; a rest shape flat to 1e-6 rad is taken as flat
  const double sgn = dval(phi) >= 0 ? 1.0 : -1.0;
  const T dev = flatOff < 1e-6 ? phi : T(sgn) * phi - T(flatOff);
  const T coef = T(k * w) * dev * (flatOff < 1e-6 ? T(1.0) : T(sgn));
  for (int a = 0; a < 12; a++) g[a] = coef * dphi[a];
  return T(0.5 * k * w) * dev * dev;
}

// Directional derivative of the bending gradient along v: H_bend v (12 values).
CSHD void bend_hvp(const double* q, const double* v, double restAngle, double edgeLen, double areaSum, double k,
                   double* out) {
  Dual qd[12], g[12];
  for (int a = 0; a < 12; a++) qd[a] = Dual(q[a], v[a]);
  bend_grad<Dual>(qd, restAngle, edgeLen, areaSum, k, g);
  for (int a = 0; a < 12; a++) out[a] = g[a].d;
}

// Gauss-Newton factor of one hinge: g = sqrt(k w) d phi / dx (12 values), so
// that g g^T is the positive semi-definite part k w (d phi)(d phi)^T of the
// bending Hessian (the term k w dev d^2 phi, small near the rest angle, is
// dropped). The exact-Newton mode of the mixed path applies it as g (g . v).
CSHD void bend_gn(const double* q, double edgeLen, double areaSum, double k, double* g) {
  double dphi[12];
  bend_angle_grad<double>(q, dphi);
  const double w = edgeLen * edgeLen / (areaSum > 1e-12 ? areaSum : 1e-12);
  const double r = sqrt(k * w);
  for (int a = 0; a < 12; a++) g[a] = r * dphi[a];
}

// Positive part of the symmetric 2x2 second Piola stress (S00, S11, S01):
// negative principal stresses are set to zero. Used in the geometric term of
// the membrane Hessian (dF S) it makes every element block positive
// semi-definite: a Newton matrix for the forward solve that leaves its
// converged solution unchanged.
CSHD void psd_stress(double& S00, double& S11, double& S01) {
  const double hm = 0.5 * (S00 + S11), hd = 0.5 * (S00 - S11);
  const double rad = sqrt(hd * hd + S01 * S01);
  const double l1 = hm + rad, l2 = hm - rad;
  if (l2 >= 0) return;
  if (l1 <= 0) {
    S00 = S11 = S01 = 0;
    return;
  }
  // S+ = l1 u u^T, u the unit eigenvector of l1
  double ux = S01, uy = l1 - S00;
  if (ux * ux + uy * uy < 1e-300) { ux = l1 - S11; uy = S01; }
  const double nn = ux * ux + uy * uy;
  if (nn < 1e-300) { ux = S00 >= S11 ? 1 : 0; uy = 1 - ux; }
  else { const double q = 1 / sqrt(nn); ux *= q; uy *= q; }
  S00 = l1 * ux * ux;
  S11 = l1 * uy * uy;
  S01 = l1 * ux * uy;
}

// Closed-form 9x9 membrane Hessian block of one triangle (the derivative of
// membrane.ts:17-80's gradient), for the mixed path's Schwarz assembly:
//   H_ab = s [ (K_a . S K_b) I3 + sum_{k,m} alpha_km F_k F_m^T ],
//   alpha_00 = C00 Ka0 Kb0 + G Ka1 Kb1,   alpha_01 = C01 Ka0 Kb1 + G Ka1 Kb0,
//   alpha_10 = C01 Ka1 Kb0 + G Ka0 Kb1,   alpha_11 = C11 Ka1 Kb1 + G Ka0 Kb0,
// with F_k the columns of F, K_0 = -(a + c, b + d), K_1 = (a, b), K_2 = (c, d)
// (the rows of the shape-function gradient) and s = thickness * area. Row-major
// h[(3a + i) * 9 + 3b + p], stored as O (double, or float for the FP32 path).
// psd: S replaced by its positive part (psd_stress).
template <class O>
CSHD void membrane_block9(const double* x0, const double* x1, const double* x2, double a, double b, double c,
                          double d, double s, double C00, double C11, double C01, double G, O* h,
                          bool psd = false) {
  const double K[3][2] = {{-(a + c), -(b + d)}, {a, b}, {c, d}};
  double F0[3], F1[3];
  for (int i = 0; i < 3; i++) {
    const double e1 = x1[i] - x0[i], e2 = x2[i] - x0[i];
    F0[i] = a * e1 + c * e2;
    F1[i] = b * e1 + d * e2;
  }
  const double E00 = 0.5 * (F0[0] * F0[0] + F0[1] * F0[1] + F0[2] * F0[2] - 1);
  const double E11 = 0.5 * (F1[0] * F1[0] + F1[1] * F1[1] + F1[2] * F1[2] - 1);
  const double E01 = 0.5 * (F0[0] * F1[0] + F0[1] * F1[1] + F0[2] * F1[2]);
  double S00 = C00 * E00 + C01 * E11, S11 = C11 * E11 + C01 * E00, S01 = 2 * G * E01;
  if (psd) psd_stress(S00, S11, S01);  // geometric term only (the material term has no S)
  for (int A = 0; A < 3; A++)
    for (int B = 0; B < 3; B++) {
      const double ka0 = K[A][0], ka1 = K[A][1], kb0 = K[B][0], kb1 = K[B][1];
      const double geo = ka0 * (S00 * kb0 + S01 * kb1) + ka1 * (S01 * kb0 + S11 * kb1);
      const double a00 = C00 * ka0 * kb0 + G * ka1 * kb1, a01 = C01 * ka0 * kb1 + G * ka1 * kb0;
      const double a10 = C01 * ka1 * kb0 + G * ka0 * kb1, a11 = C11 * ka1 * kb1 + G * ka0 * kb0;
      for (int i = 0; i < 3; i++)
        for (int p = 0; p < 3; p++) {
          const double v = (i == p ? geo : 0.0) + a00 * F0[i] * F0[p] + a01 * F0[i] * F1[p] + a10 * F1[i] * F0[p] +
                           a11 * F1[i] * F1[p];
          h[(3 * A + i) * 9 + 3 * B + p] = (O)(s * v);
        }
    }
}

}  // namespace cs
