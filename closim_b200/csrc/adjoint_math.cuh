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

}  // namespace cs
