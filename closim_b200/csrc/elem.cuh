// Per-element physics of the cloth step as device functions, templated on the
// arithmetic type. On the FP64 path (T = double, compiled with -fmad=false)
// every expression keeps the reference's operation order, so each element's
// result is bit-identical to the reference arithmetic:
//   membrane  src/physics/membrane.ts:17-80
//   hinge     src/physics/bending.ts:7-42, src/mesh/mesh.ts:129-140
//   HVP       src/physics/membrane-hvp.ts:18-75
//   9x9 block src/physics/membrane-blocks.ts:21-98
#pragma once
#include "common.cuh"
#include "jsmath.cuh"

namespace cs {

template <class T>
struct Mat {
  T C00, C11, C01, G, thickness;
};

// Orthotropic StVK membrane: energy, 9-gradient and the three Green strains.
template <class T>
__device__ __forceinline__ void tri_grad(const T* x0, const T* x1, const T* x2, T a, T b, T c, T d,
                                         T area, const Mat<T>& m, T& energy, T g[9], T E[3]) {
  const T e1x = x1[0] - x0[0], e1y = x1[1] - x0[1], e1z = x1[2] - x0[2];
  const T e2x = x2[0] - x0[0], e2y = x2[1] - x0[1], e2z = x2[2] - x0[2];
  const T F00 = a * e1x + c * e2x, F10 = a * e1y + c * e2y, F20 = a * e1z + c * e2z;
  const T F01 = b * e1x + d * e2x, F11 = b * e1y + d * e2y, F21 = b * e1z + d * e2z;
  const T C00 = F00 * F00 + F10 * F10 + F20 * F20;
  const T C11 = F01 * F01 + F11 * F11 + F21 * F21;
  const T C01 = F00 * F01 + F10 * F11 + F20 * F21;
  const T E00 = T(0.5) * (C00 - 1);
  const T E11 = T(0.5) * (C11 - 1);
  const T E01 = T(0.5) * C01;
  const T psi = T(0.5) * m.C00 * E00 * E00 + T(0.5) * m.C11 * E11 * E11 + m.C01 * E00 * E11 +
                T(2) * m.G * E01 * E01;
  energy = m.thickness * area * psi;
  const T S00 = m.C00 * E00 + m.C01 * E11;
  const T S11 = m.C11 * E11 + m.C01 * E00;
  const T S01 = T(2) * m.G * E01;
  const T Pi0[3] = {F00 * S00 + F01 * S01, F10 * S00 + F11 * S01, F20 * S00 + F21 * S01};
  const T Pi1[3] = {F00 * S01 + F01 * S11, F10 * S01 + F11 * S11, F20 * S01 + F21 * S11};
  const T s = m.thickness * area;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const T g1 = s * (Pi0[i] * a + Pi1[i] * b);
    const T g2 = s * (Pi0[i] * c + Pi1[i] * d);
    g[i] = -(g1 + g2);
    g[3 + i] = g1;
    g[6 + i] = g2;
  }
  E[0] = E00; E[1] = E11; E[2] = E01;
}

// Membrane energy only (the Armijo merit path).
template <class T>
__device__ __forceinline__ T tri_energy(const T* x0, const T* x1, const T* x2, T a, T b, T c, T d, T area,
                                        const Mat<T>& m) {
  const T e1x = x1[0] - x0[0], e1y = x1[1] - x0[1], e1z = x1[2] - x0[2];
  const T e2x = x2[0] - x0[0], e2y = x2[1] - x0[1], e2z = x2[2] - x0[2];
  const T F00 = a * e1x + c * e2x, F10 = a * e1y + c * e2y, F20 = a * e1z + c * e2z;
  const T F01 = b * e1x + d * e2x, F11 = b * e1y + d * e2y, F21 = b * e1z + d * e2z;
  const T C00 = F00 * F00 + F10 * F10 + F20 * F20;
  const T C11 = F01 * F01 + F11 * F11 + F21 * F21;
  const T C01 = F00 * F01 + F10 * F11 + F20 * F21;
  const T E00 = T(0.5) * (C00 - 1);
  const T E11 = T(0.5) * (C11 - 1);
  const T E01 = T(0.5) * C01;
  const T psi = T(0.5) * m.C00 * E00 * E00 + T(0.5) * m.C11 * E11 * E11 + m.C01 * E00 * E11 +
                T(2) * m.G * E01 * E01;
  return m.thickness * area * psi;
}

// Exact directional derivative of tri_grad along v (analytic HVP).
template <class T>
__device__ __forceinline__ void tri_hvp(const T* x0, const T* x1, const T* x2, const T* v0, const T* v1,
                                        const T* v2, T a, T b, T c, T d, T area, const Mat<T>& m, T out[9]) {
  const T e1x = x1[0] - x0[0], e1y = x1[1] - x0[1], e1z = x1[2] - x0[2];
  const T e2x = x2[0] - x0[0], e2y = x2[1] - x0[1], e2z = x2[2] - x0[2];
  const T w1x = v1[0] - v0[0], w1y = v1[1] - v0[1], w1z = v1[2] - v0[2];
  const T w2x = v2[0] - v0[0], w2y = v2[1] - v0[1], w2z = v2[2] - v0[2];
  const T F00 = a * e1x + c * e2x, F10 = a * e1y + c * e2y, F20 = a * e1z + c * e2z;
  const T F01 = b * e1x + d * e2x, F11 = b * e1y + d * e2y, F21 = b * e1z + d * e2z;
  const T dF00 = a * w1x + c * w2x, dF10 = a * w1y + c * w2y, dF20 = a * w1z + c * w2z;
  const T dF01 = b * w1x + d * w2x, dF11 = b * w1y + d * w2y, dF21 = b * w1z + d * w2z;
  const T E00 = T(0.5) * (F00 * F00 + F10 * F10 + F20 * F20 - 1);
  const T E11 = T(0.5) * (F01 * F01 + F11 * F11 + F21 * F21 - 1);
  const T E01 = T(0.5) * (F00 * F01 + F10 * F11 + F20 * F21);
  const T dC00 = T(2) * (F00 * dF00 + F10 * dF10 + F20 * dF20);
  const T dC11 = T(2) * (F01 * dF01 + F11 * dF11 + F21 * dF21);
  const T dC01 = dF00 * F01 + F00 * dF01 + dF10 * F11 + F10 * dF11 + dF20 * F21 + F20 * dF21;
  const T dE00 = T(0.5) * dC00, dE11 = T(0.5) * dC11, dE01 = T(0.5) * dC01;
  const T S00 = m.C00 * E00 + m.C01 * E11;
  const T S11 = m.C11 * E11 + m.C01 * E00;
  const T S01 = T(2) * m.G * E01;
  const T dS00 = m.C00 * dE00 + m.C01 * dE11;
  const T dS11 = m.C11 * dE11 + m.C01 * dE00;
  const T dS01 = T(2) * m.G * dE01;
  const T P[6] = {dF00 * S00 + F00 * dS00 + dF01 * S01 + F01 * dS01,
                  dF10 * S00 + F10 * dS00 + dF11 * S01 + F11 * dS01,
                  dF20 * S00 + F20 * dS00 + dF21 * S01 + F21 * dS01,
                  dF00 * S01 + F00 * dS01 + dF01 * S11 + F01 * dS11,
                  dF10 * S01 + F10 * dS01 + dF11 * S11 + F11 * dS11,
                  dF20 * S01 + F20 * dS01 + dF21 * S11 + F21 * dS11};
  const T s = m.thickness * area;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const T g1 = s * (P[i] * a + P[3 + i] * b);
    const T g2 = s * (P[i] * c + P[3 + i] * d);
    out[i] = -(g1 + g2);
    out[3 + i] = g1;
    out[6 + i] = g2;
  }
}

// Closed-form 9x9 membrane Hessian, same loop nest and accumulation order as
// the reference (zero terms skipped where it skips them).
// Rows [r0, r1) of the 9x9 block are written to h[(A - r0) * 9 + B].
template <class T>
__device__ void tri_hessian9_rows(const T* x0, const T* x1, const T* x2, T a, T b, T c, T d, T area,
                                  const Mat<T>& mt, int r0, int r1, T* h) {
  const T* X[3] = {x0, x1, x2};
  const T K[3][2] = {{-(a + c), -(b + d)}, {a, b}, {c, d}};
  T F[3][2] = {{0, 0}, {0, 0}, {0, 0}};
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int v = 0; v < 3; v++) F[i][j] += K[v][j] * X[v][i];
  T Cm[2][2] = {{0, 0}, {0, 0}};
#pragma unroll
  for (int l = 0; l < 2; l++)
#pragma unroll
    for (int mm = 0; mm < 2; mm++)
#pragma unroll
      for (int i = 0; i < 3; i++) Cm[l][mm] += F[i][l] * F[i][mm];
  const T E00 = T(0.5) * (Cm[0][0] - 1), E11 = T(0.5) * (Cm[1][1] - 1), E01 = T(0.5) * Cm[0][1];
  const T S00 = mt.C00 * E00 + mt.C01 * E11;
  const T S11 = mt.C11 * E11 + mt.C01 * E00;
  const T S01 = T(2) * mt.G * E01;
  const T S[2][2] = {{S00, S01}, {S01, S11}};
  // Voigt moduli D[k][j][l][m] (only these slots are non-zero).
  auto Dm = [&](int k, int j, int l, int m2) -> T {
    if (k == 0 && j == 0 && l == 0 && m2 == 0) return mt.C00;
    if (k == 1 && j == 1 && l == 1 && m2 == 1) return mt.C11;
    if ((k == 0 && j == 0 && l == 1 && m2 == 1) || (k == 1 && j == 1 && l == 0 && m2 == 0)) return mt.C01;
    if (k != j && l != m2) return mt.G;
    return T(0);
  };
  const T s = mt.thickness * area;
  // M[A][i][j] = (i == A % 3) ? K[A / 3][j] : 0
  for (int A = r0; A < r1; A++) {
    for (int B = 0; B < 9; B++) {
      T sum = 0;
      for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 2; j++) {
          const T mA = (i == A % 3) ? K[A / 3][j] : T(0);
          if (mA == 0) continue;
          T dP = 0;
          for (int k = 0; k < 2; k++) {
            const T mBik = (i == B % 3) ? K[B / 3][k] : T(0);
            dP += mBik * S[k][j];
            T dE = 0;
            for (int l = 0; l < 2; l++) {
              for (int m2 = 0; m2 < 2; m2++) {
                const T dd = Dm(k, j, l, m2);
                if (dd == 0) continue;
                T dElm = 0;
                for (int p = 0; p < 3; p++) {
                  const T mBpl = (p == B % 3) ? K[B / 3][l] : T(0);
                  const T mBpm = (p == B % 3) ? K[B / 3][m2] : T(0);
                  dElm += mBpl * F[p][m2] + F[p][l] * mBpm;
                }
                dE += dd * T(0.5) * dElm;
              }
            }
            dP += F[i][k] * dE;
          }
          sum += mA * dP;
        }
      }
      h[(A - r0) * 9 + B] = s * sum;
    }
  }
}

// Dihedral angle of triangles (p0,p1,p2) and (p0,p1,p3).
template <class T>
__device__ __forceinline__ T dihedral4(const T* q) {
  const T e0x = q[3] - q[0], e0y = q[4] - q[1], e0z = q[5] - q[2];
  const T e1x = q[6] - q[0], e1y = q[7] - q[1], e1z = q[8] - q[2];
  const T e2x = q[9] - q[0], e2y = q[10] - q[1], e2z = q[11] - q[2];
  const T n1x = e0y * e1z - e0z * e1y, n1y = e0z * e1x - e0x * e1z, n1z = e0x * e1y - e0y * e1x;
  const T n2x = e0y * e2z - e0z * e2y, n2y = e0z * e2x - e0x * e2z, n2z = e0x * e2y - e0y * e2x;
  const T l1 = js_hypot3(n1x, n1y, n1z) + T(1e-30);
  const T l2 = js_hypot3(n2x, n2y, n2z) + T(1e-30);
  const T cosT = js_min(T(1), js_max(T(-1), (n1x * n2x + n1y * n2y + n1z * n2z) / (l1 * l2)));
  if constexpr (sizeof(T) == 8) return js_acos(cosT);
  else return acosf(cosT);
}

// W = 0.5 k (theta - theta0)^2 edgeLen^2 / max(areaSum, 1e-12).
template <class T>
__device__ __forceinline__ T hinge_energy4(const T* q, T restAngle, T edgeLen, T areaSum, T k) {
  const T th = dihedral4(q);
  const T d = th - restAngle;
  const T w = edgeLen * edgeLen / js_max(areaSum, T(1e-12));
  return T(0.5) * k * d * d * w;
}

// Central-difference hinge gradient (eps 1e-7 over the 12 dofs, reference
// bending.ts:19-42). q holds the 4 vertices (v0..v3); out receives 12 values.
__device__ __forceinline__ void hinge_fd_grad(double* q, double restAngle, double edgeLen, double areaSum,
                                              double k, double out[12]) {
  const double eps = 1e-7;
  for (int a = 0; a < 12; a++) {
    const double old = q[a];
    q[a] = old + eps;
    const double ep = hinge_energy4(q, restAngle, edgeLen, areaSum, k);
    q[a] = old - eps;
    const double em = hinge_energy4(q, restAngle, edgeLen, areaSum, k);
    q[a] = old;
    out[a] = (ep - em) / (2 * eps);
  }
}

}  // namespace cs
