// Oracle (test infrastructure only): mesh preprocessing, element physics and
// preconditioners, restated from the reference TypeScript.
#include <algorithm>
#include <array>
#include <functional>
#include <deque>
#include <map>
#include <set>
#include <stdexcept>
#include <unordered_map>

#include "orc.hpp"
#include "jsmath.hpp"

namespace orc {

// src/mesh/mesh.ts:17-48 buildGrid: XZ plane, y = 0; triangles (a,c,b),(b,c,d).
void build_grid(int nx, int ny, double w, double h, std::vector<float>& pos,
                std::vector<float>& uv, std::vector<uint32_t>& idx) {
  int n = (nx + 1) * (ny + 1);
  pos.assign(n * 3, 0.f);
  uv.assign(n * 2, 0.f);
  for (int j = 0; j <= ny; j++) {
    for (int i = 0; i <= nx; i++) {
      int id = j * (nx + 1) + i;
      double x = ((double)i / nx) * w;
      double z = ((double)j / ny) * h;
      pos[id * 3] = fr(x);
      pos[id * 3 + 1] = 0.f;
      pos[id * 3 + 2] = fr(z);
      uv[id * 2] = fr(x);
      uv[id * 2 + 1] = fr(z);
    }
  }
  idx.clear();
  for (int j = 0; j < ny; j++) {
    for (int i = 0; i < nx; i++) {
      uint32_t a = j * (nx + 1) + i, b = a + 1, c = a + (nx + 1), d = c + 1;
      uint32_t t[6] = {a, c, b, b, c, d};
      idx.insert(idx.end(), t, t + 6);
    }
  }
}

// src/mesh/mesh.ts:129-140 dihedral (acos of the clamped normal cosine).
template <class T>
double dihedral(const T* x, int v0, int v1, int v2, int v3) {
  double e0x = (double)x[v1 * 3] - (double)x[v0 * 3], e0y = (double)x[v1 * 3 + 1] - (double)x[v0 * 3 + 1],
         e0z = (double)x[v1 * 3 + 2] - (double)x[v0 * 3 + 2];
  double e1x = (double)x[v2 * 3] - (double)x[v0 * 3], e1y = (double)x[v2 * 3 + 1] - (double)x[v0 * 3 + 1],
         e1z = (double)x[v2 * 3 + 2] - (double)x[v0 * 3 + 2];
  double e2x = (double)x[v3 * 3] - (double)x[v0 * 3], e2y = (double)x[v3 * 3 + 1] - (double)x[v0 * 3 + 1],
         e2z = (double)x[v3 * 3 + 2] - (double)x[v0 * 3 + 2];
  double n1x = e0y * e1z - e0z * e1y, n1y = e0z * e1x - e0x * e1z, n1z = e0x * e1y - e0y * e1x;
  double n2x = e0y * e2z - e0z * e2y, n2y = e0z * e2x - e0x * e2z, n2z = e0x * e2y - e0y * e2x;
  double l1 = js_hypot3(n1x, n1y, n1z) + 1e-30;
  double l2 = js_hypot3(n2x, n2y, n2z) + 1e-30;
  double cosT = js_min(1, js_max(-1, (n1x * n2x + n1y * n2y + n1z * n2z) / (l1 * l2)));
  return js_acos(cosT);
}
template double dihedral<float>(const float*, int, int, int, int);
template double dihedral<double>(const double*, int, int, int, int);

// src/mesh/mesh.ts:99-126 buildHinges: edges in first-seen order (JS Map).
static std::vector<Hinge> build_hinges(const std::vector<uint32_t>& idx, const std::vector<float>& pos,
                                       const std::vector<float>& areas) {
  int m = (int)idx.size() / 3;
  struct Ent { int tri, a, b, opp; };
  std::unordered_map<uint64_t, int> slot;
  std::vector<std::vector<Ent>> lists;
  slot.reserve(m * 2);
  for (int t = 0; t < m; t++) {
    int ids[3] = {(int)idx[t * 3], (int)idx[t * 3 + 1], (int)idx[t * 3 + 2]};
    for (int e = 0; e < 3; e++) {
      int a = ids[e], b = ids[(e + 1) % 3], opp = ids[(e + 2) % 3];
      uint64_t k = a < b ? ((uint64_t)a << 32 | (uint32_t)b) : ((uint64_t)b << 32 | (uint32_t)a);
      auto it = slot.find(k);
      if (it == slot.end()) {
        slot.emplace(k, (int)lists.size());
        lists.push_back({});
        lists.back().push_back({t, a, b, opp});
      } else {
        lists[it->second].push_back({t, a, b, opp});
      }
    }
  }
  std::vector<Hinge> hinges;
  for (auto& list : lists) {
    if (list.size() != 2) continue;
    const Ent& e0 = list[0];
    const Ent& e1 = list[1];
    Hinge hg;
    hg.v0 = e0.a; hg.v1 = e0.b; hg.v2 = e0.opp; hg.v3 = e1.opp;
    hg.restAngle = dihedral(pos.data(), hg.v0, hg.v1, hg.v2, hg.v3);
    double ax = (double)pos[hg.v0 * 3] - (double)pos[hg.v1 * 3];
    double ay = (double)pos[hg.v0 * 3 + 1] - (double)pos[hg.v1 * 3 + 1];
    double az = (double)pos[hg.v0 * 3 + 2] - (double)pos[hg.v1 * 3 + 2];
    hg.edgeLen = js_hypot3(ax, ay, az);
    hg.areaSum = (double)areas[e0.tri] + (double)areas[e1.tri];
    hinges.push_back(hg);
  }
  return hinges;
}

// src/mesh/mesh.ts:50-97 preprocess: Dm^-1, areas, lumped masses, all Float32.
Mesh preprocess(const std::vector<float>& pos, const std::vector<float>& uv,
                const std::vector<uint32_t>& idx, double arealDensity) {
  Mesh me;
  me.n = (int)pos.size() / 3;
  me.m = (int)idx.size() / 3;
  me.invDm.assign(me.m * 4, 0.f);
  me.areas.assign(me.m, 0.f);
  me.masses.assign(me.n, 0.f);
  for (int t = 0; t < me.m; t++) {
    uint32_t i0 = idx[t * 3], i1 = idx[t * 3 + 1], i2 = idx[t * 3 + 2];
    double u0 = uv[i0 * 2], v0 = uv[i0 * 2 + 1];
    double u1 = uv[i1 * 2], v1 = uv[i1 * 2 + 1];
    double u2 = uv[i2 * 2], v2 = uv[i2 * 2 + 1];
    double du1 = u1 - u0, dv1 = v1 - v0;
    double du2 = u2 - u0, dv2 = v2 - v0;
    double det = du1 * dv2 - du2 * dv1;
    if (std::fabs(det) < 1e-12) throw std::runtime_error("degenerate triangle");
    double area = 0.5 * std::fabs(det);
    me.areas[t] = fr(area);
    me.invDm[t * 4] = fr(dv2 / det);
    me.invDm[t * 4 + 1] = fr(-du2 / det);
    me.invDm[t * 4 + 2] = fr(-dv1 / det);
    me.invDm[t * 4 + 3] = fr(du1 / det);
    // `area` here is the f64 value; the reference reads `area` (the local), not areas[t].
    double tm = arealDensity * area / 3;
    me.masses[i0] = fr((double)me.masses[i0] + tm);
    me.masses[i1] = fr((double)me.masses[i1] + tm);
    me.masses[i2] = fr((double)me.masses[i2] + tm);
  }
  me.hinges = build_hinges(idx, pos, me.areas);
  me.positions = pos;
  me.rest = pos;
  me.uv = uv;
  me.idx = idx;
  return me;
}

// src/physics/membrane.ts:17-80 triangleEnergyGradient.
void tri_energy_grad(const double* x0, const double* x1, const double* x2, const double* inv,
                     double area, const Material& mat, TriGrad& out) {
  const double a = inv[0], b = inv[1], c = inv[2], d = inv[3];
  const double e1x = x1[0] - x0[0], e1y = x1[1] - x0[1], e1z = x1[2] - x0[2];
  const double e2x = x2[0] - x0[0], e2y = x2[1] - x0[1], e2z = x2[2] - x0[2];
  const double F00 = a * e1x + c * e2x, F10 = a * e1y + c * e2y, F20 = a * e1z + c * e2z;
  const double F01 = b * e1x + d * e2x, F11 = b * e1y + d * e2y, F21 = b * e1z + d * e2z;
  const double C00 = F00 * F00 + F10 * F10 + F20 * F20;
  const double C11 = F01 * F01 + F11 * F11 + F21 * F21;
  const double C01 = F00 * F01 + F10 * F11 + F20 * F21;
  const double E00 = 0.5 * (C00 - 1);
  const double E11 = 0.5 * (C11 - 1);
  const double E01 = 0.5 * C01;
  const double C00k = mat.C00, C11k = mat.C11, C01k = mat.C01, G = mat.G;
  const double psi = 0.5 * C00k * E00 * E00 + 0.5 * C11k * E11 * E11 + C01k * E00 * E11 + 2 * G * E01 * E01;
  out.energy = mat.thickness * area * psi;
  const double S00 = C00k * E00 + C01k * E11;
  const double S11 = C11k * E11 + C01k * E00;
  const double S01 = 2 * G * E01;
  const double P00 = F00 * S00 + F01 * S01;
  const double P10 = F10 * S00 + F11 * S01;
  const double P20 = F20 * S00 + F21 * S01;
  const double P01 = F00 * S01 + F01 * S11;
  const double P11 = F10 * S01 + F11 * S11;
  const double P21 = F20 * S01 + F21 * S11;
  const double s = mat.thickness * area;
  const double Pi0[3] = {P00, P10, P20}, Pi1[3] = {P01, P11, P21};
  for (int i = 0; i < 3; i++) {
    const double g1 = s * (Pi0[i] * a + Pi1[i] * b);
    const double g2 = s * (Pi0[i] * c + Pi1[i] * d);
    const double g0 = -(g1 + g2);
    out.grad[i] = g0;
    out.grad[3 + i] = g1;
    out.grad[6 + i] = g2;
  }
  out.E00 = E00; out.E11 = E11; out.E01 = E01;
}

// src/physics/membrane-hvp.ts:18-75 triangleHvp.
void tri_hvp(const double* x0, const double* x1, const double* x2, const double* v0,
             const double* v1, const double* v2, const double* inv, double area,
             const Material& mat, double out[9]) {
  const double a = inv[0], b = inv[1], c = inv[2], d = inv[3];
  const double e1x = x1[0] - x0[0], e1y = x1[1] - x0[1], e1z = x1[2] - x0[2];
  const double e2x = x2[0] - x0[0], e2y = x2[1] - x0[1], e2z = x2[2] - x0[2];
  const double w1x = v1[0] - v0[0], w1y = v1[1] - v0[1], w1z = v1[2] - v0[2];
  const double w2x = v2[0] - v0[0], w2y = v2[1] - v0[1], w2z = v2[2] - v0[2];
  const double F00 = a * e1x + c * e2x, F10 = a * e1y + c * e2y, F20 = a * e1z + c * e2z;
  const double F01 = b * e1x + d * e2x, F11 = b * e1y + d * e2y, F21 = b * e1z + d * e2z;
  const double dF00 = a * w1x + c * w2x, dF10 = a * w1y + c * w2y, dF20 = a * w1z + c * w2z;
  const double dF01 = b * w1x + d * w2x, dF11 = b * w1y + d * w2y, dF21 = b * w1z + d * w2z;
  const double C00k = mat.C00, C11k = mat.C11, C01k = mat.C01, G = mat.G;
  const double E00 = 0.5 * (F00 * F00 + F10 * F10 + F20 * F20 - 1);
  const double E11 = 0.5 * (F01 * F01 + F11 * F11 + F21 * F21 - 1);
  const double E01 = 0.5 * (F00 * F01 + F10 * F11 + F20 * F21);
  const double dC00 = 2 * (F00 * dF00 + F10 * dF10 + F20 * dF20);
  const double dC11 = 2 * (F01 * dF01 + F11 * dF11 + F21 * dF21);
  const double dC01 = dF00 * F01 + F00 * dF01 + dF10 * F11 + F10 * dF11 + dF20 * F21 + F20 * dF21;
  const double dE00 = 0.5 * dC00, dE11 = 0.5 * dC11, dE01 = 0.5 * dC01;
  const double S00 = C00k * E00 + C01k * E11;
  const double S11 = C11k * E11 + C01k * E00;
  const double S01 = 2 * G * E01;
  const double dS00 = C00k * dE00 + C01k * dE11;
  const double dS11 = C11k * dE11 + C01k * dE00;
  const double dS01 = 2 * G * dE01;
  const double dP00 = dF00 * S00 + F00 * dS00 + dF01 * S01 + F01 * dS01;
  const double dP10 = dF10 * S00 + F10 * dS00 + dF11 * S01 + F11 * dS01;
  const double dP20 = dF20 * S00 + F20 * dS00 + dF21 * S01 + F21 * dS01;
  const double dP01 = dF00 * S01 + F00 * dS01 + dF01 * S11 + F01 * dS11;
  const double dP11 = dF10 * S01 + F10 * dS01 + dF11 * S11 + F11 * dS11;
  const double dP21 = dF20 * S01 + F20 * dS01 + dF21 * S11 + F21 * dS11;
  const double s = mat.thickness * area;
  const double P[6] = {dP00, dP10, dP20, dP01, dP11, dP21};
  for (int i = 0; i < 3; i++) {
    const double Pi0 = P[i], Pi1 = P[3 + i];
    const double g1 = s * (Pi0 * a + Pi1 * b);
    const double g2 = s * (Pi0 * c + Pi1 * d);
    const double g0 = -(g1 + g2);
    out[i] = g0;
    out[3 + i] = g1;
    out[6 + i] = g2;
  }
}

// src/physics/membrane-blocks.ts:21-98 triangleHessian9 (same loop nest and
// accumulation order as the reference, including its zero-skips).
void tri_hessian9(const double* x0, const double* x1, const double* x2, const double* inv,
                  double area, const Material& mat, double h[81]) {
  const double a = inv[0], b = inv[1], c = inv[2], d = inv[3];
  const double* X[3] = {x0, x1, x2};
  const double K[3][2] = {{-(a + c), -(b + d)}, {a, b}, {c, d}};
  double F[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 2; j++)
      for (int v = 0; v < 3; v++) F[i][j] += K[v][j] * X[v][i];
  double C[2][2] = {{0, 0}, {0, 0}};
  for (int l = 0; l < 2; l++)
    for (int m = 0; m < 2; m++)
      for (int i = 0; i < 3; i++) C[l][m] += F[i][l] * F[i][m];
  const double E00 = 0.5 * (C[0][0] - 1), E11 = 0.5 * (C[1][1] - 1), E01 = 0.5 * C[0][1];
  const double C00k = mat.C00, C11k = mat.C11, C01k = mat.C01, G = mat.G;
  const double S00 = C00k * E00 + C01k * E11;
  const double S11 = C11k * E11 + C01k * E00;
  const double S01 = 2 * G * E01;
  const double S[2][2] = {{S00, S01}, {S01, S11}};
  double D[2][2][2][2] = {};
  D[0][0][0][0] = C00k;
  D[1][1][1][1] = C11k;
  D[0][0][1][1] = C01k; D[1][1][0][0] = C01k;
  D[0][1][0][1] = G; D[0][1][1][0] = G; D[1][0][0][1] = G; D[1][0][1][0] = G;
  const double s = mat.thickness * area;
  double M[9][3][2] = {};
  for (int v = 0; v < 3; v++)
    for (int ra = 0; ra < 3; ra++)
      for (int j = 0; j < 2; j++) M[v * 3 + ra][ra][j] = K[v][j];
  for (int A = 0; A < 9; A++) {
    for (int B = 0; B < 9; B++) {
      double sum = 0;
      for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 2; j++) {
          const double mA = M[A][i][j];
          if (mA == 0) continue;
          double dP = 0;
          for (int k = 0; k < 2; k++) {
            dP += M[B][i][k] * S[k][j];
            double dE = 0;
            for (int l = 0; l < 2; l++) {
              for (int m2 = 0; m2 < 2; m2++) {
                const double dd = D[k][j][l][m2];
                if (dd == 0) continue;
                double dElm = 0;
                for (int p = 0; p < 3; p++) dElm += M[B][p][l] * F[p][m2] + F[p][l] * M[B][p][m2];
                dE += dd * 0.5 * dElm;
              }
            }
            dP += F[i][k] * dE;
          }
          sum += mA * dP;
        }
      }
      h[A * 9 + B] = s * sum;
    }
  }
}

// src/physics/bending.ts:7-16 hingeEnergy.
double hinge_energy(const double* x, int v0, int v1, int v2, int v3, double restAngle,
                    double edgeLen, double areaSum, double k) {
  const double th = dihedral(x, v0, v1, v2, v3);
  const double d = th - restAngle;
  const double w = edgeLen * edgeLen / js_max(areaSum, 1e-12);
  return 0.5 * k * d * d * w;
}

// src/physics/bending.ts:19-42 addHingeGradient: central differences, eps 1e-7,
// over the 12 hinge dofs. The reference perturbs a full copy of x
// (`Float64Array.from(x)`); only the 4 hinge vertices are read, so this port
// perturbs a 4-vertex local copy instead. Results are identical.
double add_hinge_gradient(const double* x, double* grad, int v0, int v1, int v2, int v3,
                          double restAngle, double edgeLen, double areaSum, double k, double eps) {
  const int verts[4] = {v0, v1, v2, v3};
  const double e = hinge_energy(x, v0, v1, v2, v3, restAngle, edgeLen, areaSum, k);
  // Local copy: vertices renumbered 0..3 (first occurrence wins, as one shared array).
  int lid[4];
  double loc[12];
  int nl = 0;
  int uniq[4];
  for (int a = 0; a < 4; a++) {
    int found = -1;
    for (int b = 0; b < nl; b++) if (uniq[b] == verts[a]) found = b;
    if (found < 0) { uniq[nl] = verts[a]; found = nl++; }
    lid[a] = found;
  }
  for (int b = 0; b < nl; b++)
    for (int i = 0; i < 3; i++) loc[b * 3 + i] = x[uniq[b] * 3 + i];
  for (int a = 0; a < 4; a++) {
    for (int i = 0; i < 3; i++) {
      const int li = lid[a] * 3 + i;
      const double old = loc[li];
      loc[li] = old + eps;
      const double ep = hinge_energy(loc, lid[0], lid[1], lid[2], lid[3], restAngle, edgeLen, areaSum, k);
      loc[li] = old - eps;
      const double em = hinge_energy(loc, lid[0], lid[1], lid[2], lid[3], restAngle, edgeLen, areaSum, k);
      loc[li] = old;
      grad[verts[a] * 3 + i] += (ep - em) / (2 * eps);
    }
  }
  return e;
}

static inline void load3(const double* x, uint32_t v, double o[3]) {
  o[0] = x[v * 3]; o[1] = x[v * 3 + 1]; o[2] = x[v * 3 + 2];
}
static inline void inv4(const Mesh& me, int t, double o[4]) {
  for (int k = 0; k < 4; k++) o[k] = me.invDm[t * 4 + k];
}

// src/physics/fem.ts:15-54 evalInternal (grad zero-filled, then scattered).
FemEval eval_internal(const double* x, const Mesh& mesh, const Material& mat, double* grad) {
  std::fill(grad, grad + mesh.n * 3, 0.0);
  double energy = 0, maxStrain = 0;
  TriGrad r;
  for (int t = 0; t < mesh.m; t++) {
    uint32_t vs[3] = {mesh.idx[t * 3], mesh.idx[t * 3 + 1], mesh.idx[t * 3 + 2]};
    double p0[3], p1[3], p2[3], inv[4];
    load3(x, vs[0], p0); load3(x, vs[1], p1); load3(x, vs[2], p2); inv4(mesh, t, inv);
    tri_energy_grad(p0, p1, p2, inv, mesh.areas[t], mat, r);
    energy += r.energy;
    maxStrain = js_max(js_max(js_max(maxStrain, std::fabs(r.E00)), std::fabs(r.E11)), std::fabs(r.E01));
    for (int v = 0; v < 3; v++)
      for (int i = 0; i < 3; i++) grad[vs[v] * 3 + i] += r.grad[v * 3 + i];
  }
  const double kb = 0.5 * (mat.bendWarp + mat.bendWeft);
  if (kb > 0) {
    for (const Hinge& h : mesh.hinges)
      energy += add_hinge_gradient(x, grad, h.v0, h.v1, h.v2, h.v3, h.restAngle, h.edgeLen, h.areaSum, kb);
  }
  return {energy, maxStrain};
}

// src/physics/fem.ts:56-75 internalEnergyOnly.
double internal_energy_only(const double* x, const Mesh& mesh, const Material& mat) {
  double e = 0;
  TriGrad r;
  for (int t = 0; t < mesh.m; t++) {
    double p0[3], p1[3], p2[3], inv[4];
    load3(x, mesh.idx[t * 3], p0); load3(x, mesh.idx[t * 3 + 1], p1); load3(x, mesh.idx[t * 3 + 2], p2);
    inv4(mesh, t, inv);
    tri_energy_grad(p0, p1, p2, inv, mesh.areas[t], mat, r);
    e += r.energy;
  }
  const double kb = 0.5 * (mat.bendWarp + mat.bendWeft);
  if (kb > 0)
    for (const Hinge& h : mesh.hinges)
      e += hinge_energy(x, h.v0, h.v1, h.v2, h.v3, h.restAngle, h.edgeLen, h.areaSum, kb);
  return e;
}

// src/physics/fem.ts:78-104 evalMembrane.
double eval_membrane(const double* x, const Mesh& mesh, const Material& mat, double* grad) {
  std::fill(grad, grad + mesh.n * 3, 0.0);
  double energy = 0;
  TriGrad r;
  for (int t = 0; t < mesh.m; t++) {
    uint32_t vs[3] = {mesh.idx[t * 3], mesh.idx[t * 3 + 1], mesh.idx[t * 3 + 2]};
    double p0[3], p1[3], p2[3], inv[4];
    load3(x, vs[0], p0); load3(x, vs[1], p1); load3(x, vs[2], p2); inv4(mesh, t, inv);
    tri_energy_grad(p0, p1, p2, inv, mesh.areas[t], mat, r);
    energy += r.energy;
    for (int v = 0; v < 3; v++)
      for (int i = 0; i < 3; i++) grad[vs[v] * 3 + i] += r.grad[v * 3 + i];
  }
  return energy;
}

// src/physics/fem.ts:108-130 membraneHvp: central FD of the membrane gradient,
// h = eps (1 + |p|).
void membrane_hvp(const double* x, const double* p, const Mesh& mesh, const Material& mat,
                  double* out, double eps) {
  const int n3 = mesh.n * 3;
  double pNorm = 0;
  for (int i = 0; i < n3; i++) pNorm += p[i] * p[i];
  pNorm = std::sqrt(pNorm);
  const double h = eps * (1 + pNorm);
  Vec xp(n3), xm(n3), gp(n3), gm(n3);
  for (int i = 0; i < n3; i++) { xp[i] = x[i] + h * p[i]; xm[i] = x[i] - h * p[i]; }
  eval_membrane(xp.data(), mesh, mat, gp.data());
  eval_membrane(xm.data(), mesh, mat, gm.data());
  for (int i = 0; i < n3; i++) out[i] = (gp[i] - gm[i]) / (2 * h);
}

// src/physics/membrane-hvp.ts:80-108 evalMembraneHvp.
void eval_membrane_hvp(const double* x, const double* p, const Mesh& mesh, const Material& mat,
                       double* out) {
  std::fill(out, out + mesh.n * 3, 0.0);
  double o[9];
  for (int t = 0; t < mesh.m; t++) {
    uint32_t vs[3] = {mesh.idx[t * 3], mesh.idx[t * 3 + 1], mesh.idx[t * 3 + 2]};
    double p0[3], p1[3], p2[3], q0[3], q1[3], q2[3], inv[4];
    load3(x, vs[0], p0); load3(x, vs[1], p1); load3(x, vs[2], p2);
    load3(p, vs[0], q0); load3(p, vs[1], q1); load3(p, vs[2], q2);
    inv4(mesh, t, inv);
    tri_hvp(p0, p1, p2, q0, q1, q2, inv, mesh.areas[t], mat, o);
    for (int v = 0; v < 3; v++)
      for (int i = 0; i < 3; i++) out[vs[v] * 3 + i] += o[v * 3 + i];
  }
}

// src/physics/membrane-blocks.ts:102-130 evalMembraneBlocks.
void eval_membrane_blocks(const double* x, const Mesh& mesh, const Material& mat, double* blocks) {
  std::fill(blocks, blocks + mesh.n * 9, 0.0);
  double h[81];
  for (int t = 0; t < mesh.m; t++) {
    uint32_t vs[3] = {mesh.idx[t * 3], mesh.idx[t * 3 + 1], mesh.idx[t * 3 + 2]};
    double p0[3], p1[3], p2[3], inv[4];
    load3(x, vs[0], p0); load3(x, vs[1], p1); load3(x, vs[2], p2); inv4(mesh, t, inv);
    tri_hessian9(p0, p1, p2, inv, mesh.areas[t], mat, h);
    for (int vc = 0; vc < 3; vc++)
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) blocks[vs[vc] * 9 + a * 3 + b] += h[(vc * 3 + a) * 9 + (vc * 3 + b)];
  }
}

// src/mesh/incidence.ts:41-75 CSR incidence maps (element-ordered records).
static Incidence build_map(int nv, int nrec, const std::vector<std::array<int, 3>>& emits) {
  Incidence inc;
  std::vector<uint32_t> counts(nv, 0);
  for (auto& e : emits) counts[e[0]]++;
  inc.offsets.assign(nv + 1, 0);
  for (int v = 0; v < nv; v++) inc.offsets[v + 1] = inc.offsets[v] + counts[v];
  inc.ids.assign(nrec, 0);
  inc.corners.assign(nrec, 0);
  std::vector<uint32_t> cursor(inc.offsets.begin(), inc.offsets.end() - 1);
  for (auto& e : emits) {
    uint32_t k = cursor[e[0]]++;
    inc.ids[k] = e[1];
    inc.corners[k] = e[2];
  }
  return inc;
}
Incidence membrane_incidence(const Mesh& mesh) {
  std::vector<std::array<int, 3>> em;
  em.reserve(mesh.m * 3);
  for (int t = 0; t < mesh.m; t++)
    for (int c = 0; c < 3; c++) em.push_back({(int)mesh.idx[t * 3 + c], t, c});
  return build_map(mesh.n, mesh.m * 3, em);
}
Incidence hinge_incidence(const Mesh& mesh) {
  std::vector<std::array<int, 3>> em;
  int hc = (int)mesh.hinges.size();
  for (int hh = 0; hh < hc; hh++) {
    const Hinge& h = mesh.hinges[hh];
    int vs[4] = {h.v0, h.v1, h.v2, h.v3};
    for (int c = 0; c < 4; c++) {
      bool seen = false;
      for (int q = 0; q < c; q++) if (vs[q] == vs[c]) seen = true;
      if (!seen) em.push_back({vs[c], hh, c});
    }
  }
  return build_map(mesh.n, (int)em.size(), em);
}

// src/solver/schwarz.ts:27-36 morton3 over rest-space, 10 bits per axis.
static uint32_t morton3(double x, double y, double z) {
  auto q = [](double v) -> int {
    double f = std::floor(v * 1024);
    double c = js_max(0, js_min(1023, f));
    return (int)c;
  };
  int xi = q(x), yi = q(y), zi = q(z);
  uint32_t m = 0;
  for (int b = 9; b >= 0; b--)
    m = (m << 3) | (((xi >> b) & 1) << 2) | (((yi >> b) & 1) << 1) | ((zi >> b) & 1);
  return m;
}

// src/solver/schwarz.ts:44-140 buildSchwarzDomains.
SchwarzDomains build_schwarz_domains(const Mesh& mesh, const float* rest, int targetSize,
                                     int minSize, int maxSize) {
  (void)maxSize;
  const int n = mesh.n;
  const auto& idx = mesh.idx;
  std::vector<std::set<int>> adj(n);
  for (int t = 0; t < mesh.m; t++) {
    int a = idx[t * 3], b = idx[t * 3 + 1], c = idx[t * 3 + 2];
    adj[a].insert(b); adj[a].insert(c);
    adj[b].insert(a); adj[b].insert(c);
    adj[c].insert(a); adj[c].insert(b);
  }
  std::vector<std::vector<int>> adjArr(n);
  for (int v = 0; v < n; v++) adjArr[v].assign(adj[v].begin(), adj[v].end());
  double mnx = INF, mny = INF, mnz = INF, mxx = -INF, mxy = -INF, mxz = -INF;
  for (int v = 0; v < n; v++) {
    mnx = js_min(mnx, rest[v * 3]); mny = js_min(mny, rest[v * 3 + 1]); mnz = js_min(mnz, rest[v * 3 + 2]);
    mxx = js_max(mxx, rest[v * 3]); mxy = js_max(mxy, rest[v * 3 + 1]); mxz = js_max(mxz, rest[v * 3 + 2]);
  }
  const double sx = js_max(mxx - mnx, 1e-12), sy = js_max(mxy - mny, 1e-12), sz = js_max(mxz - mnz, 1e-12);
  std::vector<int> order(n);
  std::vector<uint32_t> code(n);
  for (int v = 0; v < n; v++) {
    order[v] = v;
    code[v] = morton3(((double)rest[v * 3] - mnx) / sx, ((double)rest[v * 3 + 1] - mny) / sy,
                      ((double)rest[v * 3 + 2] - mnz) / sz);
  }
  std::sort(order.begin(), order.end(), [&](int a, int b) {
    return code[a] != code[b] ? code[a] < code[b] : a < b;
  });
  const uint32_t UN = 0xffffffffu;
  std::vector<uint32_t> domainOf(n, UN);
  std::vector<std::vector<int>> members;
  for (int seed : order) {
    if (domainOf[seed] != UN) continue;
    const int id = (int)members.size();
    std::vector<int> mem{seed};
    domainOf[seed] = id;
    std::deque<int> queue{seed};
    while ((int)mem.size() < targetSize && !queue.empty()) {
      int cur = queue.front();
      queue.pop_front();
      for (int w : adjArr[cur]) {
        if ((int)mem.size() >= targetSize) break;
        if (domainOf[w] != UN) continue;
        domainOf[w] = id;
        mem.push_back(w);
        queue.push_back(w);
      }
    }
    members.push_back(mem);
  }
  for (;;) {
    int small = -1;
    for (int d = 0; d < (int)members.size(); d++) {
      int len = (int)members[d].size();
      if (len > 0 && len < minSize && n >= minSize) {
        if (small < 0 || len < (int)members[small].size()) small = d;
      }
    }
    if (small < 0) break;
    std::set<int> nb;
    for (int t = 0; t < mesh.m; t++) {
      uint32_t ds[3] = {domainOf[idx[t * 3]], domainOf[idx[t * 3 + 1]], domainOf[idx[t * 3 + 2]]};
      bool hasSmall = ds[0] == (uint32_t)small || ds[1] == (uint32_t)small || ds[2] == (uint32_t)small;
      if (!hasSmall) continue;
      for (uint32_t b : ds) if (b != (uint32_t)small) nb.insert((int)b);
    }
    int best = -1;
    for (int c : nb) {
      if (members[c].empty()) continue;
      if (best < 0 || members[c].size() < members[best].size()) best = c;
    }
    if (best < 0) break;
    for (int v : members[small]) { domainOf[v] = best; members[best].push_back(v); }
    members[small].clear();
  }
  SchwarzDomains out;
  std::vector<int> remap(members.size(), -1);
  for (size_t d = 0; d < members.size(); d++) {
    if (members[d].empty()) continue;
    remap[d] = (int)out.members.size();
    std::vector<int> mem = members[d];
    std::sort(mem.begin(), mem.end());
    out.members.push_back(mem);
  }
  out.domainOf.assign(n, 0);
  out.localOf.assign(n, 0);
  for (int v = 0; v < n; v++) out.domainOf[v] = remap[domainOf[v]];
  for (auto& mem : out.members)
    for (size_t l = 0; l < mem.size(); l++) out.localOf[mem[l]] = (uint32_t)l;
  return out;
}

// src/solver/schwarz.ts:154-252 buildSchwarzFactors.
void build_schwarz_factors(const double* x, const Mesh& mesh, const Material& mat,
                           const double* diag, const SchwarzDomains& dom, SchwarzFactors& f) {
  const auto& idx = mesh.idx;
  const int D = (int)dom.members.size();
  f.dom = &dom;
  f.data.assign(D, Vec());
  f.flag.assign(D, 0);
  std::vector<std::vector<int>> v2t(mesh.n);
  for (int t = 0; t < mesh.m; t++) {
    v2t[idx[t * 3]].push_back(t);
    v2t[idx[t * 3 + 1]].push_back(t);
    v2t[idx[t * 3 + 2]].push_back(t);
  }
  double h[81];
  for (int d = 0; d < D; d++) {
    const auto& mem = dom.members[d];
    const int dv = (int)mem.size(), dw = dv * 3;
    Vec A(dw * dw, 0.0);
    auto loc = [&](int v) -> int {
      for (int l = 0; l < dv; l++) if (mem[l] == v) return l;
      return -1;
    };
    for (int v : mem) {
      for (int t : v2t[v]) {
        int cvs[3] = {(int)idx[t * 3], (int)idx[t * 3 + 1], (int)idx[t * 3 + 2]};
        int ci = cvs[0] == v ? 0 : cvs[1] == v ? 1 : 2;
        double p0[3], p1[3], p2[3], inv[4];
        load3(x, cvs[0], p0); load3(x, cvs[1], p1); load3(x, cvs[2], p2); inv4(mesh, t, inv);
        tri_hessian9(p0, p1, p2, inv, mesh.areas[t], mat, h);
        for (int cj = 0; cj < 3; cj++) {
          int lw = loc(cvs[cj]);
          if (lw < 0) continue;
          int lv = loc(v);
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
              A[(lv * 3 + a) * dw + (lw * 3 + b)] += h[(ci * 3 + a) * 9 + (cj * 3 + b)];
        }
      }
    }
    for (int l = 0; l < dv; l++)
      for (int a = 0; a < 3; a++) A[(l * 3 + a) * dw + (l * 3 + a)] += diag[mem[l] * 3 + a];
    for (int i = 0; i < dw; i++)
      for (int j = i + 1; j < dw; j++) {
        double s = 0.5 * (A[i * dw + j] + A[j * dw + i]);
        A[i * dw + j] = s; A[j * dw + i] = s;
      }
    double scale = 0;
    for (int i = 0; i < dw; i++) scale = js_max(scale, std::fabs(A[i * dw + i]));
    const double tiny = 1e-20 * (1 + scale);
    bool ok = true;
    Vec L = A;
    for (int k = 0; k < dw && ok; k++) {
      double sum = L[k * dw + k];
      for (int s = 0; s < k; s++) sum -= L[k * dw + s] * L[k * dw + s];
      if (!(sum > tiny)) { ok = false; break; }
      L[k * dw + k] = std::sqrt(sum);
      for (int i = k + 1; i < dw; i++) {
        double s2 = L[i * dw + k];
        for (int s = 0; s < k; s++) s2 -= L[i * dw + s] * L[k * dw + s];
        L[i * dw + k] = s2 / L[k * dw + k];
      }
    }
    if (ok) {
      for (int i = 0; i < dw; i++)
        for (int j = i + 1; j < dw; j++) L[i * dw + j] = 0;
      f.data[d] = std::move(L);
      f.flag[d] = 1;
    } else {
      Vec J(dw * dw, 0.0);
      for (int l = 0; l < dv; l++)
        for (int a = 0; a < 3; a++) {
          double dd = diag[mem[l] * 3 + a];
          J[(l * 3 + a) * dw + (l * 3 + a)] = dd > 1e-12 ? 1 / dd : 0;
        }
      f.data[d] = std::move(J);
      f.flag[d] = 0;
    }
  }
}

// src/solver/schwarz.ts:255-309 solveLocal + applySchwarz.
void apply_schwarz(const SchwarzFactors& f, const double* r, double* out, int n) {
  std::fill(out, out + n * 3, 0.0);
  const auto& dom = *f.dom;
  const int D = (int)dom.members.size();
  Vec rhs, y, sol;
  for (int d = 0; d < D; d++) {
    const auto& mem = dom.members[d];
    const int dv = (int)mem.size(), dw = dv * 3;
    rhs.assign(dw, 0.0); y.assign(dw, 0.0); sol.assign(dw, 0.0);
    for (int l = 0; l < dv; l++)
      for (int k = 0; k < 3; k++) rhs[l * 3 + k] = r[mem[l] * 3 + k];
    const Vec& M = f.data[d];
    if (f.flag[d] == 1) {
      for (int i = 0; i < dw; i++) {
        double s = rhs[i];
        for (int j = 0; j < i; j++) s -= M[i * dw + j] * y[j];
        y[i] = s / M[i * dw + i];
      }
      for (int i = dw - 1; i >= 0; i--) {
        double s = y[i];
        for (int j = i + 1; j < dw; j++) s -= M[j * dw + i] * sol[j];
        sol[i] = s / M[i * dw + i];
      }
    } else {
      for (int i = 0; i < dw; i++) {
        double s = 0;
        for (int j = 0; j < dw; j++) s += M[i * dw + j] * rhs[j];
        sol[i] = s;
      }
    }
    for (int l = 0; l < dv; l++)
      for (int k = 0; k < 3; k++) out[mem[l] * 3 + k] += sol[l * 3 + k];
  }
}

// src/solver/block-jacobi.ts:30-104 buildBlockFactors / applyBlockFactors.
void build_block_factors(const double* x, const Mesh& mesh, const Material& mat, const double* diag,
                         BlockFactors& f) {
  const int n = mesh.n;
  Vec blocks(n * 9);
  eval_membrane_blocks(x, mesh, mat, blocks.data());
  f.inv.assign(n * 9, 0.0);
  f.flag.assign(n, 0);
  for (int v = 0; v < n; v++) {
    const double* hb = &blocks[v * 9];
    const double h00 = hb[0], h01 = hb[1], h02 = hb[2], h10 = hb[3], h11 = hb[4], h12 = hb[5],
                 h20 = hb[6], h21 = hb[7], h22 = hb[8];
    const double d0 = diag[v * 3], d1 = diag[v * 3 + 1], d2 = diag[v * 3 + 2];
    const double B00 = h00 + d0, B11 = h11 + d1, B22 = h22 + d2;
    const double B01 = 0.5 * (h01 + h10), B02 = 0.5 * (h02 + h20), B12 = 0.5 * (h12 + h21);
    const double tr = std::fabs(B00) + std::fabs(B11) + std::fabs(B22);
    const double tiny = 1e-20 * (1 + tr);
    bool ok = true;
    if (!(B00 > tiny)) ok = false;
    if (ok && !(B00 * B11 - B01 * B01 > tiny * (1 + std::fabs(B00) + std::fabs(B11)))) ok = false;
    const double det = B00 * (B11 * B22 - B12 * B12) - B01 * (B01 * B22 - B12 * B02) +
                       B02 * (B01 * B12 - B11 * B02);
    if (ok && !(det > tiny * (1 + tr) * (1 + tr))) ok = false;
    double* o = &f.inv[v * 9];
    if (ok) {
      const double s = 1 / det;
      o[0] = (B11 * B22 - B12 * B12) * s;
      o[1] = (B02 * B12 - B01 * B22) * s;
      o[2] = (B01 * B12 - B11 * B02) * s;
      o[3] = (B02 * B12 - B01 * B22) * s;
      o[4] = (B00 * B22 - B02 * B02) * s;
      o[5] = (B01 * B02 - B00 * B12) * s;
      o[6] = (B01 * B12 - B11 * B02) * s;
      o[7] = (B01 * B02 - B00 * B12) * s;
      o[8] = (B00 * B11 - B01 * B01) * s;
      f.flag[v] = 1;
    } else {
      o[0] = d0 > 1e-12 ? 1 / d0 : 0;
      o[4] = d1 > 1e-12 ? 1 / d1 : 0;
      o[8] = d2 > 1e-12 ? 1 / d2 : 0;
      f.flag[v] = 0;
    }
  }
}
void apply_block_factors(const BlockFactors& f, const double* r, double* out, int n) {
  for (int v = 0; v < n; v++) {
    const double r0 = r[v * 3], r1 = r[v * 3 + 1], r2 = r[v * 3 + 2];
    const double* b = &f.inv[v * 9];
    out[v * 3] = b[0] * r0 + b[1] * r1 + b[2] * r2;
    out[v * 3 + 1] = b[3] * r0 + b[4] * r1 + b[5] * r2;
    out[v * 3 + 2] = b[6] * r0 + b[7] * r1 + b[8] * r2;
  }
}

}  // namespace orc
