// Oracle: two-level additive Schwarz (test infrastructure, restating the
// reference's src/solver/mas.ts; used by tests/ only, never by the product).
//
// Aggregates are the Schwarz domains. The coarse space holds one constant
// vector per domain and component, with the normalized restriction
// R[(d,a)][(v,a)] = 1/sqrt(|d|) for v in d (mas.ts:1-13):
//   mas2  z = Schwarz1(r) + P (omega Dc^-1) R r, Dc = diag(R A P)   (mas.ts:103-139)
//   masX  z = Schwarz1(r) + P Ac^-1 R r, Ac = R A P dense + Cholesky (mas.ts:143-250)
// A is the membrane Hessian from the analytic 9x9 blocks plus the Jacobi
// diagonal, as in the Schwarz factors. Loops and accumulation orders follow
// the reference so that PCG iteration counts reproduce its published ones.
#include <cmath>

#include "orc.hpp"

namespace orc {

// restrictCoarse (mas.ts:22-38): rc[d*3+a] = sum_{v in d} r[v*3+a] / sqrt(|d|).
void restrict_coarse(const double* r, const SchwarzDomains& dom, double* rc) {
  const int D = (int)dom.members.size();
  for (int i = 0; i < D * 3; i++) rc[i] = 0.0;
  for (int d = 0; d < D; d++) {
    const double s = 1 / std::sqrt((double)dom.members[d].size());
    for (int v : dom.members[d])
      for (int a = 0; a < 3; a++) rc[d * 3 + a] += r[v * 3 + a] * s;
  }
}

// prolongateAdd (mas.ts:40-55): z[v*3+a] += c[d*3+a] / sqrt(|d|).
void prolongate_add(const double* c, const SchwarzDomains& dom, double* z) {
  const int D = (int)dom.members.size();
  for (int d = 0; d < D; d++) {
    const double s = 1 / std::sqrt((double)dom.members[d].size());
    for (int v : dom.members[d])
      for (int a = 0; a < 3; a++) z[v * 3 + a] += c[d * 3 + a] * s;
  }
}

// buildCoarseDiag (mas.ts:57-101): the within-domain diagonal entries of the
// triangle blocks, then the Jacobi diagonal, each spread as 1/|d|.
Vec build_coarse_diag(const double* x, const Mesh& mesh, const Material& mat, const double* diag,
                      const SchwarzDomains& dom) {
  const int D = (int)dom.members.size();
  Vec dc((size_t)D * 3, 0.0);
  for (int t = 0; t < mesh.m; t++) {
    const int cv[3] = {(int)mesh.idx[t * 3], (int)mesh.idx[t * 3 + 1], (int)mesh.idx[t * 3 + 2]};
    double p0[3], p1[3], p2[3], inv[4], h[81];
    for (int k = 0; k < 3; k++) { p0[k] = x[cv[0] * 3 + k]; p1[k] = x[cv[1] * 3 + k]; p2[k] = x[cv[2] * 3 + k]; }
    for (int k = 0; k < 4; k++) inv[k] = mesh.invDm[t * 4 + k];
    tri_hessian9(p0, p1, p2, inv, mesh.areas[t], mat, h);
    for (int ci = 0; ci < 3; ci++)
      for (int cj = 0; cj < 3; cj++) {
        const int d1 = (int)dom.domainOf[cv[ci]], d2 = (int)dom.domainOf[cv[cj]];
        if (d1 != d2) continue;
        const double s = 1.0 / (double)dom.members[d1].size();
        for (int a = 0; a < 3; a++) dc[d1 * 3 + a] += s * h[(ci * 3 + a) * 9 + (cj * 3 + a)];
      }
  }
  for (int d = 0; d < D; d++) {
    const double s = 1.0 / (double)dom.members[d].size();
    for (int v : dom.members[d])
      for (int a = 0; a < 3; a++) dc[d * 3 + a] += s * diag[v * 3 + a];
  }
  return dc;
}

// applyMasTwoLevel (mas.ts:110-145).
void apply_mas2(const SchwarzFactors& sf, const Vec& dc, double omega, const double* r, double* out, int n) {
  apply_schwarz(sf, r, out, n);
  const SchwarzDomains& dom = *sf.dom;
  const int D = (int)dom.members.size();
  Vec rc((size_t)D * 3);
  restrict_coarse(r, dom, rc.data());
  for (int i = 0; i < D * 3; i++) rc[i] = dc[i] > 1e-12 ? (omega * rc[i]) / dc[i] : 0.0;
  prolongate_add(rc.data(), dom, out);
}

// buildCoarseExact (mas.ts:153-222): dense Ac = R A P + diagonal spread,
// symmetrized, Cholesky (row-oriented, the reference's loop order) or the
// inverse diagonal when a pivot fails.
void build_coarse_exact(const double* x, const Mesh& mesh, const Material& mat, const double* diag,
                        const SchwarzDomains& dom, CoarseExact& ce) {
  const int D = (int)dom.members.size(), dc = D * 3;
  ce.dom = &dom;
  ce.n = dc;
  Vec ac((size_t)dc * dc, 0.0);
  for (int t = 0; t < mesh.m; t++) {
    const int cv[3] = {(int)mesh.idx[t * 3], (int)mesh.idx[t * 3 + 1], (int)mesh.idx[t * 3 + 2]};
    double p0[3], p1[3], p2[3], inv[4], h[81];
    for (int k = 0; k < 3; k++) { p0[k] = x[cv[0] * 3 + k]; p1[k] = x[cv[1] * 3 + k]; p2[k] = x[cv[2] * 3 + k]; }
    for (int k = 0; k < 4; k++) inv[k] = mesh.invDm[t * 4 + k];
    tri_hessian9(p0, p1, p2, inv, mesh.areas[t], mat, h);
    for (int ci = 0; ci < 3; ci++)
      for (int cj = 0; cj < 3; cj++) {
        const int d1 = (int)dom.domainOf[cv[ci]], d2 = (int)dom.domainOf[cv[cj]];
        const double s = 1 / std::sqrt((double)dom.members[d1].size() * (double)dom.members[d2].size());
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++)
            ac[(size_t)(d1 * 3 + a) * dc + (d2 * 3 + b)] += s * h[(ci * 3 + a) * 9 + (cj * 3 + b)];
      }
  }
  for (int d = 0; d < D; d++) {
    const double s = 1.0 / (double)dom.members[d].size();
    for (int v : dom.members[d])
      for (int a = 0; a < 3; a++) ac[(size_t)(d * 3 + a) * dc + (d * 3 + a)] += s * diag[v * 3 + a];
  }
  for (int i = 0; i < dc; i++)
    for (int j = i + 1; j < dc; j++) {
      const double s = 0.5 * (ac[(size_t)i * dc + j] + ac[(size_t)j * dc + i]);
      ac[(size_t)i * dc + j] = s;
      ac[(size_t)j * dc + i] = s;
    }
  Vec L = ac;
  double scale = 0;
  for (int i = 0; i < dc; i++) scale = std::fmax(scale, std::fabs(L[(size_t)i * dc + i]));
  const double tiny = 1e-20 * (1 + scale);
  bool ok = true;
  for (int k = 0; k < dc && ok; k++) {
    double sum = L[(size_t)k * dc + k];
    for (int s = 0; s < k; s++) sum -= L[(size_t)k * dc + s] * L[(size_t)k * dc + s];
    if (!(sum > tiny)) { ok = false; break; }
    L[(size_t)k * dc + k] = std::sqrt(sum);
    for (int i = k + 1; i < dc; i++) {
      double s2 = L[(size_t)i * dc + k];
      for (int s = 0; s < k; s++) s2 -= L[(size_t)i * dc + s] * L[(size_t)k * dc + s];
      L[(size_t)i * dc + k] = s2 / L[(size_t)k * dc + k];
    }
  }
  if (ok) {
    for (int i = 0; i < dc; i++)
      for (int j = i + 1; j < dc; j++) L[(size_t)i * dc + j] = 0;
    ce.chol = std::move(L);
    ce.flag = 1;
    return;
  }
  Vec J((size_t)dc * dc, 0.0);
  for (int i = 0; i < dc; i++) {
    const double a = ac[(size_t)i * dc + i];
    J[(size_t)i * dc + i] = a > 1e-12 ? 1 / a : 0.0;
  }
  ce.chol = std::move(J);
  ce.flag = 0;
}

// solveCoarseExact (mas.ts:225-250).
void solve_coarse_exact(const CoarseExact& ce, const double* rhs, double* out) {
  const int dc = ce.n;
  if (ce.flag == 1) {
    Vec y(dc);
    for (int i = 0; i < dc; i++) {
      double s = rhs[i];
      for (int j = 0; j < i; j++) s -= ce.chol[(size_t)i * dc + j] * y[j];
      y[i] = s / ce.chol[(size_t)i * dc + i];
    }
    for (int i = dc - 1; i >= 0; i--) {
      double s = y[i];
      for (int j = i + 1; j < dc; j++) s -= ce.chol[(size_t)j * dc + i] * out[j];
      out[i] = s / ce.chol[(size_t)i * dc + i];
    }
  } else {
    for (int i = 0; i < dc; i++) {
      double s = 0;
      for (int j = 0; j < dc; j++) s += ce.chol[(size_t)i * dc + j] * rhs[j];
      out[i] = s;
    }
  }
}

// The masX apply of tests/preconditioner-compare.test.ts:160-180:
// Schwarz1, then the exact coarse correction.
void apply_masx(const SchwarzFactors& sf, const CoarseExact& ce, const double* r, double* out, int n) {
  apply_schwarz(sf, r, out, n);
  Vec rc(ce.n), cc(ce.n);
  restrict_coarse(r, *sf.dom, rc.data());
  solve_coarse_exact(ce, rc.data(), cc.data());
  prolongate_add(cc.data(), *sf.dom, out);
}

}  // namespace orc
