// Oracle (test infrastructure only): src/math/pcg.ts:11-95 restated.
// Filtered PCG from x0 = 0; stops on pAp <= 1e-30 (returns current x) or
// ||r|| < max(tol * max(||b||, 1e-12), 1e-12). Optional custom M^-1.
#pragma once
#include <cmath>
#include <functional>
#include <vector>

#include "orc.hpp"

namespace orc {

inline double dot_self(const Vec& a) {
  double s = 0;
  for (double v : a) s += v * v;
  return s;
}

template <class Hvp, class Filter>
PcgResult pcg_impl(const Vec& b, Hvp&& hvp, const Vec& diag, int maxIters, double tol,
                   Filter&& filter, bool hasFilter,
                   const std::function<void(const Vec&, Vec&)>* prec, Vec& x) {
  const size_t n = b.size();
  x.assign(n, 0.0);
  Vec r = b, z(n, 0.0), p(n, 0.0), Ap(n, 0.0);
  if (hasFilter) filter(r.data());
  if (prec) (*prec)(r, z);
  else
    for (size_t i = 0; i < n; i++) z[i] = diag[i] > 1e-12 ? r[i] / diag[i] : r[i];
  if (hasFilter) filter(z.data());
  p = z;
  double rz = 0;
  for (size_t i = 0; i < n; i++) rz += r[i] * z[i];
  const double bNorm = std::sqrt(dot_self(b));
  const double absTol = js_max(tol * js_max(bNorm, 1e-12), 1e-12);
  double residual = std::sqrt(dot_self(r));
  if (residual < absTol) return {0, residual, true};
  for (int k = 0; k < maxIters; k++) {
    if (hasFilter) filter(p.data());
    hvp(p, Ap);
    if (hasFilter) filter(Ap.data());
    double pAp = 0;
    for (size_t i = 0; i < n; i++) pAp += p[i] * Ap[i];
    if (!(pAp > 1e-30)) return {k, residual, residual < absTol};
    const double alpha = rz / pAp;
    for (size_t i = 0; i < n; i++) {
      x[i] += alpha * p[i];
      r[i] -= alpha * Ap[i];
    }
    if (hasFilter) { filter(x.data()); filter(r.data()); }
    residual = std::sqrt(dot_self(r));
    if (residual < absTol) return {k + 1, residual, true};
    if (prec) (*prec)(r, z);
    else
      for (size_t i = 0; i < n; i++) z[i] = diag[i] > 1e-12 ? r[i] / diag[i] : r[i];
    if (hasFilter) filter(z.data());
    double rzNew = 0;
    for (size_t i = 0; i < n; i++) rzNew += r[i] * z[i];
    const double beta = rzNew / rz;
    for (size_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    rz = rzNew;
  }
  return {maxIters, residual, false};
}

template <class Hvp, class Prec, class Filter>
PcgResult pcg(const Vec& b, Hvp&& hvp, const Vec& diag, int maxIters, double tol, Filter&& filter,
              bool hasFilter, Prec* prec, Vec& x) {
  return pcg_impl(b, hvp, diag, maxIters, tol, filter, hasFilter, prec, x);
}

}  // namespace orc
