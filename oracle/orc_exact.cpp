// Oracle (test infrastructure only): the pieces of the CUDA solver's
// exact-Newton mode, restated for the CPU so the mode's converged steps can be
// checked against an independent implementation. The reference has no such
// mode; each piece is the mathematics of a reference term:
//   - the hinge gradient and Hessian of bending.ts:7-16's energy,
//     differentiated exactly (the reference takes central differences,
//     bending.ts:19-42) through the signed bend angle, with hyper-dual numbers
//     over atan2;
//   - the membrane Hessian of membrane-hvp.ts:18-75 with the stress of its
//     geometric term replaced by its positive part;
//   - the lagged Coulomb friction of friction.ts:14-23 as the potential
//     D = mu lambda sqrt(|P u|^2 + eps^2) of the relative slip u
//     (contact-assembly.ts:344-367), with lambda and the normal n frozen at the
//     Newton iterate; its gradient is the reference's friction force on floor
//     and one-sided static contacts (on cloth-cloth contacts the reference's
//     force is the gradient of no potential).
#include <cmath>
#include <functional>
#include <stdexcept>

#include "orc.hpp"
#include "orc_pcg.hpp"

namespace orc {

namespace {

// Hyper-dual number v + a e1 + b e2 + ab e1 e2 (e1^2 = e2^2 = 0). One pass of
// a function over it gives the value, the derivatives along the two seeds and
// the mixed second derivative, all exact.
struct HD {
  double v, a, b, ab;
};
inline HD operator+(HD x, HD y) { return {x.v + y.v, x.a + y.a, x.b + y.b, x.ab + y.ab}; }
inline HD operator-(HD x, HD y) { return {x.v - y.v, x.a - y.a, x.b - y.b, x.ab - y.ab}; }
inline HD operator*(HD x, HD y) {
  return {x.v * y.v, x.a * y.v + x.v * y.a, x.b * y.v + x.v * y.b, x.ab * y.v + x.a * y.b + x.b * y.a + x.v * y.ab};
}
// f(x) from f, f' and f'' at x.v
inline HD chain(HD x, double f, double f1, double f2) {
  return {f, f1 * x.a, f1 * x.b, f1 * x.ab + f2 * x.a * x.b};
}
inline HD operator/(HD x, HD y) {
  const double r = 1 / y.v;
  return x * chain(y, r, -r * r, 2 * r * r * r);
}
inline HD hsqrt(HD x) {
  const double s = std::sqrt(x.v);
  return chain(x, s, 0.5 / s, -0.25 / (s * s * s));
}
// atan2(y, x): first partials (x, -y) / r^2, second (-2xy, 2xy, y^2 - x^2) / r^4
// for (yy, xx, xy); defined at every angle.
inline HD hatan2(HD y, HD x) {
  const double r2 = x.v * x.v + y.v * y.v, r4 = r2 * r2;
  const double fy = x.v / r2, fx = -y.v / r2;
  const double fyy = -2 * x.v * y.v / r4, fxx = 2 * x.v * y.v / r4, fxy = (y.v * y.v - x.v * x.v) / r4;
  return {std::atan2(y.v, x.v), fy * y.a + fx * x.a, fy * y.b + fx * x.b,
          fy * y.ab + fx * x.ab + fyy * y.a * y.b + fxx * x.a * x.b + fxy * (x.a * y.b + y.a * x.b)};
}

// Signed bend angle phi of a hinge (v0, v1 shared; v2, v3 the wings) from its
// 12 coordinates: with e0 = x1 - x0, n1 = e0 x (x2 - x0) and m2 = (x3 - x0) x e0
// (the second normal flipped, so a flat hinge has phi = 0),
// phi = atan2((n1 x m2) . e0 / |e0|, n1 . m2). The reference's dihedral
// (mesh.ts:129-140), acos of the normals' cosine, equals pi - |phi|.
HD bend_phi(const HD* q) {
  HD e0[3], e1[3], e2[3];
  for (int i = 0; i < 3; i++) {
    e0[i] = q[3 + i] - q[i];
    e1[i] = q[6 + i] - q[i];
    e2[i] = q[9 + i] - q[i];
  }
  auto cross = [](const HD* a, const HD* b, HD* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
  };
  HD n1[3], m2[3], c[3];
  cross(e0, e1, n1);
  cross(e2, e0, m2);
  cross(n1, m2, c);
  const HD el = hsqrt(e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2]);
  const HD s = (c[0] * e0[0] + c[1] * e0[1] + c[2] * e0[2]) / el;
  const HD co = n1[0] * m2[0] + n1[1] * m2[1] + n1[2] * m2[2];
  return hatan2(s, co);
}

// phi, its gradient, and (when hphi) its 12x12 Hessian at q12.
double bend_phi_derivs(const double* q12, double* dphi, double* hphi) {
  HD q[12];
  for (int j = 0; j < 12; j++) q[j] = {q12[j], 0.0, 0.0, 0.0};
  double phi = 0;
  for (int i = 0; i < 12; i++) {
    q[i].a = 1;
    if (!hphi) {
      const HD p = bend_phi(q);
      phi = p.v;
      dphi[i] = p.a;
    } else {
      for (int j = i; j < 12; j++) {
        q[j].b = 1;
        const HD p = bend_phi(q);
        q[j].b = 0;
        phi = p.v;
        if (j == i) dphi[i] = p.a;
        hphi[i * 12 + j] = hphi[j * 12 + i] = p.ab;
      }
    }
    q[i].a = 0;
  }
  return phi;
}

}  // namespace

// E = k w (theta - rest)^2 / 2 with theta = pi - |phi|, w = edgeLen^2 / areaSum
// (bending.ts:7-16): grad E = -k w (theta - rest) sgn(phi) grad phi.
void hinge_grad_exact(const double* q12, double restAngle, double edgeLen, double areaSum, double k,
                      double* g12) {
  const double w = edgeLen * edgeLen / js_max(areaSum, 1e-12);
  double dphi[12];
  const double phi = bend_phi_derivs(q12, dphi, nullptr);
  const double theta = M_PI - std::fabs(phi);
  const double c = -k * w * (theta - restAngle) * (phi >= 0 ? 1.0 : -1.0);
  for (int j = 0; j < 12; j++) g12[j] = c * dphi[j];
}

// Hessian of the same energy: k w (grad phi grad phi^T - (theta - rest) sgn(phi) Hess phi).
void hinge_hess_exact(const double* q12, double restAngle, double edgeLen, double areaSum, double k,
                      double* h144) {
  const double w = edgeLen * edgeLen / js_max(areaSum, 1e-12);
  double dphi[12], hphi[144];
  const double phi = bend_phi_derivs(q12, dphi, hphi);
  const double theta = M_PI - std::fabs(phi);
  const double c = -(theta - restAngle) * (phi >= 0 ? 1.0 : -1.0);
  for (int i = 0; i < 12; i++)
    for (int j = 0; j < 12; j++) h144[i * 12 + j] = k * w * (dphi[i] * dphi[j] + c * hphi[i * 12 + j]);
}

void hinge_hessians(const double* x, const Mesh& mesh, const Material& mat, std::vector<double>& out) {
  const double kb = 0.5 * (mat.bendWarp + mat.bendWeft);
  out.assign(mesh.hinges.size() * 144, 0.0);
  if (kb <= 0) return;
  for (size_t hI = 0; hI < mesh.hinges.size(); hI++) {
    const Hinge& h = mesh.hinges[hI];
    const int vs[4] = {h.v0, h.v1, h.v2, h.v3};
    double q[12];
    for (int a = 0; a < 4; a++)
      for (int i = 0; i < 3; i++) q[a * 3 + i] = x[vs[a] * 3 + i];
    hinge_hess_exact(q, h.restAngle, h.edgeLen, h.areaSum, kb, out.data() + hI * 144);
  }
}

FemEval eval_internal_exact(const double* x, const Mesh& mesh, const Material& mat, double* grad) {
  std::fill(grad, grad + mesh.n * 3, 0.0);
  double energy = 0, maxStrain = 0;
  TriGrad r;
  for (int t = 0; t < mesh.m; t++) {
    const uint32_t vs[3] = {mesh.idx[t * 3], mesh.idx[t * 3 + 1], mesh.idx[t * 3 + 2]};
    double p[3][3], inv[4];
    for (int v = 0; v < 3; v++)
      for (int i = 0; i < 3; i++) p[v][i] = x[vs[v] * 3 + i];
    for (int k = 0; k < 4; k++) inv[k] = mesh.invDm[t * 4 + k];
    tri_energy_grad(p[0], p[1], p[2], inv, mesh.areas[t], mat, r);
    energy += r.energy;
    maxStrain = js_max(js_max(js_max(maxStrain, std::fabs(r.E00)), std::fabs(r.E11)), std::fabs(r.E01));
    for (int v = 0; v < 3; v++)
      for (int i = 0; i < 3; i++) grad[vs[v] * 3 + i] += r.grad[v * 3 + i];
  }
  const double kb = 0.5 * (mat.bendWarp + mat.bendWeft);
  if (kb > 0)
    for (const Hinge& h : mesh.hinges) {
      const int vs[4] = {h.v0, h.v1, h.v2, h.v3};
      double q[12], g[12];
      for (int a = 0; a < 4; a++)
        for (int i = 0; i < 3; i++) q[a * 3 + i] = x[vs[a] * 3 + i];
      energy += hinge_energy(x, h.v0, h.v1, h.v2, h.v3, h.restAngle, h.edgeLen, h.areaSum, kb);
      hinge_grad_exact(q, h.restAngle, h.edgeLen, h.areaSum, kb, g);
      for (int a = 0; a < 4; a++)
        for (int i = 0; i < 3; i++) grad[vs[a] * 3 + i] += g[a * 3 + i];
    }
  return {energy, maxStrain};
}

// The positive part of a symmetric 2x2 stress [[s00, s01], [s01, s11]].
void stress_positive_part(double& s00, double& s11, double& s01) {
  const double mean = 0.5 * (s00 + s11), half = 0.5 * (s00 - s11);
  const double rad = std::sqrt(half * half + s01 * s01);
  const double hi = mean + rad, lo = mean - rad;
  if (lo >= 0) return;
  if (hi <= 0) {
    s00 = s11 = s01 = 0;
    return;
  }
  // eigenvector of hi: (s01, hi - s00), or (hi - s11, s01) when that vanishes
  double ex = s01, ey = hi - s00;
  if (ex * ex + ey * ey < 1e-300) { ex = hi - s11; ey = s01; }
  double nn = ex * ex + ey * ey;
  if (nn < 1e-300) { ex = s00 >= s11 ? 1 : 0; ey = 1 - ex; nn = 1; }
  const double inv = 1 / std::sqrt(nn);
  ex *= inv;
  ey *= inv;
  s00 = hi * ex * ex;
  s11 = hi * ey * ey;
  s01 = hi * ex * ey;
}

// membrane-hvp.ts:18-75 triangleHvp with S+ in the geometric term dF S.
static void tri_hvp_psd(const double* x0, const double* x1, const double* x2, const double* v0, const double* v1,
                        const double* v2, const double* inv, double area, const Material& mat, double out[9]) {
  const double a = inv[0], b = inv[1], c = inv[2], d = inv[3];
  double F[2][3], dF[2][3];
  for (int i = 0; i < 3; i++) {
    const double e1 = x1[i] - x0[i], e2 = x2[i] - x0[i], w1 = v1[i] - v0[i], w2 = v2[i] - v0[i];
    F[0][i] = a * e1 + c * e2;
    F[1][i] = b * e1 + d * e2;
    dF[0][i] = a * w1 + c * w2;
    dF[1][i] = b * w1 + d * w2;
  }
  auto dot = [](const double* u, const double* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; };
  const double E00 = 0.5 * (dot(F[0], F[0]) - 1), E11 = 0.5 * (dot(F[1], F[1]) - 1), E01 = 0.5 * dot(F[0], F[1]);
  const double dE00 = dot(F[0], dF[0]), dE11 = dot(F[1], dF[1]), dE01 = 0.5 * (dot(dF[0], F[1]) + dot(F[0], dF[1]));
  double S00 = mat.C00 * E00 + mat.C01 * E11, S11 = mat.C11 * E11 + mat.C01 * E00, S01 = 2 * mat.G * E01;
  const double dS00 = mat.C00 * dE00 + mat.C01 * dE11, dS11 = mat.C11 * dE11 + mat.C01 * dE00,
               dS01 = 2 * mat.G * dE01;
  stress_positive_part(S00, S11, S01);
  const double s = mat.thickness * area;
  for (int i = 0; i < 3; i++) {
    const double P0 = dF[0][i] * S00 + dF[1][i] * S01 + F[0][i] * dS00 + F[1][i] * dS01;
    const double P1 = dF[0][i] * S01 + dF[1][i] * S11 + F[0][i] * dS01 + F[1][i] * dS11;
    const double g1 = s * (P0 * a + P1 * b), g2 = s * (P0 * c + P1 * d);
    out[i] = -(g1 + g2);
    out[3 + i] = g1;
    out[6 + i] = g2;
  }
}

void internal_hvp_exact(const double* x, const double* p, const Mesh& mesh, const Material& mat, double* out,
                        const double* hinH) {
  std::fill(out, out + mesh.n * 3, 0.0);
  for (int t = 0; t < mesh.m; t++) {
    const uint32_t vs[3] = {mesh.idx[t * 3], mesh.idx[t * 3 + 1], mesh.idx[t * 3 + 2]};
    double xv[3][3], pv[3][3], inv[4], o[9];
    for (int v = 0; v < 3; v++)
      for (int i = 0; i < 3; i++) { xv[v][i] = x[vs[v] * 3 + i]; pv[v][i] = p[vs[v] * 3 + i]; }
    for (int k = 0; k < 4; k++) inv[k] = mesh.invDm[t * 4 + k];
    tri_hvp_psd(xv[0], xv[1], xv[2], pv[0], pv[1], pv[2], inv, mesh.areas[t], mat, o);
    for (int v = 0; v < 3; v++)
      for (int i = 0; i < 3; i++) out[vs[v] * 3 + i] += o[v * 3 + i];
  }
  // bending: the exact hinge Hessian along p (precomputed in hinH, 144 per hinge, or here)
  const double kb = 0.5 * (mat.bendWarp + mat.bendWeft);
  if (kb <= 0) return;
  double own[144];
  for (size_t hI = 0; hI < mesh.hinges.size(); hI++) {
    const Hinge& h = mesh.hinges[hI];
    const int vs[4] = {h.v0, h.v1, h.v2, h.v3};
    double pq[12];
    for (int a = 0; a < 4; a++)
      for (int i = 0; i < 3; i++) pq[a * 3 + i] = p[vs[a] * 3 + i];
    const double* H = hinH ? hinH + hI * 144 : own;
    if (!hinH) {
      double q[12];
      for (int a = 0; a < 4; a++)
        for (int i = 0; i < 3; i++) q[a * 3 + i] = x[vs[a] * 3 + i];
      hinge_hess_exact(q, h.restAngle, h.edgeLen, h.areaSum, kb, own);
    }
    for (int r = 0; r < 12; r++) {
      double sum = 0;
      for (int c = 0; c < 12; c++) sum += H[r * 12 + c] * pq[c];
      out[vs[r / 3] * 3 + r % 3] += sum;
    }
  }
}

// ---- friction as a frozen potential ---------------------------------------------

// Slip Jacobian of relativeSlip (contact-assembly.ts:344-367) as (vertex, weight)
// terms: VT reads its third triangle vertex as D(c.d) (a static id, zero
// displacement), so that vertex has no term.
static int slip_terms(const Frozen& c, int vs[4], double ws[4]) {
  if (c.kind == 2) { vs[0] = c.p; ws[0] = 1; return 1; }
  if (c.kind == 0) {
    vs[0] = c.p; ws[0] = 1;
    vs[1] = c.a; ws[1] = -c.w0;
    vs[2] = c.b; ws[2] = -c.w1;
    return 3;
  }
  vs[0] = c.a; ws[0] = c.w0;
  vs[1] = c.b; ws[1] = c.w1;
  vs[2] = c.c; ws[2] = c.w2;
  vs[3] = c.d; ws[3] = c.w3;
  return 4;
}

void ContactSystem::friction_potential_freeze(const double* x) {
  const double dHat = params.dHat, kappa = params.kappa, mu = params.mu, eps = params.eps;
  fric.assign(active.size(), FricTerm{});
  for (size_t i = 0; i < active.size(); i++) {
    const Frozen& c = active[i];
    const double d = js_max(frozen_dist(x, c), 1e-12);
    if (d >= dHat) continue;
    auto it = lagged.find(contact_key(c));
    const bool has = it != lagged.end();
    FricTerm& f = fric[i];
    f.nx = has ? it->second.nx : c.nx;
    f.ny = has ? it->second.ny : c.ny;
    f.nz = has ? it->second.nz : c.nz;
    const double lambdaN = has ? it->second.lambdaN : barrier_normal_force(d, dHat, kappa, 1);
    f.ml = mu * js_max(0, lambdaN);
    double u[3];
    relative_slip(x, c, u);
    const double un = u[0] * f.nx + u[1] * f.ny + u[2] * f.nz;
    f.tx = u[0] - un * f.nx; f.ty = u[1] - un * f.ny; f.tz = u[2] - un * f.nz;
    f.r = std::sqrt(f.tx * f.tx + f.ty * f.ty + f.tz * f.tz + eps * eps);
  }
}

double ContactSystem::friction_potential(const double* x) const {
  const double eps = params.eps;
  double e = 0;
  for (size_t i = 0; i < fric.size(); i++) {
    const FricTerm& f = fric[i];
    if (f.ml == 0) continue;
    double u[3];
    relative_slip(x, active[i], u);
    const double un = u[0] * f.nx + u[1] * f.ny + u[2] * f.nz;
    const double t[3] = {u[0] - un * f.nx, u[1] - un * f.ny, u[2] - un * f.nz};
    e += f.ml * std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2] + eps * eps);
  }
  return e;
}

// Hessian of the frozen potential along v: (ml / r) (P du - t (t . P du) / r^2)
// with du the slip Jacobian applied to v, scattered back through it.
void ContactSystem::friction_hvp(const double* v, double* out, int n3) const {
  std::fill(out, out + n3, 0.0);
  for (size_t i = 0; i < fric.size(); i++) {
    const FricTerm& f = fric[i];
    if (f.ml == 0) continue;
    int vs[4];
    double ws[4];
    const int nt = slip_terms(active[i], vs, ws);
    double du[3] = {0, 0, 0};
    for (int k = 0; k < nt; k++) {
      if (vs[k] < 0) continue;
      for (int a = 0; a < 3; a++) du[a] += ws[k] * v[vs[k] * 3 + a];
    }
    const double nd = du[0] * f.nx + du[1] * f.ny + du[2] * f.nz;
    const double pu[3] = {du[0] - nd * f.nx, du[1] - nd * f.ny, du[2] - nd * f.nz};
    const double td = (pu[0] * f.tx + pu[1] * f.ty + pu[2] * f.tz) / (f.r * f.r);
    const double s = f.ml / f.r;
    const double F[3] = {s * (pu[0] - td * f.tx), s * (pu[1] - td * f.ty), s * (pu[2] - td * f.tz)};
    for (int k = 0; k < nt; k++) {
      if (vs[k] < 0) continue;
      for (int a = 0; a < 3; a++) out[vs[k] * 3 + a] += ws[k] * F[a];
    }
  }
}

// ---- the step ----------------------------------------------------------------

// implicit_step (newton.ts:27-232) in the CUDA solver's exact-Newton mode. What
// differs from the reference step:
//   - the first iterate is x0 + h v when drift is set (yHat stays the inertial
//     target of the energy);
//   - the gradient takes the exact hinge gradient;
//   - every Newton iteration freezes the lagged friction at x as a potential,
//     which enters the merit and the Newton matrix (whose membrane part has its
//     stress clamped to the positive part);
//   - every Newton iteration re-evaluates the Armijo base energy at x with its
//     active set and friction potential (the reference keeps the previous
//     trial's energy, which misses contacts that entered the set since);
//   - PCG runs to pcgTol;
//   - once gradNorm < 1e-7 a CCD-valid full step is taken without the Armijo
//     test, whose energy decrease is then below the rounding of the sums.
// The gradient itself (barrier and the reference's friction force) is the
// reference's, so a converged step is a stationary point of the same equations.
StepStats implicit_step_exact(Scene& scene, double h, const StepperOptions& opts,
                              const SchwarzDomains* domains, double pcgTol, bool drift) {
  const int newtonIters = opts.newtonIters, pcgMaxIters = opts.pcgMaxIters, lsIters = opts.lsIters;
  const double gradTol = opts.gradTol;
  const Mesh& mesh = scene.mesh;
  const int n = mesh.n, n3 = n * 3;
  const float* M = mesh.masses.data();
  const Vec x0 = scene.positions;
  const double* v0 = scene.velocities.data();
  const double gv[3] = {scene.gravity[0], scene.gravity[1], scene.gravity[2]};
  Vec yHat(n3), x(n3);
  for (int i = 0; i < n3; i++) {
    yHat[i] = x0[i] + h * v0[i] + h * h * gv[i % 3];
    x[i] = drift ? x0[i] + h * v0[i] : yHat[i];
  }
  enforce_pins(scene, x.data());
  auto filter = [&](double* v) { pin_filter(scene, v); };
  ContactSystem* contact = scene.contact;
  if (contact) {
    contact->fric.clear();
    contact->begin_step(x0.data(), n3);
    if (!contact->check_trial(x.data(), n3).valid) {
      double lo = 0, hi = 1;
      Vec probe(n3);
      for (int b = 0; b < 8; b++) {
        const double mid = 0.5 * (lo + hi);
        for (int i = 0; i < n3; i++) probe[i] = x0[i] + mid * (x[i] - x0[i]);
        enforce_pins(scene, probe.data());
        if (contact->check_trial(probe.data(), n3).valid) lo = mid;
        else hi = mid;
        if (hi - lo < 1e-4) break;
      }
      for (int i = 0; i < n3; i++) x[i] = x0[i] + lo * (x[i] - x0[i]);
      enforce_pins(scene, x.data());
    }
  }
  const Material& mat = scene.material;
  const bool fricOn = contact && contact->params.mu > 0;
  auto total_energy = [&](const double* xx) {
    double e = 0;
    for (int i = 0; i < n3; i++) {
      const double d = xx[i] - yHat[i];
      e += 0.5 * M[i / 3] * d * d / (h * h);
    }
    e += internal_energy_only(xx, mesh, mat);
    if (contact) e += contact->merit_energy(xx) + contact->friction_potential(xx);
    return e;
  };
  if (contact) contact->update_active_set(x.data(), n3);
  double energy = total_energy(x.data());
  double gradNorm = INF, maxStrain = 0;
  int pcgItersTotal = 0, itersUsed = 0, trials = 0;
  bool converged = false;
  const double invH2 = 1 / (h * h);
  const double beta = js_max(js_max(mat.C00, mat.C11), mat.G) * mat.thickness * 0.1 + 1e-6;
  Vec diag(n3);
  for (int i = 0; i < n3; i++) diag[i] = M[i / 3] * invH2 + beta;
  Vec cHp(n3), fHp(n3), egrad(n3), cgrad(n3), g(n3), b(n3), Hp(n3), xt(n3);
  SchwarzFactors sf;
  BlockFactors bf;
  std::vector<double> hinH;
  for (int ni = 0; ni < newtonIters; ni++) {
    itersUsed = ni + 1;
    const FemEval ev = eval_internal_exact(x.data(), mesh, mat, egrad.data());
    maxStrain = ev.maxStrain;
    for (int i = 0; i < n3; i++) g[i] = M[i / 3] * (x[i] - yHat[i]) * invH2 + egrad[i];
    if (contact) {
      contact->update_active_set(x.data(), n3);
      contact->energy_grad(x.data(), cgrad.data(), n3);
      for (int i = 0; i < n3; i++) g[i] += cgrad[i];
      contact->add_diag_estimate(diag.data(), x.data());
      if (fricOn) contact->friction_potential_freeze(x.data());
      energy = total_energy(x.data());
    }
    filter(g.data());
    double gs = 0;
    for (int i = 0; i < n3; i++) gs += g[i] * g[i];
    gradNorm = std::sqrt(gs);
    if (!std::isfinite(gradNorm)) throw std::runtime_error("non-finite gradient");
    if (gradNorm < gradTol) { converged = true; break; }
    for (int i = 0; i < n3; i++) b[i] = -g[i];
    hinge_hessians(x.data(), mesh, mat, hinH);
    auto hvp = [&](const Vec& p, Vec& out) {
      internal_hvp_exact(x.data(), p.data(), mesh, mat, Hp.data(), hinH.data());
      for (int i = 0; i < n3; i++) out[i] = M[i / 3] * p[i] * invH2 + Hp[i];
      if (contact) {
        contact->apply_hvp(x.data(), p.data(), cHp.data(), n3);
        for (int i = 0; i < n3; i++) out[i] += cHp[i];
        if (fricOn) {
          contact->friction_hvp(p.data(), fHp.data(), n3);
          for (int i = 0; i < n3; i++) out[i] += fHp[i];
        }
      }
    };
    std::function<void(const Vec&, Vec&)> prec;
    Vec coarseDiag;
    if (opts.precond == PRECOND_SCHWARZ) {
      build_schwarz_factors(x.data(), mesh, mat, diag.data(), *domains, sf);
      prec = [&](const Vec& r, Vec& z) { apply_schwarz(sf, r.data(), z.data(), n); };
    } else if (opts.precond == PRECOND_MAS2) {
      build_schwarz_factors(x.data(), mesh, mat, diag.data(), *domains, sf);
      coarseDiag = build_coarse_diag(x.data(), mesh, mat, diag.data(), *domains);
      prec = [&](const Vec& r, Vec& z) { apply_mas2(sf, coarseDiag, 0.5, r.data(), z.data(), n); };
    } else if (opts.precond == PRECOND_BLOCK) {
      build_block_factors(x.data(), mesh, mat, diag.data(), bf);
      prec = [&](const Vec& r, Vec& z) { apply_block_factors(bf, r.data(), z.data(), n); };
    }
    Vec dx;
    const PcgResult res = pcg(b, hvp, diag, pcgMaxIters, pcgTol, filter, true, prec ? &prec : nullptr, dx);
    pcgItersTotal += res.iters;
    double gtdx = 0;
    for (int i = 0; i < n3; i++) gtdx += g[i] * dx[i];
    if (!std::isfinite(gtdx) || gtdx >= 0) {
      for (int i = 0; i < n3; i++) dx[i] = -g[i] / diag[i];
      gtdx = 0;
      for (int i = 0; i < n3; i++) gtdx += g[i] * dx[i];
    }
    double maxDx = 0;
    for (int i = 0; i < n3; i++) maxDx = std::max(maxDx, std::fabs(dx[i]));
    if (maxDx > 0.002) {
      const double s = 0.002 / maxDx;
      for (int i = 0; i < n3; i++) dx[i] *= s;
      gtdx *= s;
    }
    double alpha = 1;
    bool accepted = false;
    for (int li = 0; li < lsIters; li++) {
      trials++;
      for (int i = 0; i < n3; i++) xt[i] = x[i] + alpha * dx[i];
      enforce_pins(scene, xt.data());
      if (contact && !contact->check_trial(xt.data(), n3).valid) {
        contact->add_rejection();
        alpha *= 0.5;
        continue;
      }
      const double eNew = total_energy(xt.data());
      if (!std::isfinite(eNew)) {
        if (contact) contact->add_rejection();
        alpha *= 0.5;
        continue;
      }
      const bool nearConverged = gradNorm < 1e-7 && alpha == 1;
      if (nearConverged || eNew <= energy + 1e-4 * alpha * gtdx) {
        x = xt;
        energy = eNew;
        accepted = true;
        if (contact) contact->commit(xt.data());
        break;
      }
      if (contact) contact->add_rejection();
      alpha *= 0.5;
    }
    if (!accepted) break;
    if (alpha < 1e-6) break;
  }
  if (contact) contact->fric.clear();
  const double damp = 1 - js_min(js_max(mat.damping, 0), 0.1);
  for (int i = 0; i < n3; i++) scene.velocities[i] = ((x[i] - x0[i]) / h) * damp;
  if (contact) kill_approach_velocity(*contact, scene, x.data());
  scene.positions = x;
  enforce_pins(scene, scene.positions.data());
  StepStats st{};
  st.newtonIters = newtonIters;
  st.pcgIters = pcgItersTotal;
  st.gradNorm = gradNorm;
  st.energy = energy;
  st.maxStrain = maxStrain;
  st.converged = converged;
  st.hasContact = contact != nullptr;
  if (contact) st.contact = contact->diag;
  st.newtonItersUsed = itersUsed;
  st.armijoTrials = trials;
  return st;
}

}  // namespace orc
