// Oracle (test infrastructure only): matrix-free PCG and the implicit-Euler
// Newton step, restated from src/math/pcg.ts and src/solver/newton.ts.
#include <algorithm>
#include <functional>
#include <stdexcept>

#include "orc.hpp"
#include "orc_pcg.hpp"

namespace orc {

// src/physics/scene.ts:38-55 enforcePins / makePinFilter.
void enforce_pins(const Scene& s, double* x) {
  for (size_t k = 0; k < s.pinIds.size(); k++) {
    const int id = s.pinIds[k];
    x[id * 3] = s.pinPos[k * 3];
    x[id * 3 + 1] = s.pinPos[k * 3 + 1];
    x[id * 3 + 2] = s.pinPos[k * 3 + 2];
  }
}
void pin_filter(const Scene& s, double* v) {
  for (int id : s.pinIds) { v[id * 3] = 0; v[id * 3 + 1] = 0; v[id * 3 + 2] = 0; }
}

// src/solver/newton.ts:238-303 killApproachVelocity (restitution 0, one
// deterministic sweep over the active list; each contact sees earlier updates).
void kill_approach_velocity(ContactSystem& contact, Scene& scene, const double* x) {
  const int n3 = (int)scene.positions.size();
  contact.update_active_set(x, n3);
  double* v = scene.velocities.data();
  for (const Frozen& c : contact.active) {
    if (c.kind == 2) {
      const double vy = v[c.p * 3 + 1];
      if (vy < 0) v[c.p * 3 + 1] = 0;
      continue;
    }
    if (c.kind == 0) {
      const double vp[3] = {v[c.p * 3], v[c.p * 3 + 1], v[c.p * 3 + 2]};
      double tx = 0, ty = 0, tz = 0;
      const double ws[3] = {c.w0, c.w1, c.w2};
      const int vs[3] = {c.a, c.b, c.c};
      for (int k = 0; k < 3; k++) {
        if (vs[k] < 0) continue;
        tx += ws[k] * v[vs[k] * 3];
        ty += ws[k] * v[vs[k] * 3 + 1];
        tz += ws[k] * v[vs[k] * 3 + 2];
      }
      const double rel = (vp[0] - tx) * c.nx + (vp[1] - ty) * c.ny + (vp[2] - tz) * c.nz;
      if (rel < 0) {
        const double j = -0.5 * rel;
        v[c.p * 3] += j * c.nx;
        v[c.p * 3 + 1] += j * c.ny;
        v[c.p * 3 + 2] += j * c.nz;
        for (int k = 0; k < 3; k++) {
          if (vs[k] < 0) continue;
          v[vs[k] * 3] -= j * ws[k] * c.nx;
          v[vs[k] * 3 + 1] -= j * ws[k] * c.ny;
          v[vs[k] * 3 + 2] -= j * ws[k] * c.nz;
        }
      }
      continue;
    }
    auto avg = [&](int a, int b, double o[3]) {
      double xa[3] = {0, 0, 0}, xb[3] = {0, 0, 0};
      if (a >= 0) { xa[0] = v[a * 3]; xa[1] = v[a * 3 + 1]; xa[2] = v[a * 3 + 2]; }
      if (b >= 0) { xb[0] = v[b * 3]; xb[1] = v[b * 3 + 1]; xb[2] = v[b * 3 + 2]; }
      for (int i = 0; i < 3; i++) o[i] = (xa[i] + xb[i]) / 2;
    };
    double A[3], C[3];
    avg(c.a, c.b, A);
    avg(c.c, c.d, C);
    const double rel = (A[0] - C[0]) * c.nx + (A[1] - C[1]) * c.ny + (A[2] - C[2]) * c.nz;
    if (rel < 0) {
      const double j = -0.25 * rel;
      for (int vv : {c.a, c.b}) {
        if (vv < 0) continue;
        v[vv * 3] += j * c.nx; v[vv * 3 + 1] += j * c.ny; v[vv * 3 + 2] += j * c.nz;
      }
      for (int vv : {c.c, c.d}) {
        if (vv < 0) continue;
        v[vv * 3] -= j * c.nx; v[vv * 3 + 1] -= j * c.ny; v[vv * 3 + 2] -= j * c.nz;
      }
    }
  }
}

// src/solver/newton.ts:27-232 implicitStep. The preconditioner option wires
// src/solver/schwarz.ts (or block-jacobi.ts) through pcg's applyPreconditioner
// the way tests/preconditioner-compare.test.ts:145,234-236 does, with factors
// rebuilt once per Newton iteration from the Jacobi diagonal.
StepStats implicit_step(Scene& scene, double h, const StepperOptions& opts,
                        const SchwarzDomains* domains) {
  const int newtonIters = opts.newtonIters, pcgMaxIters = opts.pcgMaxIters, lsIters = opts.lsIters;
  const double gradTol = opts.gradTol;
  const Mesh& mesh = scene.mesh;
  const int n = mesh.n, n3 = n * 3;
  const float* M = mesh.masses.data();
  const Vec x0 = scene.positions;
  const double* v0 = scene.velocities.data();
  const double gx = scene.gravity[0], gy = scene.gravity[1], gz = scene.gravity[2];
  Vec yHat(n3);
  for (int i = 0; i < n; i++) {
    yHat[i * 3] = x0[i * 3] + h * v0[i * 3] + h * h * gx;
    yHat[i * 3 + 1] = x0[i * 3 + 1] + h * v0[i * 3 + 1] + h * h * gy;
    yHat[i * 3 + 2] = x0[i * 3 + 2] + h * v0[i * 3 + 2] + h * h * gz;
  }
  Vec x = yHat;
  enforce_pins(scene, x.data());
  auto filter = [&](double* v) { pin_filter(scene, v); };
  ContactSystem* contact = scene.contact;
  if (contact) {
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
  auto total_energy = [&](const double* xx) {
    double e = 0;
    for (int i = 0; i < n; i++) {
      const double m = M[i];
      for (int k = 0; k < 3; k++) {
        const double d = xx[i * 3 + k] - yHat[i * 3 + k];
        e += 0.5 * m * d * d / (h * h);
      }
    }
    e += internal_energy_only(xx, mesh, scene.material);
    if (contact) e += contact->merit_energy(xx);
    return e;
  };
  double energy = 0;
  if (contact) contact->update_active_set(x.data(), n3);
  energy = total_energy(x.data());
  double gradNorm = INF, maxStrain = 0;
  int pcgItersTotal = 0, itersUsed = 0, trials = 0;
  bool converged = false;
  const double invH2 = 1 / (h * h);
  const Material& mat = scene.material;
  const double beta = js_max(js_max(mat.C00, mat.C11), mat.G) * mat.thickness * 0.1 + 1e-6;
  Vec diag(n3);
  for (int i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) diag[i * 3 + k] = M[i] * invH2 + beta;
  Vec cHp(n3), egrad(n3), cgrad(n3), g(n3), b(n3), Hp(n3), xt(n3);
  SchwarzFactors sf;
  BlockFactors bf;
  for (int ni = 0; ni < newtonIters; ni++) {
    itersUsed = ni + 1;
    const FemEval ev = eval_internal(x.data(), mesh, mat, egrad.data());
    maxStrain = ev.maxStrain;
    for (int i = 0; i < n3; i++) {
      const int vi = i / 3;
      g[i] = M[vi] * (x[i] - yHat[i]) * invH2 + egrad[i];
    }
    if (contact) {
      contact->update_active_set(x.data(), n3);
      contact->energy_grad(x.data(), cgrad.data(), n3);
      for (int i = 0; i < n3; i++) g[i] += cgrad[i];
      contact->add_diag_estimate(diag.data(), x.data());
    }
    filter(g.data());
    double gs = 0;
    for (int i = 0; i < n3; i++) gs = gs + g[i] * g[i];
    gradNorm = std::sqrt(gs);
    if (!std::isfinite(gradNorm)) throw std::runtime_error("non-finite gradient — blow up; reduce dt/stiffness");
    if (gradNorm < gradTol) { converged = true; break; }
    for (int i = 0; i < n3; i++) b[i] = -g[i];
    auto hvpFull = [&](const Vec& p, Vec& out) {
      membrane_hvp(x.data(), p.data(), mesh, mat, Hp.data());
      for (int i = 0; i < n3; i++) {
        const int vi = i / 3;
        out[i] = M[vi] * p[i] * invH2 + Hp[i];
      }
      if (contact) {
        contact->apply_hvp(x.data(), p.data(), cHp.data(), n3);
        for (int i = 0; i < n3; i++) out[i] += cHp[i];
      }
    };
    std::function<void(const Vec&, Vec&)> prec;
    Vec coarseDiag;
    if (opts.precond == PRECOND_SCHWARZ) {
      build_schwarz_factors(x.data(), mesh, mat, diag.data(), *domains, sf);
      prec = [&](const Vec& r, Vec& z) { apply_schwarz(sf, r.data(), z.data(), n); };
    } else if (opts.precond == PRECOND_MAS2) {
      // two-level Schwarz (src/solver/mas.ts buildMasTwoLevel / applyMasTwoLevel, omega 0.5)
      build_schwarz_factors(x.data(), mesh, mat, diag.data(), *domains, sf);
      coarseDiag = build_coarse_diag(x.data(), mesh, mat, diag.data(), *domains);
      prec = [&](const Vec& r, Vec& z) { apply_mas2(sf, coarseDiag, 0.5, r.data(), z.data(), n); };
    } else if (opts.precond == PRECOND_BLOCK) {
      build_block_factors(x.data(), mesh, mat, diag.data(), bf);
      prec = [&](const Vec& r, Vec& z) { apply_block_factors(bf, r.data(), z.data(), n); };
    }
    Vec dx;
    const PcgResult res = pcg(b, hvpFull, diag, pcgMaxIters, 1e-3, filter, true,
                              prec ? &prec : nullptr, dx);
    pcgItersTotal += res.iters;
    double gtdx = 0;
    for (int i = 0; i < n3; i++) gtdx += g[i] * dx[i];
    if (!std::isfinite(gtdx) || gtdx >= 0) {
      for (int i = 0; i < n3; i++) dx[i] = -g[i] / diag[i];
      gtdx = 0;
      for (int i = 0; i < n3; i++) gtdx += g[i] * dx[i];
    }
    {
      double maxDx = 0;
      for (int i = 0; i < n3; i++) {
        const double m = std::fabs(dx[i]);
        if (m > maxDx) maxDx = m;
      }
      const double TRUST = 0.002;
      if (maxDx > TRUST) {
        const double s = TRUST / maxDx;
        for (int i = 0; i < n3; i++) dx[i] *= s;
        gtdx *= s;
      }
    }
    double alpha = 1;
    bool accepted = false;
    for (int li = 0; li < lsIters; li++) {
      trials++;
      for (int i = 0; i < n3; i++) xt[i] = x[i] + alpha * dx[i];
      enforce_pins(scene, xt.data());
      if (contact) {
        const TrialResult chk = contact->check_trial(xt.data(), n3);
        if (!chk.valid) { contact->add_rejection(); alpha *= 0.5; continue; }
      }
      const double eNew = total_energy(xt.data());
      if (!std::isfinite(eNew)) {
        if (contact) contact->add_rejection();
        alpha *= 0.5;
        continue;
      }
      if (eNew <= energy + 1e-4 * alpha * gtdx) {
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
