// Oracle (test infrastructure only): flat C API over the restatement, loaded
// by tests/ and bench.py's CPU-baseline leg through ctypes (oracle/oracle.py).
// Material = double[9]: arealDensity, thickness, C00, C11, C01, G, bendWarp,
// bendWeft, damping. Contact params = double[5]: dHat, kappa, dMin, mu, eps.
#include <cstring>
#include <stdexcept>

#include "orc.hpp"
#include "orc_pcg.hpp"

using namespace orc;

static Material mat_of(const double* m) {
  Material o;
  o.arealDensity = m[0]; o.thickness = m[1]; o.C00 = m[2]; o.C11 = m[3]; o.C01 = m[4];
  o.G = m[5]; o.bendWarp = m[6]; o.bendWeft = m[7]; o.damping = m[8];
  return o;
}

extern "C" {

int orc_build_grid(int nx, int ny, double w, double h, float* pos, float* uv, uint32_t* idx) {
  std::vector<float> p, u;
  std::vector<uint32_t> ix;
  build_grid(nx, ny, w, h, p, u, ix);
  std::memcpy(pos, p.data(), p.size() * 4);
  std::memcpy(uv, u.data(), u.size() * 4);
  std::memcpy(idx, ix.data(), ix.size() * 4);
  return 0;
}

void* orc_mesh_create(int n, int m, const float* pos, const float* uv, const uint32_t* idx, double density) {
  try {
    std::vector<float> p(pos, pos + n * 3), u(uv, uv + n * 2);
    std::vector<uint32_t> ix(idx, idx + m * 3);
    return new Mesh(preprocess(p, u, ix, density));
  } catch (...) {
    return nullptr;
  }
}
void orc_mesh_destroy(void* h) { delete (Mesh*)h; }
void orc_mesh_counts(void* h, int* out3) {
  Mesh* me = (Mesh*)h;
  out3[0] = me->n; out3[1] = me->m; out3[2] = (int)me->hinges.size();
}
void orc_mesh_arrays(void* h, float* invDm, float* areas, float* masses, int32_t* hinge4, double* hingeMeta3) {
  Mesh* me = (Mesh*)h;
  std::memcpy(invDm, me->invDm.data(), me->invDm.size() * 4);
  std::memcpy(areas, me->areas.data(), me->areas.size() * 4);
  std::memcpy(masses, me->masses.data(), me->masses.size() * 4);
  for (size_t k = 0; k < me->hinges.size(); k++) {
    const Hinge& g = me->hinges[k];
    hinge4[k * 4] = g.v0; hinge4[k * 4 + 1] = g.v1; hinge4[k * 4 + 2] = g.v2; hinge4[k * 4 + 3] = g.v3;
    hingeMeta3[k * 3] = g.restAngle; hingeMeta3[k * 3 + 1] = g.edgeLen; hingeMeta3[k * 3 + 2] = g.areaSum;
  }
}
void orc_incidence(void* h, int kind, uint32_t* offsets, uint32_t* ids, uint32_t* corners, int* nrec) {
  Mesh* me = (Mesh*)h;
  Incidence inc = kind == 0 ? membrane_incidence(*me) : hinge_incidence(*me);
  *nrec = (int)inc.ids.size();
  if (offsets) std::memcpy(offsets, inc.offsets.data(), inc.offsets.size() * 4);
  if (ids) std::memcpy(ids, inc.ids.data(), inc.ids.size() * 4);
  if (corners) std::memcpy(corners, inc.corners.data(), inc.corners.size() * 4);
}

double orc_js_hypot3(double a, double b, double c) { return js_hypot3(a, b, c); }

void orc_tri_energy_grad(const double* x9, const double* inv4, double area, const double* mat, double* out13) {
  TriGrad r;
  tri_energy_grad(x9, x9 + 3, x9 + 6, inv4, area, mat_of(mat), r);
  out13[0] = r.energy;
  for (int i = 0; i < 9; i++) out13[1 + i] = r.grad[i];
  out13[10] = r.E00; out13[11] = r.E11; out13[12] = r.E01;
}
void orc_tri_hvp(const double* x9, const double* v9, const double* inv4, double area, const double* mat, double* out9) {
  tri_hvp(x9, x9 + 3, x9 + 6, v9, v9 + 3, v9 + 6, inv4, area, mat_of(mat), out9);
}
void orc_tri_hessian9(const double* x9, const double* inv4, double area, const double* mat, double* out81) {
  tri_hessian9(x9, x9 + 3, x9 + 6, inv4, area, mat_of(mat), out81);
}
double orc_dihedral(const double* x, int v0, int v1, int v2, int v3) { return dihedral(x, v0, v1, v2, v3); }
double orc_hinge_energy(const double* x, const int* v4, const double* meta3, double k) {
  return hinge_energy(x, v4[0], v4[1], v4[2], v4[3], meta3[0], meta3[1], meta3[2], k);
}

void orc_hinge_grad_exact(const double* q12, const double* meta3, double k, double* g12) {
  hinge_grad_exact(q12, meta3[0], meta3[1], meta3[2], k, g12);
}
void orc_hinge_hess_exact(const double* q12, const double* meta3, double k, double* h144) {
  hinge_hess_exact(q12, meta3[0], meta3[1], meta3[2], k, h144);
}
void orc_stress_positive_part(double* s3) { stress_positive_part(s3[0], s3[1], s3[2]); }
void orc_eval_internal_exact(void* mh, const double* mat, const double* x, double* grad, double* out2) {
  FemEval ev = eval_internal_exact(x, *(Mesh*)mh, mat_of(mat), grad);
  out2[0] = ev.energy; out2[1] = ev.maxStrain;
}
void orc_internal_hvp_exact(void* mh, const double* mat, const double* x, const double* p, double* out) {
  internal_hvp_exact(x, p, *(Mesh*)mh, mat_of(mat), out);
}
// Friction potential of the active contacts frozen at xf: its value at x, its
// Hessian along v (out, 3n) when v is given.
double orc_contact_friction_potential(void* c, const double* xf, const double* x, const double* v, double* out,
                                      int n3) {
  ContactSystem* cs = (ContactSystem*)c;
  cs->friction_potential_freeze(xf);
  if (v) cs->friction_hvp(v, out, n3);
  const double e = cs->friction_potential(x);
  cs->fric.clear();
  return e;
}

void orc_eval_internal(void* mh, const double* mat, const double* x, double* grad, double* out2) {
  FemEval ev = eval_internal(x, *(Mesh*)mh, mat_of(mat), grad);
  out2[0] = ev.energy; out2[1] = ev.maxStrain;
}
double orc_internal_energy_only(void* mh, const double* mat, const double* x) {
  return internal_energy_only(x, *(Mesh*)mh, mat_of(mat));
}
double orc_eval_membrane(void* mh, const double* mat, const double* x, double* grad) {
  return eval_membrane(x, *(Mesh*)mh, mat_of(mat), grad);
}
void orc_membrane_hvp(void* mh, const double* mat, const double* x, const double* p, double* out) {
  membrane_hvp(x, p, *(Mesh*)mh, mat_of(mat), out);
}
void orc_eval_membrane_hvp(void* mh, const double* mat, const double* x, const double* p, double* out) {
  eval_membrane_hvp(x, p, *(Mesh*)mh, mat_of(mat), out);
}
void orc_eval_membrane_blocks(void* mh, const double* mat, const double* x, double* out) {
  eval_membrane_blocks(x, *(Mesh*)mh, mat_of(mat), out);
}

void orc_closest_vt(const double* q12, double* out6) {
  Closest c = closest_vt(q12[0], q12[1], q12[2], q12[3], q12[4], q12[5], q12[6], q12[7], q12[8], q12[9], q12[10], q12[11]);
  out6[0] = c.s; out6[1] = c.t; out6[2] = c.dist; out6[3] = c.rx; out6[4] = c.ry; out6[5] = c.rz;
}
void orc_closest_ee(const double* q12, double* out6) {
  Closest c = closest_ee(q12[0], q12[1], q12[2], q12[3], q12[4], q12[5], q12[6], q12[7], q12[8], q12[9], q12[10], q12[11]);
  out6[0] = c.s; out6[1] = c.t; out6[2] = c.dist; out6[3] = c.rx; out6[4] = c.ry; out6[5] = c.rz;
}
double orc_vt_ccd(const double* P0, const double* P1, double th) { return vt_ccd(P0, P1, th); }
double orc_ee_ccd(const double* P0, const double* P1, double th) { return ee_ccd(P0, P1, th); }
int orc_solve_cubic01(double a3, double a2, double a1, double a0, double* out3) {
  auto r = solve_cubic01(a3, a2, a1, a0);
  for (size_t i = 0; i < r.size() && i < 3; i++) out3[i] = r[i];
  return (int)r.size();
}
double orc_barrier_value(double d, double dHat) { return barrier_value(d, dHat); }
double orc_barrier_grad_scalar(double d, double dHat, double k, double w) { return barrier_grad_scalar(d, dHat, k, w); }
void orc_coulomb_force(const double* u3, const double* n3, double lambdaN, double mu, double eps, double* f3) {
  coulomb_force(u3[0], u3[1], u3[2], n3[0], n3[1], n3[2], lambdaN, mu, eps, f3);
}

// ---- ContactSystem ----
void* orc_contact_create(const double* params5, const uint32_t* idx, int m) {
  ContactParams p{params5[0], params5[1], params5[2], params5[3], params5[4]};
  std::vector<uint32_t> ix(idx, idx + m * 3);
  return new ContactSystem(p, ix);
}
void orc_contact_destroy(void* c) { delete (ContactSystem*)c; }
void orc_contact_set_floor(void* c, int on, double y) { ((ContactSystem*)c)->set_floor(on != 0, y); }
void orc_contact_set_static(void* c, const float* pos, int ns, const uint32_t* idx, int ms) {
  ((ContactSystem*)c)->set_static_mesh(std::vector<float>(pos, pos + ns * 3), std::vector<uint32_t>(idx, idx + ms * 3));
}
void orc_contact_begin_step(void* c, const double* x0, int n3) { ((ContactSystem*)c)->begin_step(x0, n3); }
void orc_contact_update_active_set(void* c, const double* x, int n3) { ((ContactSystem*)c)->update_active_set(x, n3); }
double orc_contact_energy_grad(void* c, const double* x, double* grad, int n3) {
  return ((ContactSystem*)c)->energy_grad(x, grad, n3);
}
void orc_contact_apply_hvp(void* c, const double* x, const double* v, double* out, int n3) {
  ((ContactSystem*)c)->apply_hvp(x, v, out, n3);
}
double orc_contact_merit_energy(void* c, const double* x) { return ((ContactSystem*)c)->merit_energy(x); }
void orc_contact_add_diag_estimate(void* c, double* dg, const double* x) { ((ContactSystem*)c)->add_diag_estimate(dg, x); }
void orc_contact_commit(void* c, const double* x) { ((ContactSystem*)c)->commit(x); }
int orc_contact_check_trial(void* c, const double* xT, int n3, double* out2) {
  TrialResult r = ((ContactSystem*)c)->check_trial(xT, n3);
  out2[0] = r.minDist; out2[1] = r.minTOI;
  return r.valid ? 1 : 0;
}
int orc_contact_active(void* c, int32_t* ids6, double* w7) {
  ContactSystem* cs = (ContactSystem*)c;
  if (ids6)
    for (size_t i = 0; i < cs->active.size(); i++) {
      const Frozen& f = cs->active[i];
      int32_t* o = ids6 + i * 6;
      o[0] = f.kind; o[1] = f.p; o[2] = f.a; o[3] = f.b; o[4] = f.c; o[5] = f.d;
      double* w = w7 + i * 7;
      w[0] = f.w0; w[1] = f.w1; w[2] = f.w2; w[3] = f.w3; w[4] = f.nx; w[5] = f.ny; w[6] = f.nz;
    }
  return (int)cs->active.size();
}
int orc_contact_candidates(void* c, const double* x, double pad, int32_t* ids6, int cap) {
  ContactSystem* cs = (ContactSystem*)c;
  std::vector<Cand> v = cs->build_candidates(x, pad);
  if (ids6)
    for (size_t i = 0; i < v.size() && (int)i < cap; i++) {
      int32_t* o = ids6 + i * 6;
      o[0] = v[i].kind; o[1] = v[i].p; o[2] = v[i].a; o[3] = v[i].b; o[4] = v[i].c; o[5] = v[i].d;
    }
  return (int)v.size();
}
int orc_tri_pairs(const double* x0, const double* x1, const uint32_t* idx, int m, double pad, int32_t* out2, int cap) {
  TriBvh b;
  b.build(x0, x1, idx, m, pad);
  auto ex = adjacency_exclusions(idx, m);
  auto pr = b.self_pairs(ex);
  if (out2)
    for (size_t i = 0; i < pr.size() && (int)i < cap; i++) { out2[i * 2] = pr[i].first; out2[i * 2 + 1] = pr[i].second; }
  return (int)pr.size();
}
void orc_contact_diag(void* c, double* out11) {
  const ContactDiag& d = ((ContactSystem*)c)->diag;
  double v[11] = {d.candidatePairs, d.activePairs, d.vtPairs, d.eePairs, d.floorPairs, d.minDistance,
                  d.minTOI, d.barrierEnergy, d.frictionWork, d.rejectedLineSearchSteps, d.ccdFailures};
  std::memcpy(out11, v, sizeof v);
}

// ---- Schwarz domains ----
void* orc_schwarz_domains(void* mh, const float* rest, int target, int minSize, int maxSize) {
  return new SchwarzDomains(build_schwarz_domains(*(Mesh*)mh, rest, target, minSize, maxSize));
}
void orc_schwarz_destroy(void* d) { delete (SchwarzDomains*)d; }
int orc_schwarz_info(void* d, uint32_t* domainOf, uint32_t* localOf, int n) {
  SchwarzDomains* s = (SchwarzDomains*)d;
  if (domainOf) std::memcpy(domainOf, s->domainOf.data(), n * 4);
  if (localOf) std::memcpy(localOf, s->localOf.data(), n * 4);
  return (int)s->members.size();
}

// PCG on one Newton system as tests/preconditioner-compare.test.ts:91-98,234-237
// builds it: hvpFull = M/h^2 p + FD membrane HVP (+ contact HVP), no pin filter.
// precond: 0 Jacobi, 1 Schwarz (domains required), 2 block-Jacobi.
int orc_pcg_solve(void* mh, const double* mat, const double* x, void* contact, double invH2,
                  const double* diag, const double* b, int maxIters, double tol, int precond,
                  void* domains, double* xout, double* residual_out) {
  Mesh& me = *(Mesh*)mh;
  const Material mt = mat_of(mat);
  const int n = me.n, n3 = n * 3;
  ContactSystem* cs = (ContactSystem*)contact;
  Vec bb(b, b + n3), dg(diag, diag + n3), Hp(n3), cHp(n3), X(x, x + n3);
  auto hvp = [&](const Vec& p, Vec& out) {
    membrane_hvp(X.data(), p.data(), me, mt, Hp.data());
    for (int i = 0; i < n3; i++) out[i] = (double)me.masses[i / 3] * p[i] * invH2 + Hp[i];
    if (cs) {
      cs->apply_hvp(X.data(), p.data(), cHp.data(), n3);
      for (int i = 0; i < n3; i++) out[i] += cHp[i];
    }
  };
  SchwarzFactors sf;
  BlockFactors bf;
  std::function<void(const Vec&, Vec&)> prec;
  if (precond == 1) {
    build_schwarz_factors(X.data(), me, mt, dg.data(), *(SchwarzDomains*)domains, sf);
    prec = [&](const Vec& r, Vec& z) { apply_schwarz(sf, r.data(), z.data(), n); };
  } else if (precond == 2) {
    build_block_factors(X.data(), me, mt, dg.data(), bf);
    prec = [&](const Vec& r, Vec& z) { apply_block_factors(bf, r.data(), z.data(), n); };
  }
  // two-level additive Schwarz: 3 = mas2 (damped-Jacobi coarse, omega 0.5), 4 = masX (exact coarse)
  Vec coarseDiag;
  CoarseExact ce;
  if (precond == 3 || precond == 4) {
    const SchwarzDomains& dom = *(SchwarzDomains*)domains;
    build_schwarz_factors(X.data(), me, mt, dg.data(), dom, sf);
    if (precond == 3) {
      coarseDiag = build_coarse_diag(X.data(), me, mt, dg.data(), dom);
      prec = [&](const Vec& r, Vec& z) { apply_mas2(sf, coarseDiag, 0.5, r.data(), z.data(), n); };
    } else {
      build_coarse_exact(X.data(), me, mt, dg.data(), dom, ce);
      prec = [&](const Vec& r, Vec& z) { apply_masx(sf, ce, r.data(), z.data(), n); };
    }
  }
  Vec xo;
  auto nofilter = [](double*) {};
  PcgResult r = pcg(bb, hvp, dg, maxIters, tol, nofilter, false, prec ? &prec : nullptr, xo);
  std::memcpy(xout, xo.data(), n3 * 8);
  *residual_out = r.residual;
  return r.iters;
}

// ---- scene + implicit step ----
struct SceneBox {
  Scene s;
  SchwarzDomains dom;
  bool hasDom = false;
};
void* orc_scene_create(void* mh, const double* mat, const double* grav3, const double* x, const double* v) {
  SceneBox* b = new SceneBox();
  b->s.mesh = *(Mesh*)mh;
  b->s.material = mat_of(mat);
  for (int k = 0; k < 3; k++) b->s.gravity[k] = grav3[k];
  const int n3 = b->s.mesh.n * 3;
  b->s.positions.assign(x, x + n3);
  b->s.velocities.assign(v, v + n3);
  return b;
}
void orc_scene_destroy(void* h) { delete (SceneBox*)h; }
void orc_scene_set_material(void* h, const double* mat) { ((SceneBox*)h)->s.material = mat_of(mat); }
void orc_scene_set_pins(void* h, int k, const int32_t* ids, const double* pos) {
  Scene& s = ((SceneBox*)h)->s;
  s.pinIds.assign(ids, ids + k);
  s.pinPos.assign(pos, pos + k * 3);
}
void orc_scene_set_contact(void* h, void* contact) { ((SceneBox*)h)->s.contact = (ContactSystem*)contact; }
void orc_scene_set_state(void* h, const double* x, const double* v) {
  Scene& s = ((SceneBox*)h)->s;
  if (x) std::memcpy(s.positions.data(), x, s.positions.size() * 8);
  if (v) std::memcpy(s.velocities.data(), v, s.velocities.size() * 8);
}
void orc_scene_get_state(void* h, double* x, double* v) {
  Scene& s = ((SceneBox*)h)->s;
  if (x) std::memcpy(x, s.positions.data(), s.positions.size() * 8);
  if (v) std::memcpy(v, s.velocities.data(), s.velocities.size() * 8);
}
void orc_scene_build_schwarz(void* h, int target, int minSize, int maxSize) {
  SceneBox* b = (SceneBox*)h;
  b->dom = build_schwarz_domains(b->s.mesh, b->s.mesh.rest.data(), target, minSize, maxSize);
  b->hasDom = true;
}
// Stats out (double[20]): newtonIters, pcgIters, gradNorm, energy, maxStrain,
// converged, hasContact, contact diag[11] (orc_contact_diag order),
// newtonItersUsed, armijoTrials. Returns 0, or 2 on the non-finite-gradient throw.
// exact < 0: the reference step; otherwise exact-Newton mode with PCG tolerance
// pcgTol and the drift start when exact == 1 (implicit_step_exact).
static int step_any(void* h, double dt, int newtonIters, int pcgMaxIters, double gradTol, int lsIters,
                    int precond, int exact, double pcgTol, double* stats20) {
  SceneBox* b = (SceneBox*)h;
  StepperOptions o;
  o.newtonIters = newtonIters; o.pcgMaxIters = pcgMaxIters; o.gradTol = gradTol; o.lsIters = lsIters;
  o.precond = precond;
  if ((precond == PRECOND_SCHWARZ || precond == PRECOND_MAS2) && !b->hasDom) {
    b->dom = build_schwarz_domains(b->s.mesh, b->s.mesh.rest.data(), 8, 1, 8);
    b->hasDom = true;
  }
  try {
    StepStats st = exact < 0 ? implicit_step(b->s, dt, o, &b->dom)
                             : implicit_step_exact(b->s, dt, o, &b->dom, pcgTol, exact == 1);
    const ContactDiag& d = st.contact;
    double v[20] = {(double)st.newtonIters, (double)st.pcgIters, st.gradNorm, st.energy, st.maxStrain,
                    st.converged ? 1.0 : 0.0, st.hasContact ? 1.0 : 0.0, d.candidatePairs, d.activePairs,
                    d.vtPairs, d.eePairs, d.floorPairs, d.minDistance, d.minTOI, d.barrierEnergy,
                    d.frictionWork, d.rejectedLineSearchSteps, d.ccdFailures, (double)st.newtonItersUsed,
                    (double)st.armijoTrials};
    if (stats20) std::memcpy(stats20, v, sizeof v);
    return 0;
  } catch (const std::exception&) {
    return 2;
  }
}
int orc_step(void* h, double dt, int newtonIters, int pcgMaxIters, double gradTol, int lsIters,
             int precond, double* stats20) {
  return step_any(h, dt, newtonIters, pcgMaxIters, gradTol, lsIters, precond, -1, 0, stats20);
}
int orc_step_exact(void* h, double dt, int newtonIters, int pcgMaxIters, double gradTol, int lsIters,
                   int precond, double pcgTol, int drift, double* stats20) {
  return step_any(h, dt, newtonIters, pcgMaxIters, gradTol, lsIters, precond, drift ? 1 : 0, pcgTol, stats20);
}

// ---- FP32 LBVH mirror ----
void* orc_lbvh_build(const double* x0, const double* x1, const uint32_t* idx, int m, double pad, long capacity) {
  LbvhMirror* o = new LbvhMirror();
  auto ex = adjacency_exclusions(idx, m);
  lbvh_mirror_build(x0, x1, idx, m, pad, ex, capacity, *o);
  return o;
}
void orc_lbvh_destroy(void* h) { delete (LbvhMirror*)h; }
// info: root, depth, pairCount, scanned, overflow
void orc_lbvh_info(void* h, long* info5) {
  LbvhMirror* o = (LbvhMirror*)h;
  info5[0] = o->root; info5[1] = o->depth; info5[2] = (long)o->pairs.size(); info5[3] = o->scanned; info5[4] = o->overflow;
}
void orc_lbvh_arrays(void* h, float* aabb, float* centroid, uint32_t* morton, uint32_t* payload, float* nodeMin,
                     float* nodeMax, int32_t* left, int32_t* right, int32_t* leafTri, int32_t* pairs2) {
  LbvhMirror* o = (LbvhMirror*)h;
  auto cp = [](void* dst, const void* src, size_t bytes) { if (dst && bytes) std::memcpy(dst, src, bytes); };
  cp(aabb, o->aabb.data(), o->aabb.size() * 4);
  cp(centroid, o->centroid.data(), o->centroid.size() * 4);
  cp(morton, o->morton.data(), o->morton.size() * 4);
  cp(payload, o->payload.data(), o->payload.size() * 4);
  cp(nodeMin, o->nodeMin.data(), o->nodeMin.size() * 4);
  cp(nodeMax, o->nodeMax.data(), o->nodeMax.size() * 4);
  cp(left, o->nodeLeft.data(), o->nodeLeft.size() * 4);
  cp(right, o->nodeRight.data(), o->nodeRight.size() * 4);
  cp(leafTri, o->nodeLeafTri.data(), o->nodeLeafTri.size() * 4);
  if (pairs2)
    for (size_t i = 0; i < o->pairs.size(); i++) { pairs2[i * 2] = o->pairs[i].first; pairs2[i * 2 + 1] = o->pairs[i].second; }
}

}  // extern "C"

#include "jsmath.hpp"
extern "C" {
double orc_js_acos(double x) { return orc::js_acos(x); }
double orc_js_log(double x) { return orc::js_log(x); }
double orc_js_cbrt(double x) { return orc::js_cbrt(x); }
}
