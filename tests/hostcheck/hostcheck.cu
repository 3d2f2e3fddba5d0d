// Test helper: host builds of the solver's device-side contact primitives
// (closim_b200/csrc/contact_math.cuh, jsmath.cuh), exported for CPU checks
// against the oracle. Built with -fmad=false like the FP64 device path.
#include "../../closim_b200/csrc/contact_math.cuh"
#include "../../closim_b200/csrc/adjoint_math.cuh"

extern "C" {
double hc_js_acos(double x) { return cs::js_acos(x); }
double hc_js_log(double x) { return cs::js_log(x); }
double hc_js_cbrt(double x) { return cs::js_cbrt(x); }
double hc_hypot3(double a, double b, double c) { return cs::js_hypot3(a, b, c); }
void hc_closest_vt(const double* q, double* o) {
  cs::Closest c = cs::closest_vt(q, q + 3, q + 6, q + 9);
  o[0] = c.s; o[1] = c.t; o[2] = c.dist; o[3] = c.rx; o[4] = c.ry; o[5] = c.rz;
}
void hc_closest_ee(const double* q, double* o) {
  cs::Closest c = cs::closest_ee(q, q + 3, q + 6, q + 9);
  o[0] = c.s; o[1] = c.t; o[2] = c.dist; o[3] = c.rx; o[4] = c.ry; o[5] = c.rz;
}
double hc_vt_ccd(const double* P0, const double* P1, double th) { return cs::vt_ccd(P0, P1, th); }
double hc_ee_ccd(const double* P0, const double* P1, double th) { return cs::ee_ccd(P0, P1, th); }
// The trial kernel's gated CCD: distance at P1 first, then trial_ccd.
double hc_trial_ccd(const double* P0, const double* P1, double th, int kind) {
  const double dT = kind == 0 ? cs::closest_vt(P1, P1 + 3, P1 + 6, P1 + 9).dist
                              : cs::closest_ee(P1, P1 + 3, P1 + 6, P1 + 9).dist;
  return cs::trial_ccd(kind, P0, P1, dT, th);
}
int hc_solve_cubic01(double a3, double a2, double a1, double a0, double* o) { return cs::solve_cubic01(a3, a2, a1, a0, o); }
double hc_barrier_value(double d, double dh) { return cs::barrier_value(d, dh); }
double hc_barrier_grad(double d, double dh, double k) { return cs::barrier_grad_scalar(d, dh, k, 1); }
double hc_barrier_curv(double d, double dh, double k) { return cs::barrier_curvature(d, dh, k); }
double hc_bend_grad(const double* q, const double* meta, double k, double* g) {
  return cs::bend_grad<double>(q, meta[0], meta[1], meta[2], k, g);
}
void hc_bend_hvp(const double* q, const double* v, const double* meta, double k, double* o) {
  cs::bend_hvp(q, v, meta[0], meta[1], meta[2], k, o);
}
void hc_membrane_block9(const double* x9, const double* inv4, double s, const double* C4, double* h) {
  cs::membrane_block9<double>(x9, x9 + 3, x9 + 6, inv4[0], inv4[1], inv4[2], inv4[3], s, C4[0], C4[1], C4[2], C4[3], h);
}
// Exact-Newton mode: the block with the stress's positive part, and the clamp itself.
void hc_membrane_block9_psd(const double* x9, const double* inv4, double s, const double* C4, double* h) {
  cs::membrane_block9<double>(x9, x9 + 3, x9 + 6, inv4[0], inv4[1], inv4[2], inv4[3], s, C4[0], C4[1], C4[2], C4[3], h,
                              true);
}
void hc_psd_stress(double* s3) { cs::psd_stress(s3[0], s3[1], s3[2]); }
}
