// Oracle (test infrastructure only): a CPU FP64 restatement of the reference
// CpuSolver hot path of mohdabraralikhan/closim. The tests compare the CUDA
// solver with it, and it is the timed CPU baseline; nothing in the product links it.
//
// Every function follows the reference TypeScript line by line, with the same
// floating-point operation order (compile with -ffp-contract=off so a*b+c is
// never fused, as in V8). Citations are file:line within the reference repo.
//
// Parity pins: the reference's own known-answer tests (gradient check, barrier
// FD, CCD KATs, friction invariants) and the exact PCG iteration counts that
// G5_PRECONDITIONER_REPORT.md:65-76 publishes for
// tests/preconditioner-compare.test.ts. The TypeScript itself cannot run here
// (no JavaScript runtime), so parity with V8's libm (acos/log/cbrt/cos) is
// unpinned at the ulp level; Math.hypot is restated from V8's algorithm.
#pragma once
#include <cmath>
#include <cstdint>
#include <limits>
#include <string>
#include <unordered_map>
#include <vector>

namespace orc {

constexpr double INF = std::numeric_limits<double>::infinity();

// ---- JavaScript Math semantics ---------------------------------------------

// Math.max / Math.min of two numbers: NaN if either is NaN.
inline double js_max(double a, double b) {
  if (std::isnan(a) || std::isnan(b)) return NAN;
  if (a == 0 && b == 0) return std::signbit(a) ? b : a;
  return a > b ? a : b;
}
inline double js_min(double a, double b) {
  if (std::isnan(a) || std::isnan(b)) return NAN;
  if (a == 0 && b == 0) return std::signbit(a) ? a : b;
  return a < b ? a : b;
}
// Math.hypot(a, b, c) as V8 computes it (builtins math.tq MathHypot): scale by
// the largest magnitude, Kahan-compensated sum of squares, sqrt, rescale.
inline double js_hypot3(double a, double b, double c) {
  if (std::isinf(a) || std::isinf(b) || std::isinf(c)) return INF;
  if (std::isnan(a) || std::isnan(b) || std::isnan(c)) return NAN;
  double v[3] = {std::fabs(a), std::fabs(b), std::fabs(c)};
  double mx = 0;
  for (double x : v) if (x > mx) mx = x;
  if (mx == 0) return 0;
  double sum = 0, comp = 0;
  for (double x : v) {
    double nn = x / mx;
    double summand = nn * nn - comp;
    double prelim = sum + summand;
    comp = (prelim - sum) - summand;
    sum = prelim;
  }
  return std::sqrt(sum) * mx;
}
inline float fr(double v) { return (float)v; }  // Math.fround

// ---- data model --------------------------------------------------------------

// ClothMaterial (src/physics/types.ts:1-12).
struct Material {
  double arealDensity = 0.15, thickness = 0.001;
  double C00 = 20000, C11 = 20000, C01 = 0, G = 5000;
  double bendWarp = 1e-5, bendWeft = 1e-5, damping = 0.001;
};

// Hinge (src/physics/types.ts:28-36).
struct Hinge {
  int v0, v1, v2, v3;
  double restAngle, edgeLen, areaSum;
};

// ClothMeshData (src/mesh/mesh.ts:3-14): mesh constants are Float32.
struct Mesh {
  int n = 0, m = 0;
  std::vector<float> positions, rest, uv;
  std::vector<uint32_t> idx;
  std::vector<float> invDm, areas, masses;
  std::vector<Hinge> hinges;
};

// ContactParams (src/collision/types.ts:27-47).
struct ContactParams {
  double dHat = 0.002, kappa = 50, dMin = 1e-4, mu = 0.3, eps = 1e-4;
};

// ContactDiagnostics (src/collision/types.ts:49-77).
struct ContactDiag {
  double candidatePairs = 0, activePairs = 0, vtPairs = 0, eePairs = 0, floorPairs = 0;
  double minDistance = INF, minTOI = INF, barrierEnergy = 0, frictionWork = 0;
  double rejectedLineSearchSteps = 0, ccdFailures = 0;
};

// ---- mesh (src/mesh/mesh.ts) ------------------------------------------------

void build_grid(int nx, int ny, double w, double h, std::vector<float>& pos,
                std::vector<float>& uv, std::vector<uint32_t>& idx);
Mesh preprocess(const std::vector<float>& pos, const std::vector<float>& uv,
                const std::vector<uint32_t>& idx, double arealDensity);
template <class T>
double dihedral(const T* x, int v0, int v1, int v2, int v3);

// ---- element physics --------------------------------------------------------

struct TriGrad { double energy; double grad[9]; double E00, E11, E01; };
void tri_energy_grad(const double* x0, const double* x1, const double* x2,
                     const double* inv, double area, const Material& mat, TriGrad& out);
void tri_hvp(const double* x0, const double* x1, const double* x2, const double* v0,
             const double* v1, const double* v2, const double* inv, double area,
             const Material& mat, double out[9]);
void tri_hessian9(const double* x0, const double* x1, const double* x2, const double* inv,
                  double area, const Material& mat, double h[81]);

double hinge_energy(const double* x, int v0, int v1, int v2, int v3, double restAngle,
                    double edgeLen, double areaSum, double k);
double add_hinge_gradient(const double* x, double* grad, int v0, int v1, int v2, int v3,
                          double restAngle, double edgeLen, double areaSum, double k,
                          double eps = 1e-7);

struct FemEval { double energy; double maxStrain; };
FemEval eval_internal(const double* x, const Mesh& mesh, const Material& mat, double* grad);

// Exact-Newton mode pieces (orc_exact.cpp): the hinge gradient differentiated
// exactly and its Hessian, eval_internal with the exact gradient, the hinge Hessians of
// a mesh (144 per hinge), the membrane HVP with the stress of its geometric
// term replaced by its positive part plus the bending HVP (from hinH when
// given), and the positive part of a symmetric 2x2 stress.
void hinge_grad_exact(const double* q12, double restAngle, double edgeLen, double areaSum, double k,
                      double* g12);
FemEval eval_internal_exact(const double* x, const Mesh& mesh, const Material& mat, double* grad);
void hinge_hess_exact(const double* q12, double restAngle, double edgeLen, double areaSum, double k,
                      double* h144);
void hinge_hessians(const double* x, const Mesh& mesh, const Material& mat, std::vector<double>& out);
void internal_hvp_exact(const double* x, const double* p, const Mesh& mesh, const Material& mat, double* out,
                        const double* hinH = nullptr);
void stress_positive_part(double& s00, double& s11, double& s01);
double internal_energy_only(const double* x, const Mesh& mesh, const Material& mat);
double eval_membrane(const double* x, const Mesh& mesh, const Material& mat, double* grad);
void membrane_hvp(const double* x, const double* p, const Mesh& mesh, const Material& mat,
                  double* out, double eps = 1e-8);
void eval_membrane_hvp(const double* x, const double* p, const Mesh& mesh,
                       const Material& mat, double* out);
void eval_membrane_blocks(const double* x, const Mesh& mesh, const Material& mat,
                          double* blocks);

// ---- CSR incidence (src/mesh/incidence.ts) ------------------------------------
struct Incidence { std::vector<uint32_t> offsets, ids, corners; };
Incidence membrane_incidence(const Mesh& mesh);
Incidence hinge_incidence(const Mesh& mesh);

// ---- linear solve -----------------------------------------------------------

using Vec = std::vector<double>;
struct PcgResult { int iters; double residual; bool converged; };
template <class Hvp, class Prec, class Filter>
PcgResult pcg(const Vec& b, Hvp&& hvp, const Vec& diag, int maxIters, double tol,
              Filter&& filter, bool hasFilter, Prec* prec, Vec& x);

struct SchwarzDomains {
  std::vector<uint32_t> domainOf, localOf;
  std::vector<std::vector<int>> members;
};
SchwarzDomains build_schwarz_domains(const Mesh& mesh, const float* rest, int target,
                                     int minSize, int maxSize);
struct SchwarzFactors {
  const SchwarzDomains* dom = nullptr;
  std::vector<Vec> data;
  std::vector<uint8_t> flag;
};
void build_schwarz_factors(const double* x, const Mesh& mesh, const Material& mat,
                           const double* diag, const SchwarzDomains& dom, SchwarzFactors& f);
void apply_schwarz(const SchwarzFactors& f, const double* r, double* out, int n);

// Two-level additive Schwarz (mas.ts): coarse space = one constant per domain
// and component.
void restrict_coarse(const double* r, const SchwarzDomains& dom, double* rc);
void prolongate_add(const double* c, const SchwarzDomains& dom, double* z);
Vec build_coarse_diag(const double* x, const Mesh& mesh, const Material& mat, const double* diag,
                      const SchwarzDomains& dom);
void apply_mas2(const SchwarzFactors& sf, const Vec& dc, double omega, const double* r, double* out, int n);
struct CoarseExact {
  const SchwarzDomains* dom = nullptr;
  int n = 0;     // 3 D
  Vec chol;      // n x n: Cholesky L (lower) when flag, else the inverse diagonal
  int flag = 0;
};
void build_coarse_exact(const double* x, const Mesh& mesh, const Material& mat, const double* diag,
                        const SchwarzDomains& dom, CoarseExact& ce);
void solve_coarse_exact(const CoarseExact& ce, const double* rhs, double* out);
void apply_masx(const SchwarzFactors& sf, const CoarseExact& ce, const double* r, double* out, int n);

struct BlockFactors { Vec inv; std::vector<uint8_t> flag; };
void build_block_factors(const double* x, const Mesh& mesh, const Material& mat,
                         const double* diag, BlockFactors& f);
void apply_block_factors(const BlockFactors& f, const double* r, double* out, int n);

// ---- collision primitives ----------------------------------------------------

struct Closest { double s, t, dist, rx, ry, rz; };
Closest closest_vt(double px, double py, double pz, double ax, double ay, double az,
                   double bx, double by, double bz, double cx, double cy, double cz);
Closest closest_ee(double ax, double ay, double az, double bx, double by, double bz,
                   double cx, double cy, double cz, double dx, double dy, double dz);
// CCD over x(t) = P0 + t (P1 - P0) for the four stencil points (12 doubles each).
double vt_ccd(const double* P0, const double* P1, double thickness);
double ee_ccd(const double* P0, const double* P1, double thickness);
std::vector<double> solve_cubic01(double a3, double a2, double a1, double a0);

double barrier_value(double d, double dHat);
double barrier_grad_scalar(double d, double dHat, double kappa, double w);
double barrier_normal_force(double d, double dHat, double kappa, double w);
void coulomb_force(double ux, double uy, double uz, double nx, double ny, double nz,
                   double lambdaN, double mu, double eps, double f[3]);

// ---- broadphase (src/collision/bvh.ts, aabb.ts) ---------------------------
struct Aabb { double minX, minY, minZ, maxX, maxY, maxZ; };
inline bool overlaps(const Aabb& a, const Aabb& b) {
  return a.minX <= b.maxX && a.maxX >= b.minX && a.minY <= b.maxY && a.maxY >= b.minY &&
         a.minZ <= b.maxZ && a.maxZ >= b.minZ;
}
struct BvhNode { Aabb box; int left, right, tri; };
struct TriBvh {
  std::vector<BvhNode> nodes;
  int root = -1;
  void build(const double* x0, const double* x1, const uint32_t* idx, int triCount, double pad);
  std::vector<std::pair<int, int>> self_pairs(const std::vector<int64_t>& excludedSorted) const;
 private:
  int build_rec(std::vector<int>& order, const std::vector<Aabb>& boxes, const Vec& cx,
                const Vec& cy, const Vec& cz);
};
std::vector<int64_t> adjacency_exclusions(const uint32_t* idx, int triCount);

// ---- ContactSystem (src/collision/contact-assembly.ts) -----------------------
struct Cand { int kind, p, a, b, c, d; };
struct Frozen {
  int kind, p, a, b, c, d;
  double w0, w1, w2, w3, nx, ny, nz;
};
struct Lagged { double nx, ny, nz, lambdaN; };
struct Key4 {
  int k[5];
  bool operator==(const Key4& o) const {
    for (int i = 0; i < 5; i++) if (k[i] != o.k[i]) return false;
    return true;
  }
};
struct Key4Hash {
  size_t operator()(const Key4& a) const {
    uint64_t h = 1469598103934665603ull;
    for (int i = 0; i < 5; i++) { h ^= (uint32_t)a.k[i]; h *= 1099511628211ull; }
    return (size_t)h;
  }
};
Key4 contact_key(const Frozen& c);

struct TrialResult { bool valid; double minDist, minTOI; };

// Exact-Newton mode: one contact's friction potential mu lambda sqrt(|P u|^2 +
// eps^2), frozen at a Newton iterate: ml = mu max(0, lambda), the normal n of
// P = I - n n^T, and t = P u, r = sqrt(|t|^2 + eps^2) at the freeze point.
struct FricTerm { double ml = 0, nx = 0, ny = 0, nz = 0, tx = 0, ty = 0, tz = 0, r = 1; };

class ContactSystem {
 public:
  ContactParams params;
  std::vector<uint32_t> clothIdx;
  int triCount = 0;
  std::vector<int64_t> exclusions;  // sorted triPairKey values
  bool hasFloor = false;
  double floorY = 0;
  std::vector<float> staticPos;
  std::vector<uint32_t> staticIdx;
  Vec xStep;
  std::unordered_map<Key4, Lagged, Key4Hash> lagged;
  std::vector<Frozen> active;
  std::vector<Cand> candidates;
  ContactDiag diag;
  TriBvh bvh;

  ContactSystem(const ContactParams& p, const std::vector<uint32_t>& clothIndices);
  void set_floor(bool on, double y) { hasFloor = on; floorY = y; }
  void set_static_mesh(const std::vector<float>& pos, const std::vector<uint32_t>& idx) {
    staticPos = pos; staticIdx = idx;
  }
  void begin_step(const double* x0, int n3);
  void add_rejection() { diag.rejectedLineSearchSteps++; }
  std::vector<Cand> build_candidates(const double* x, double pad);
  void update_active_set(const double* x, int n3);
  double energy_grad(const double* x, double* grad, int n3);
  void apply_hvp(const double* x, const double* v, double* out, int n3);
  double merit_energy(const double* x);
  void add_diag_estimate(double* diag, const double* x);
  void commit(const double* x);
  TrialResult check_trial(const double* xT, int n3);
  // helpers
  void pos_of(const double* x, int v, double out[3]) const;
  double frozen_dist(const double* x, const Frozen& c) const;
  void add_dist_grad(double* grad, const Frozen& c, double g) const;
  void add_friction_force(double* grad, const Frozen& c, double fx, double fy, double fz) const;
  void relative_slip(const double* x, const Frozen& c, double u[3]) const;
  double dist_jvp(const Frozen& c, const double* v) const;
  double exact_dist(const double* x, const Cand& q) const;
  // Exact-Newton mode (orc_exact.cpp): freeze the friction potential of every
  // active contact at x, its value at x, and its Hessian along v.
  std::vector<FricTerm> fric;
  void friction_potential_freeze(const double* x);
  double friction_potential(const double* x) const;
  void friction_hvp(const double* v, double* out, int n3) const;
 private:
  std::vector<std::pair<int, int>> query_bvh_all(const std::vector<Aabb>& sBoxes) const;
};

// ---- scene + stepper (src/physics/scene.ts, src/solver/newton.ts) ------------
struct Scene {
  Mesh mesh;
  Material material;
  double gravity[3] = {0, -9.81, 0};
  std::vector<int> pinIds;            // pinned vertex ids (Map key order)
  std::vector<double> pinPos;         // 3 per pin
  Vec positions, velocities;
  ContactSystem* contact = nullptr;
};
void enforce_pins(const Scene& s, double* x);
void pin_filter(const Scene& s, double* v);
void kill_approach_velocity(ContactSystem& contact, Scene& scene, const double* x);

enum Precond { PRECOND_JACOBI = 0, PRECOND_SCHWARZ = 1, PRECOND_BLOCK = 2, PRECOND_MAS2 = 3 };
struct StepperOptions {
  int newtonIters = 10, pcgMaxIters = 60;
  double gradTol = 1e-5;
  int lsIters = 10;
  int precond = PRECOND_JACOBI;
};
struct StepStats {
  int newtonIters, pcgIters;
  double gradNorm, energy, maxStrain;
  bool converged;
  bool hasContact;
  ContactDiag contact;
  int newtonItersUsed;   // extension: iterations actually run
  int armijoTrials;      // extension: total line-search trials
};
StepStats implicit_step(Scene& scene, double h, const StepperOptions& opts,
                        const SchwarzDomains* domains);
// Exact-Newton mode of the CUDA solver (orc_exact.cpp): implicit_step with the
// exact hinge gradient, the positive-semi-definite Newton matrix, friction as a
// frozen potential, PCG to tolerance pcgTol, the drift start x0 + h v when
// drift is set, and a CCD-valid full step taken once gradNorm < 1e-7.
StepStats implicit_step_exact(Scene& scene, double h, const StepperOptions& opts,
                              const SchwarzDomains* domains, double pcgTol, bool drift);

// ---- FP32 LBVH mirror (src/backend/webgpu/gpu-broadphase.ts) -----------------
struct LbvhMirror {
  std::vector<float> aabb, centroid;
  std::vector<uint32_t> morton, payload;
  std::vector<float> nodeMin, nodeMax;
  std::vector<int32_t> nodeLeft, nodeRight, nodeLeafTri;
  int root = 0, depth = 1;
  std::vector<std::pair<int, int>> pairs;
  long scanned = 0;
  int overflow = 0;
};
uint32_t morton_key_of(const float c[3], const float sMin[3], const float sMax[3]);
void lbvh_mirror_build(const double* x0, const double* x1, const uint32_t* idx, int m,
                       double pad, const std::vector<int64_t>& exclusionsSorted,
                       long capacity, LbvhMirror& out);

}  // namespace orc
