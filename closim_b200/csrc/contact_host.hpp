// Host side of the ContactSystem (reference src/collision/contact-assembly.ts):
// device buffers of the frozen active set, broadphase and CCD, and the calls
// the Newton step makes into them.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "../../include/closim_cuda.h"
#include "broadphase.cuh"
#include "graph_ctx.hpp"
#include "plain.cuh"

namespace cs {

class Solver;

struct CapacityError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// Device-resident contact diagnostics (ContactDiagnostics, types.ts:49-62).
struct DevDiag {
  double minDistance, minTOI, barrierEnergy, frictionWork, ccdFailures;
  double trialMinDist, trialMinTOI;
  double killStall;  // set if the restitution rounds ran out (never expected)
};

// Device counters read back by the host (int32).
enum CInt { CI_SELF = 0, CI_STATIC, CI_OVERFLOW, CI_NCAND, CI_NFLOOR, CI_NVT, CI_VALID, CI_FIRSTNF, CI_MOVED,
            CI_FLOORBAD, CI_NBAD, CI_N = 16 };
// Failing trial candidates listed by index for the second key pass.
constexpr int kBadCap = 4096;
// Device-side counts of a graph-captured step (ContactHost::acnt, int32): the
// frozen set layout, the lag table, the superset sizes and an error word. In a
// captured step every launch is sized for its buffer's capacity and the kernels
// read these; the host reads them once, after the step.
// AC_QSELF / AC_QSTATIC: the pair counts of the last active-set query (the
// step's candidatePairs diagnostic).
enum ACnt { AC_NCAND = 0, AC_NFLOOR, AC_NVT, AC_NA, AC_LAG, AC_COMMIT, AC_NSUP, AC_NSUPS, AC_ERR, AC_NREC, AC_NTOT,
            AC_QSELF, AC_QSTATIC, AC_N = 16 };
// AC_ERR bits: a buffer capacity was exceeded, or a query fell outside a
// freshly rebuilt superset; the step is then repeated on the host-driven path.
enum ACErr { ACE_CAPACITY = 1, ACE_SUPERSET = 2 };

class ContactHost {
 public:
  cs_contact_params p{};
  bool hasFloor = false;
  double floorY = 0;
  int n = 0, m = 0, ns = 0, ms = 0;
  double rejections = 0;
  double candidatePairs = 0, activePairs = 0, vtPairs = 0, eePairs = 0, floorPairs = 0;
  int nCand = 0, nFloor = 0, nVT = 0;  // current frozen set layout
  int commitNo = 0, lagCount = 0;

  // static mesh
  float* spos = nullptr;
  uint32_t* sidx = nullptr;
  // broadphase
  BvhBufs bvh;
  int2* spairs = nullptr;
  unsigned long long* badKey = nullptr;  // smallest failing (key, status) of a trial
  int idBits = 24;             // bits per id in the candidate order key
  bool topoValid = false;      // hierarchy built for the current step
  // Superset of candidate pairs for the queries of a step: built for the
  // segment x0 -> xBase with the pad widened by kSupTravel; a later query whose
  // positions stay within kSupTravel (max norm) of xBase is covered and filters
  // it exactly, one that moved further rebuilds it around its own positions.
  static constexpr double kSupTravel = 0.004;
  double* supBase = nullptr;   // 3n positions the superset was built around
  int2* supPairs = nullptr;
  int2* supSPairs = nullptr;
  size_t supCap = 0, supSCap = 0;
  int nSup = 0, nSupS = 0;
  bool supValid = false;
  void build_superset(Solver& s, const double* x, double padSup);
  size_t pairCap = 0, spairCap = 0;
  CandBufs cand;
  uint32_t* cflag = nullptr;   // per-candidate trial status (flagCap, the superset's candidate bound + 1)
  size_t flagCap = 0;
  int smCount = 148;
  uint32_t* fflag = nullptr;   // per-vertex floor flag / offset (n + 1)
  unsigned long long* omin = nullptr;  // ordered images of the trial / active-set minima (3)
  int* badList = nullptr;      // failing trial candidates (kBadCap)
  // frozen set
  size_t actCap = 0;
  Frozen* active = nullptr;
  double* dd = nullptr;
  double* cg = nullptr;        // 4 per contact
  double* tc = nullptr;        // per-contact chain terms (merit)
  double* tf = nullptr;        // per-contact chain terms (friction work)
  // Captured steps rebuild the vertex -> record CSR only when the active
  // list's (kind, slot vertices) changed since the last build: csrIds holds
  // them (5 ints per contact), csrMemo[0] their count (-1: no valid build,
  // e.g. after a host-driven build), csrMemo[1] the mismatch flag.
  int* csrIds = nullptr;
  int* csrMemo = nullptr;
  // Captured steps keep the pair superset across steps while the step start
  // and the first iterate stay within kSupTravel of its base: supMemo[0] = 1
  // when supPairs / supSPairs / supBase hold a superset of the current contact
  // configuration, supMemo[1..2] its pair counts. Host-driven builds, static
  // mesh moves and buffer growth clear it.
  int* supMemo = nullptr;
  // Captured steps: 1 when x changed since the last active-set update (set at
  // the step start and when a trial is accepted). An update at unchanged
  // positions would rebuild the same active set, so it is skipped.
  int* actDirty = nullptr;
  Key<1>* rk0 = nullptr; Key<1>* rk1 = nullptr;
  uint32_t* rp0 = nullptr; uint32_t* rp1 = nullptr; uint32_t* rhist = nullptr;
  uint32_t* cOff = nullptr;    // n + 1
  int* kpred = nullptr;        // 4 per contact: predecessor on each vertex (restitution pass)
  double* recScratch = nullptr;  // 6 per record (4 per contact): per-record contact shares before their ordered sums
  // exact-Newton friction potential (see Contact::fric): 8 + 3 per contact
  double* fh = nullptr;
  double* fdd = nullptr;
  bool fricOn = false;         // set by friction_terms for the rest of the step
  // lagged normals / multipliers
  double* lagFloor = nullptr;  // n
  uint8_t* lagFloorOk = nullptr;
  size_t lagCap = 0;
  Key<6>* lk0 = nullptr; Key<6>* lk1 = nullptr;
  uint32_t* lp0 = nullptr; uint32_t* lp1 = nullptr; uint32_t* lhist = nullptr;
  double4* lval = nullptr;     // appended values, indexed by payload
  double4* lsorted = nullptr;  // values in sorted key order
  // probes
  double* probe = nullptr;
  DevDiag* diag = nullptr;
  int* cint = nullptr;
  int* hint = nullptr;         // pinned mirror of cint
  DevDiag* hdiag = nullptr;    // pinned mirror of diag

  ~ContactHost();
  void init(Solver& s, const cs_contact_params* prm, int floor_on, double floor_y, const float* sp, int nsv,
            const uint32_t* si, int msv);
  void begin_step_and_bisect(Solver& s);
  // Start of an independent evaluation at a new segment (the adjoint sweep):
  // the hierarchy is rebuilt at the next query.
  void begin_segment(Solver& s) {
    topoValid = false;
    supValid = false;
    (void)s;
  }
  void update_active_set(Solver& s, double* x);
  void merit_energy(Solver& s, const double* x);
  // Exact-Newton mode: freeze the friction potential at the current iterate
  // (fh) and include it in the merit and the Newton matrix from now on.
  void friction_terms(Solver& s);
  void gradient_terms(Solver& s);
  // Trial validity with one host synchronization (bisection, commit).
  bool check_trial(Solver& s, const double* xt);
  // The same split around the caller's own synchronization: trial_launch
  // enqueues the check and the copy of its counters, trial_result reads them.
  // gradGate: the device copy of the iteration's gradient norm when the trial
  // is enqueued before the convergence test (see k_trial_final).
  void trial_launch(Solver& s, const double* xt, const double* gradGate = nullptr, double gradTol = 0);
  int trial_result();
  bool trial_redo(Solver& s, const double* xt);
  void commit(Solver& s, const double* x);
  void kill_approach_velocity(Solver& s);
  void fill_stats(Solver& s, cs_step_stats& st);
  // Replaces the static mesh's vertex positions (same triangles), for a
  // collider that moves between steps (ContactSystem.setStaticMesh with the
  // sampled pose, avatar-collider.ts:205-237).
  void update_static_positions(Solver& s, const float* sp, int nsv);
  // The frozen active set of the last update (kind, p, a, b, c, d and
  // w0..w3, n), in active-list order; returns its size.
  int read_active(Solver& s, int cap, int32_t* ids6, double* w7);
  // broadphase stage only: the pairs of a segment xStep -> x with pad, counted on the device
  void launch_query(Solver& s, const double* x, double pad);
  void bind(Solver& s);  // refresh the Contact view inside the solver's Dev

  // ---- graph-captured step (graph_step.cu): the same work, launched into a
  // capture with every count read on the device (acnt) and every launch sized
  // for its buffer's capacity; overflows set acnt[AC_ERR] instead of growing.
  int* acnt = nullptr;         // AC_N device ints
  void cap_bind(Solver& s);
  void cap_begin_step(Solver& s, GraphCtx& g);
  void cap_superset(Solver& s, GraphCtx& g, const double* x);
  void cap_superset_step(Solver& s, GraphCtx& g, const double* x);
  void cap_mark_moved(GraphCtx& g);
  void cap_update_active_set_body(Solver& s, GraphCtx& g, const double* x);
  void cap_query(Solver& s, GraphCtx& g, const double* x, double pad);
  void cap_update_active_set(Solver& s, GraphCtx& g, const double* x);
  void cap_gradient_terms(Solver& s, GraphCtx& g);
  void cap_friction_terms(Solver& s, GraphCtx& g);
  void cap_merit_energy(Solver& s, GraphCtx& g, const double* x);
  void cap_trial(Solver& s, GraphCtx& g, const double* xt);
  void cap_commit(Solver& s, GraphCtx& g, const double* x);
  void cap_kill_approach_velocity(Solver& s, GraphCtx& g);
  // After a replay (one host read): the stats the host path keeps on the host.
  void cap_collect(const int* hacnt, const int* hcint, double rejectionsDev);
  // After a replay that set AC_ERR: grow every capacity a captured step cannot.
  void cap_grow(Solver& s, const int* hacnt, const int* hcint);
  int cand_blocks_cap() const;
 private:
  void read_ints(Solver& s);
  void ensure_pairs(size_t np, size_t nsp);
  void ensure_cands(size_t nc);
  void ensure_flags(size_t nc);
  int cand_blocks() const;
  double sup_pad() const { return std::max(p.dhat, p.dmin) + kSupTravel + 1e-9; }
  void ensure_active(Solver& s, size_t na);
  void ensure_lag(size_t nl);
};

void set_contact(Solver& s, const cs_contact_params* p, int floor_on, double floor_y, const float* sp, int ns,
                 const uint32_t* si, int ms);

}  // namespace cs
