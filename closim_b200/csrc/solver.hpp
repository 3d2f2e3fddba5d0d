// The CUDA cloth solver instance: device buffers, set-up and the host
// orchestration of one implicit-Euler step (shared by solver.cu and contact.cu).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/closim_cuda.h"
#include "adjoint.cuh"
#include "cluster_plan.hpp"
#include "contact_host.hpp"
#include "mixed.cuh"
#include "plain.cuh"
#include "setup.hpp"

namespace cs {

inline int64_t& launch_counter() {
  static int64_t c = 0;
  return c;
}

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
#define CK(x)                                                                                    \
  do {                                                                                           \
    cudaError_t e_ = (x);                                                                        \
    if (e_ != cudaSuccess) throw CudaError(std::string(#x) + ": " + cudaGetErrorString(e_));   \
  } while (0)

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t k) {
    free();
    n = k;
    if (k) CK(cudaMalloc(&p, k * sizeof(T)));
  }
  void upload(const T* h, size_t k, cudaStream_t s) {
    if (k > n) alloc(k);
    if (k) CK(cudaMemcpyAsync(p, h, k * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DBuf() { free(); }
};

struct NonFinite : std::runtime_error {
  NonFinite() : std::runtime_error("non-finite gradient — blow up; reduce dt/stiffness") {}
};

// Phases of a step for the wall-time breakdown (cs_profile mode 2).
struct AdjStats {
  long pcgIters = 0;
  int solves = 0, recomputedSteps = 0;
  double maxRelResidual = 0;
  int forwardConverged = 0;  // steps of the last cs_forward that reached gradTol
};

enum Phase { PH_OTHER = 0, PH_BROADPHASE, PH_ACTIVE_SET, PH_GRADIENT, PH_PRECOND, PH_PCG, PH_TRIAL, PH_ENERGY,
             PH_COMMIT, PH_N };

class Solver {
 public:
  int precision = CS_PRECISION_FP64;
  int device = 0;
  bool ready = false;
  cudaStream_t stream = nullptr;
  HostMesh mesh;
  cs_material mat{};
  double gravity[3] = {0, -9.81, 0};
  cs_stepper_options opts{10, 60, 10, CS_PRECOND_JACOBI, 1e-5};
  cs_step_stats stats{};
  bool haveStats = false;
  std::vector<int> pinIds;
  std::vector<double> pinPos;
  std::unique_ptr<ContactHost> contact;

  // device buffers
  DBuf<uint32_t> idx, memOff, memRec, hinOff, hinRec;
  DBuf<float4> inv;
  DBuf<float> area, mass;
  DBuf<int4> hinge;
  DBuf<double> hmeta;
  DBuf<uint8_t> pinned;
  DBuf<int> pinIdsD, domStart, domVerts, v2tOff, v2t;
  DBuf<double> pinPosD;
  DBuf<double> vx, vv, vx0, vyHat, vg, vdiag, vdx, vr, vz, vp, vAp, vxt, vcgrad, vcHp, elem, helem, part, scal, L;
  DBuf<double> T0, T1, T2, T3, Tc;
  DBuf<uint8_t> domFlag;
  DBuf<double> dcoarse;
  double* hscal = nullptr;  // pinned host mirror of scal
  int pcgBlocks = 1;
  // mixed-precision path
  DBuf<float> fr, fz, fp, fAp, fx, felem, ftris, fh9, fLinv, fp2;
  DBuf<float4> fvrec, fdc;
  DBuf<uint32_t> triSlot;
  MixBufs mb{};
  int mxBlocks = 1;
  int mxCluster = 0;  // CTAs of the one-cluster PCG (0: grid-wide cooperative PCG)
  // Per-CTA element lists of the one-cluster PCG's resident phase A; clRes[k]
  // (k = 1 with the Gauss-Newton bending term) says whether they fit.
  ClusterPlanHost clHost;
  DBuf<int> clVb, clHaloOff, clHalo, clTriOff, clTriId, clHinOff, clHinId, clIncOff, clIncHin, clOwnHalo, clVDst;
  DBuf<uint16_t> clTriLoc, clHinLoc;
  DBuf<uint32_t> clInc;
  ClPlan clPlan{};
  bool clRes[2] = {false, false};
  size_t clSmem[2] = {0, 0};  // launch's dynamic shared memory
  int clCap[2] = {0, 0};      // on-chip contact records per CTA
  Dev d{};
  // profiling of the linear-solve kernel
  bool prof = false;
  cudaEvent_t pev0 = nullptr, pev1 = nullptr;
  double profMs = 0, profLaunches = 0, profBytes = 0, profIters = 0;
  bool profPending = false;
  // Wall time per phase of the step (cs_profile mode 2): the stream is
  // synchronized at every phase boundary, so each phase is charged its host
  // launch overhead plus its device time. Diagnostic only (slows the step).
  bool profPhases = false;
  int curPhase = PH_OTHER;
  double phaseMs[PH_N] = {};
  std::chrono::steady_clock::time_point phaseT0{};
  int phase(int p) {
    const int prev = curPhase;
    if (!profPhases) { curPhase = p; return prev; }
    CK(cudaStreamSynchronize(stream));
    const auto now = std::chrono::steady_clock::now();
    phaseMs[curPhase] += std::chrono::duration<double, std::milli>(now - phaseT0).count();
    phaseT0 = now;
    curPhase = p;
    return prev;
  }

  // Algorithmic bytes of one k_pcg launch that ran `iters` iterations: per
  // iteration the FD HVP reads x, p (2 x 24 B per vertex), Dm^-1, area and 3
  // indices per triangle (32 B), writes and re-reads 18 element doubles
  // (2 x 144 B per triangle), reads mass (4 B) and writes Ap (24 B); the vector
  // update reads p, Ap, x, r, diag and writes x, r, z, p (9 x 24 B per vertex);
  // Schwarz adds one read of its 24x24 factors (4608 B per domain).
  double pcg_bytes(int iters) const {
    const double n = mesh.n, m = mesh.m;
    if (precision == CS_PRECISION_MIXED) {
      // FP32 path per iteration: per triangle the stored F/S/Dm^-1 record (64 B),
      // 3 indices, the 9-float element result written and gathered (2 x 36 B) and
      // its incidence records (12 B); per vertex p and mass read, Ap written, the
      // x/r/z/p updates (read p, Ap, x, r, z; write x, r, z, p: 9 x 12 B) and the
      // CSR offset; Schwarz reads one 24x24 FP32 inverse per domain.
      const double tri = 64 + 12 + 72 + 12;
      const double vert = 12 + 4 + 12 + 9 * 12 + 4;
      const double dom = d.precond >= 1 ? 2304.0 + 2 * 96 : 0.0;
      return 5 * 12 * n + iters * (tri * m + vert * n + dom * mesh.D) + 4 * 24 * n;
    }
    double hvp = 2 * 24 * n + 32 * m + 2 * 144 * m + 4 * n + 24 * n;
    double vec = 9 * 24 * n + (d.precond >= 1 ? 4608.0 * mesh.D : 0.0);
    double init = 6 * 24 * n;
    double post = 4 * 24 * n;
    return init + iters * (hvp + vec) + post;
  }
  void prof_collect(int iters) {
    if (!profPending) return;
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, pev0, pev1));
    profMs += ms;
    profLaunches += 1;
    profBytes += pcg_bytes(iters);
    profIters += iters;
    profPending = false;
  }

  ~Solver() {
    graph_release();
    if (pev0) cudaEventDestroy(pev0);
    if (pev1) cudaEventDestroy(pev1);
    if (hscal) cudaFreeHost(hscal);
    if (hNan) cudaFreeHost(hNan);
    if (stream) cudaStreamDestroy(stream);
  }

  void create(int prec, int dev) {
    precision = prec;
    device = dev;
    CK(cudaSetDevice(dev));
    CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    CK(cudaMallocHost(&hscal, S_NSCALARS * sizeof(double)));
    CK(cudaEventCreate(&pev0));
    CK(cudaEventCreate(&pev1));
  }

  // d.precond: 0 Jacobi, 1 one-level Schwarz, 2 two-level Schwarz (mas2).
  int precond_code() const {
    return opts.precond == CS_PRECOND_SCHWARZ ? 1 : opts.precond == CS_PRECOND_MAS2 ? 2 : 0;
  }

  void set_material(const cs_material& m) {
    mat = m;
    d.mat = Mat<double>{m.stretch_warp, m.stretch_weft, m.stretch_coupling, m.shear, m.thickness};
    d.kb = 0.5 * (m.bend_warp + m.bend_weft);
    mb.C00 = (float)m.stretch_warp; mb.C11 = (float)m.stretch_weft; mb.C01 = (float)m.stretch_coupling;
    mb.G = (float)m.shear;
  }
  bool mixed() const { return precision == CS_PRECISION_MIXED; }
  void energy_of(const double* x) {
    int64_t& lc = launch_counter();
    if (mixed()) { launch_energy_terms(d, x, stream); lc += 1; mx_energy_final(d, stream, &lc); }
    else { launch_energy(d, x, stream); lc += 3; }
  }

  void initialize(const cs_mesh& cm, const cs_material& m, const double* g, const double* x, const double* v) {
    CK(cudaSetDevice(device));
    if (cm.n <= 0 || cm.m <= 0 || cm.hg < 0) throw std::invalid_argument("bad mesh sizes");
    if (!cm.indices || !cm.rest || !cm.inv_dm || !cm.area || !cm.mass || (cm.hg > 0 && (!cm.hinge || !cm.hinge_meta)))
      throw std::invalid_argument("null mesh array");
    mesh = HostMesh();
    mesh.n = cm.n; mesh.m = cm.m; mesh.hg = cm.hg;
    mesh.idx.assign(cm.indices, cm.indices + 3 * (size_t)cm.m);
    for (uint32_t q : mesh.idx)
      if ((int)q >= cm.n) throw std::invalid_argument("triangle index out of range");
    mesh.rest.assign(cm.rest, cm.rest + 3 * (size_t)cm.n);
    mesh.inv.assign(cm.inv_dm, cm.inv_dm + 4 * (size_t)cm.m);
    mesh.area.assign(cm.area, cm.area + cm.m);
    mesh.mass.assign(cm.mass, cm.mass + cm.n);
    mesh.hinge.assign(cm.hinge, cm.hinge + 4 * (size_t)cm.hg);
    for (int q : mesh.hinge)
      if (q < 0 || q >= cm.n) throw std::invalid_argument("hinge index out of range");
    mesh.hmeta.assign(cm.hinge_meta, cm.hinge_meta + 3 * (size_t)cm.hg);
    build_topology(mesh);
    build_schwarz(mesh, 8, 1);
    if (mesh.maxDomain > 8) throw std::runtime_error("Schwarz domain larger than 8 vertices");
    for (int k = 0; k < 3; k++) gravity[k] = g ? g[k] : (k == 1 ? -9.81 : 0.0);
    set_material(m);
    const size_t n3 = 3 * (size_t)cm.n;
    idx.upload(mesh.idx.data(), mesh.idx.size(), stream);
    inv.alloc(cm.m);
    if (cm.m) CK(cudaMemcpyAsync(inv.p, mesh.inv.data(), (size_t)cm.m * 16, cudaMemcpyHostToDevice, stream));
    area.upload(mesh.area.data(), cm.m, stream);
    mass.upload(mesh.mass.data(), cm.n, stream);
    hinge.alloc(std::max(cm.hg, 1));
    if (cm.hg) CK(cudaMemcpyAsync(hinge.p, mesh.hinge.data(), (size_t)cm.hg * 16, cudaMemcpyHostToDevice, stream));
    hmeta.upload(mesh.hmeta.data(), mesh.hmeta.size(), stream);
    memOff.upload(mesh.memOff.data(), mesh.memOff.size(), stream);
    memRec.upload(mesh.memRec.data(), mesh.memRec.size(), stream);
    hinOff.upload(mesh.hinOff.data(), mesh.hinOff.size(), stream);
    hinRec.alloc(std::max<size_t>(mesh.hinRec.size(), 1));
    hinRec.upload(mesh.hinRec.data(), mesh.hinRec.size(), stream);
    v2tOff.upload((const int*)mesh.v2tOff.data(), mesh.v2tOff.size(), stream);
    v2t.alloc(std::max<size_t>(mesh.v2t.size(), 1));
    v2t.upload((const int*)mesh.v2t.data(), mesh.v2t.size(), stream);
    domStart.upload(mesh.domStart.data(), mesh.domStart.size(), stream);
    domVerts.upload(mesh.domVerts.data(), mesh.domVerts.size(), stream);
    domFlag.alloc(std::max(mesh.D, 1));
    L.alloc((size_t)std::max(mesh.D, 1) * 576);
    dcoarse.alloc((size_t)std::max(mesh.D, 1) * 3);
    for (DBuf<double>* b : {&vx, &vv, &vx0, &vyHat, &vg, &vdiag, &vdx, &vr, &vz, &vp, &vAp, &vxt, &vcgrad, &vcHp})
      b->alloc(n3);
    CK(cudaMemsetAsync(vcgrad.p, 0, n3 * 8, stream));
    CK(cudaMemsetAsync(vcHp.p, 0, n3 * 8, stream));
    const size_t tcap = std::max(n3, (size_t)cm.m + (size_t)cm.hg);
    for (DBuf<double>* b : {&T0, &T1, &T2, &T3}) b->alloc(tcap);
    Tc.alloc(1);
    elem.alloc(std::max<size_t>((size_t)cm.m * 18, 1));
    helem.alloc(std::max<size_t>((size_t)cm.hg * 12, 1));
    const int partStride = (int)((std::max(std::max(n3, (size_t)cm.m), (size_t)cm.hg) + kThreads - 1) / kThreads) + 1;
    part.alloc((size_t)NPART * partStride);
    scal.alloc(S_NSCALARS);
    CK(cudaMemsetAsync(scal.p, 0, S_NSCALARS * 8, stream));
    pinned.alloc(cm.n);
    CK(cudaMemsetAsync(pinned.p, 0, cm.n, stream));
    vx.upload(x, n3, stream);
    if (v) vv.upload(v, n3, stream);
    else CK(cudaMemsetAsync(vv.p, 0, n3 * 8, stream));
    d = Dev{};
    d.n = cm.n; d.m = cm.m; d.hg = cm.hg;
    d.idx = idx.p; d.inv = inv.p; d.area = area.p; d.mass = mass.p; d.hinge = hinge.p; d.hmeta = hmeta.p;
    d.memOff = memOff.p; d.memRec = memRec.p; d.hinOff = hinOff.p; d.hinRec = hinRec.p;
    d.pinned = pinned.p;
    d.x = vx.p; d.v = vv.p; d.x0 = vx0.p; d.yHat = vyHat.p; d.g = vg.p; d.diag = vdiag.p; d.dx = vdx.p;
    d.r = vr.p; d.z = vz.p; d.p = vp.p; d.Ap = vAp.p; d.xt = vxt.p; d.cgrad = vcgrad.p; d.cHp = vcHp.p;
    d.elem = elem.p; d.helem = helem.p; d.part = part.p; d.partStride = partStride; d.scal = scal.p;
    d.D = mesh.D; d.domStart = domStart.p; d.domVerts = domVerts.p; d.v2tOff = v2tOff.p; d.v2t = v2t.p;
    d.L = L.p; d.domFlag = domFlag.p; d.dcoarse = dcoarse.p;
    d.T0 = T0.p; d.T1 = T1.p; d.T2 = T2.p; d.T3 = T3.p; d.Tc = Tc.p;
    set_material(m);
    for (int k = 0; k < 3; k++) d.gravity[k] = gravity[k];
    pcgBlocks = pcg_grid_blocks(d);
    if (precision == CS_PRECISION_MIXED) {
      for (DBuf<float>* b : {&fr, &fz, &fp, &fAp, &fx}) b->alloc(n3);
      felem.alloc((size_t)cm.m * 9);
      ftris.alloc((size_t)cm.m * 16);
      fh9.alloc((size_t)cm.m * 81);
      fLinv.alloc((size_t)std::max(mesh.D, 1) * 576);
      fdc.alloc((size_t)std::max(mesh.D, 1));
      mb.r = fr.p; mb.z = fz.p; mb.p = fp.p; mb.Ap = fAp.p; mb.x = fx.p;
      mb.elem = felem.p; mb.tris = ftris.p; mb.h9 = fh9.p; mb.Linv = fLinv.p;
      build_schwarz_assembly();
      mxBlocks = mx_pcg_grid_blocks(d);
      // Sheets up to 20k vertices solve inside one thread-block cluster
      // (on-GPC barriers); larger ones use the grid-wide kernel.
      // CLOSIM_MX_PCG=grid|cluster overrides the choice.
      const char* env = std::getenv("CLOSIM_MX_PCG");
      const bool wantCluster = env ? std::string(env) == "cluster" : mesh.n <= 20000;
      mxCluster = wantCluster && mesh.maxDomain <= 8 ? mx_cluster_size() : 0;
      if (mxCluster > 0) {
        fp2.alloc(n3);
        std::vector<uint32_t> slot(3 * (size_t)cm.m);
        for (size_t q = 0; q < mesh.memRec.size(); q++) {
          const uint32_t rec = mesh.memRec[q];
          slot[(rec >> 2) * 3 + (rec & 3)] = (uint32_t)q;
        }
        triSlot.upload(slot.data(), slot.size(), stream);
        fvrec.alloc(5 * 3 * (size_t)cm.m);
        mb.vrec = fvrec.p;
        mb.triSlot = triSlot.p;
        build_cluster_resident();
      }
    }
    upload_pins();
    contact.reset();
    if (precision == CS_PRECISION_MIXED && mxCluster > 0) contact_free_valid();
    CK(cudaStreamSynchronize(stream));
    initEpoch++;
    ready = true;
  }

  void set_pins(int k, const int* ids, const double* pos) {
    for (int i = 0; i < k; i++)
      if (ids[i] < 0 || ids[i] >= mesh.n) throw std::invalid_argument("pin id out of range");
    pinIds.assign(ids, ids + k);
    pinPos.assign(pos, pos + 3 * (size_t)k);
    if (ready) upload_pins();
  }

  void upload_pins() {
    std::vector<uint8_t> mask(mesh.n, 0);
    for (int id : pinIds) mask[id] = 1;
    CK(cudaMemcpyAsync(pinned.p, mask.data(), mesh.n, cudaMemcpyHostToDevice, stream));
    const int k = (int)pinIds.size();
    if (k) {
      pinIdsD.upload(pinIds.data(), k, stream);
      pinPosD.upload(pinPos.data(), 3 * (size_t)k, stream);
    }
    d.npins = k;
    d.pinIds = pinIdsD.p;
    d.pinPos = pinPosD.p;
    CK(cudaStreamSynchronize(stream));  // host vectors above are temporaries
  }

  void read_scalars() {
    CK(cudaMemcpyAsync(hscal, scal.p, S_NSCALARS * 8, cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
  }

  // ---- graph-captured step (graph_step.cu) ---------------------------------------
  struct GraphStep;
  GraphStep* gstep = nullptr;
  int graphMode = 1;           // 1: the captured step where it applies (cs_set_graph_mode)
  int64_t graphSteps = 0, graphFallbacks = 0;
  int initEpoch = 0;           // bumped by initialize / set_contact: the captured graph is stale
  DBuf<int> validOne;          // an always-valid trial flag for steps without contact
  void graph_release();
  std::vector<double> graph_key(double h) const;
  void graph_capture(double h);
  const int* contact_free_valid();
  // One step as a captured graph replay with the decisions on the device;
  // false when the configuration is not covered (or a buffer overflowed and
  // the state was restored), and the caller runs the host-driven step.
  bool step_graph(double h);

  // One implicit-Euler step (newton.ts:27-232).
  void step(double h) {
    if (!ready) throw std::logic_error("CpuSolver not initialized");
    if (step_graph(h)) return;
    d.h = h;
    d.invH2 = 1 / (h * h);
    for (int k = 0; k < 3; k++) d.gravity[k] = gravity[k];
    d.precond = precond_code();
    d.hasContact = contact ? 1 : 0;
    d.driftGuess = newtonMode == 1 && driftGuess ? 1 : 0;
    int64_t& lc = launch_counter();
    if (profPhases) { CK(cudaStreamSynchronize(stream)); phaseT0 = std::chrono::steady_clock::now(); curPhase = PH_OTHER; }
    launch_predict(d, stream);
    lc += 1 + (d.npins > 0);
    if (contact) contact->begin_step_and_bisect(*this);
    if (contact) contact->update_active_set(*this, d.x);
    if (contact) contact->merit_energy(*this, d.x);
    energy_of(d.x);
    const double beta = std::max(std::max(mat.stretch_warp, mat.stretch_weft), mat.shear) * mat.thickness * 0.1 + 1e-6;
    launch_diag_init(d, beta, stream);
    lc += 1;
    read_scalars();
    double energy = hscal[S_ENERGY_TRIAL];
    double gradNorm = INFINITY, maxStrain = 0;
    int pcgTotal = 0, used = 0, trials = 0;
    bool converged = false;
    for (int ni = 0; ni < opts.newton_iters; ni++) {
      used = ni + 1;
      phase(PH_ACTIVE_SET);
      if (contact) contact->gradient_terms(*this);  // active set, barrier+friction grad, diag estimate
      phase(PH_GRADIENT);
      if (mixed()) {
        launch_grad_terms(d, stream, true);
        lc += 2 + (d.kb > 0 && d.hg > 0);
        mx_grad_final(d, stream, &lc);
      } else {
        // Exact-Newton mode takes the analytic hinge gradient: the reference's
        // central differences of an acos-based angle carry rounding noise near
        // flat hinges (about 1e-3 in |g| on a flat sheet), a floor no tight
        // tolerance can get under.
        launch_grad(d, stream, newtonMode == 1);
        lc += 3 + (d.kb > 0 && d.hg > 0);
      }
      // Exact-Newton mode: the lagged friction becomes a potential frozen for
      // this iteration (in the merit and the Newton matrix, so the Newton
      // direction is a descent direction of the merit), and the Armijo base
      // energy is re-evaluated at x with it and with this iteration's active
      // set (contacts that enter the set while Newton moves the sheet would
      // otherwise be missing from the base energy but present in every trial's).
      const bool fricExact = newtonMode == 1 && contact && contact->p.mu > 0;
      const bool meritAgain = newtonMode == 1 && contact;
      if (fricExact) contact->friction_terms(*this);
      if (meritAgain) {
        contact->merit_energy(*this, d.x);
        energy_of(d.x);
      }
      // The convergence test needs the gradient norm on the host. With a line
      // search ahead, the solve and the first trial are enqueued before it is
      // read and the norm comes back with the trial's synchronization: when
      // the gradient turns out converged (or non-finite) that work is dropped,
      // and the trial's contact check leaves no record (it reads the norm on
      // the device). Without one, the norm is read here.
      const bool speculate = newtonMode == 0 && opts.ls_iters > 0;
      bool gradRead = false, stop = false;
      if (!speculate) {
        read_scalars();
        gradNorm = hscal[S_GRADNORM];
        maxStrain = hscal[S_MAXSTRAIN];
        if (meritAgain) energy = hscal[S_ENERGY_TRIAL];
        if (!std::isfinite(gradNorm)) throw NonFinite();
        if (gradNorm < opts.grad_tol) { converged = true; break; }
        gradRead = true;
      }
      phase(PH_PRECOND);
      // Exact-Newton mode on the mixed path (one-cluster sheets): the FP32 PCG
      // solves the positive semi-definite Newton matrix (clamped membrane
      // stress, Gauss-Newton bending, frozen barrier) to a tolerance FP32 can
      // reach; larger sheets take the FP64 exact solve.
      const bool exactMixed = newtonMode == 1 && mixed() && mxCluster > 0;
      mb.psd = exactMixed ? 1 : 0;
      mb.hrec = exactMixed && d.kb > 0 && d.hg > 0 ? ensure_hrec() : nullptr;
      mb.dcoarse = d.precond == 2 ? fdc.p : nullptr;
      if (newtonMode == 1 && !exactMixed) {
        if (d.precond >= 1) { launch_schwarz_factor(d, stream); lc += d.precond; }
      } else if (mixed()) {
        mx_prepare(d, mb, d.precond >= 1, stream, &lc);
      } else if (d.precond >= 1) {
        launch_schwarz_factor(d, stream);
        lc += 1;
      }
      phase(PH_PCG);
      if (prof) CK(cudaEventRecord(pev0, stream));
      if (newtonMode == 1 && !exactMixed) {
        ensure_adj_buffers();
        AdjArgs a{d, adjRhs.p, d.dx, adjR.p, adjZ.p, adjP.p, adjAp.p, adjTri.p, adjHin.p, d.kb, 1,
                  opts.pcg_max_iters, newtonTol, adjOut.p};
        CK((cudaError_t)newton_exact_solve(a, adj_grid_blocks(d), stream));
        lc += 3;
      } else if (mixed() && mxCluster > 0)
        CK((cudaError_t)mx_launch_pcg_cluster(d, mb, cluster_plan_for(mb), fp.p, fp2.p, d.hasContact ? d.c.dd : nullptr,
                                              opts.pcg_max_iters, exactMixed ? std::max(newtonTol, kMixedTolFloor) : 1e-3,
                                              mxCluster, stream));
      else if (mixed()) CK((cudaError_t)mx_launch_pcg(d, mb, opts.pcg_max_iters, 1e-3, mxBlocks, stream));
      else CK((cudaError_t)launch_pcg(d, opts.pcg_max_iters, 1e-3, pcgBlocks, stream));
      if (prof) { CK(cudaEventRecord(pev1, stream)); profPending = true; }
      lc += 1;
      double alpha = 1;
      bool accepted = false;
      bool haveSlope = false;
      double gtdx = 0;
      for (int li = 0; li < opts.ls_iters; li++) {
        trials++;
        phase(PH_TRIAL);
        launch_trial(d, alpha, stream);
        lc += 1 + (d.npins > 0);
        // The trial's validity check and its energy are enqueued together and
        // read with one synchronization; the energy has no side effects and is
        // used only when the trial is valid, as in the reference.
        if (contact) contact->trial_launch(*this, d.xt, gradRead ? nullptr : scal.p + S_GRADNORM, opts.grad_tol);
        phase(PH_ENERGY);
        if (contact) contact->merit_energy(*this, d.xt);
        energy_of(d.xt);
        read_scalars();
        if (!gradRead) {
          gradRead = true;
          gradNorm = hscal[S_GRADNORM];
          maxStrain = hscal[S_MAXSTRAIN];
          if (!std::isfinite(gradNorm)) throw NonFinite();
          if (gradNorm < opts.grad_tol) {
            converged = true;
            stop = true;
            trials--;
            profPending = false;
            break;
          }
        }
        if (contact) {
          int r = contact->trial_result();
          if (r < 0) r = contact->trial_redo(*this, d.xt) ? 1 : 0;
          if (!r) {
            contact->rejections++;
            alpha *= 0.5;
            continue;
          }
        }
        if (!haveSlope) {
          gtdx = hscal[S_GTDX];
          pcgTotal += (int)hscal[S_PCG_ITERS];
          prof_collect((int)hscal[S_PCG_ITERS]);
          haveSlope = true;
        }
        const double eNew = hscal[S_ENERGY_TRIAL];
        if (!std::isfinite(eNew)) {
          if (contact) contact->rejections++;
          alpha *= 0.5;
          continue;
        }
        // Exact-Newton mode, close to convergence: the energy decrease of a full
        // step falls below the rounding of the energy sum, so Armijo is decided
        // by noise; a CCD-valid full step is taken (local quadratic convergence).
        const bool nearConverged = newtonMode == 1 && gradNorm < 1e-7 && alpha == 1;
        if (nearConverged || eNew <= energy + 1e-4 * alpha * gtdx) {
          std::swap(d.x, d.xt);
          energy = eNew;
          accepted = true;
          phase(PH_COMMIT);
          if (contact) contact->commit(*this, d.x);
          break;
        }
        if (contact) contact->rejections++;
        alpha *= 0.5;
      }
      if (stop) break;
      if (!haveSlope) {
        read_scalars();
        pcgTotal += (int)hscal[S_PCG_ITERS];
        prof_collect((int)hscal[S_PCG_ITERS]);
      }
      if (!accepted) break;
      if (alpha < 1e-6) break;
    }
    phase(PH_OTHER);
    const double damp = 1 - std::min(std::max(mat.damping, 0.0), 0.1);
    launch_velocity(d, damp, stream);
    lc += 1;
    if (contact) contact->kill_approach_velocity(*this);
    launch_pins(d, d.x, stream);
    lc += (d.npins > 0);
    // keep the state in the primary buffer
    if (d.x != vx.p) {
      CK(cudaMemcpyAsync(vx.p, d.x, 3 * (size_t)mesh.n * 8, cudaMemcpyDeviceToDevice, stream));
      d.xt = d.x;
      d.x = vx.p;
    }
    stats = cs_step_stats{};
    stats.newton_iters = opts.newton_iters;
    stats.pcg_iters = pcgTotal;
    stats.grad_norm = gradNorm;
    stats.energy = energy;
    stats.max_strain = maxStrain;
    stats.converged = converged;
    stats.has_contact = contact ? 1 : 0;
    stats.newton_iters_used = used;
    stats.armijo_trials = trials;
    if (contact) contact->fill_stats(*this, stats);
    phase(PH_OTHER);
    haveStats = true;
  }

  // membraneHvp (fem.ts:108-130) at x along p; host arrays of 3n doubles.
  void membrane_hvp(const double* x, const double* p, double* out) {
    if (!ready) throw std::logic_error("CpuSolver not initialized");
    const size_t b = 3 * (size_t)mesh.n * 8;
    CK(cudaMemcpyAsync(vr.p, x, b, cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(vz.p, p, b, cudaMemcpyHostToDevice, stream));
    launch_membrane_hvp(idx.p, inv.p, area.p, d.mat, mesh.n, mesh.m, memOff.p, memRec.p, vr.p, vz.p, vAp.p, T3.p,
                        scal.p + S_CH3, elem.p, stream);
    launch_counter() += 4;
    CK(cudaMemcpyAsync(out, vAp.p, b, cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
  }

  // ---- material model (material-model.ts:232-296) on the current material ----------
  // energy: internalEnergyOnly (fem.ts:56-75); grad (3n, may be null):
  // evalInternal's gradient (fem.ts:15-54) with its max strain. Host arrays.
  void internal_eval(const double* x, double* energy, double* grad, double* maxStrain) {
    if (!ready) throw std::logic_error("CpuSolver not initialized");
    const size_t b = 3 * (size_t)mesh.n * 8;
    CK(cudaMemcpyAsync(vr.p, x, b, cudaMemcpyHostToDevice, stream));
    launch_internal_eval(d, vr.p, grad ? vAp.p : nullptr, scal.p + S_CH0, stream);
    launch_counter() += grad ? 4 + (d.kb > 0 && d.hg > 0) : 2;
    if (grad) CK(cudaMemcpyAsync(grad, vAp.p, b, cudaMemcpyDeviceToHost, stream));
    read_scalars();
    if (energy) *energy = hscal[S_CH0];
    if (maxStrain) *maxStrain = grad ? hscal[S_CH1] : 0.0;
  }
  // evalMembraneHvp (membrane-hvp.ts:80-108): analytic membrane HVP at x along p.
  void membrane_hvp_analytic(const double* x, const double* p, double* out) {
    if (!ready) throw std::logic_error("CpuSolver not initialized");
    const size_t b = 3 * (size_t)mesh.n * 8;
    CK(cudaMemcpyAsync(vr.p, x, b, cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(vz.p, p, b, cudaMemcpyHostToDevice, stream));
    launch_membrane_hvp_analytic(d, vr.p, vz.p, vAp.p, stream);
    launch_counter() += 2;
    CK(cudaMemcpyAsync(out, vAp.p, b, cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
  }

  // ---- differentiable rollout (no reference counterpart) -------------------------
  // forward(): `steps` steps of size h from the current state with the pins
  // fixed, keeping (x, v) at every K-th step start; backward(): the reverse
  // sweep through the implicit-function theorem, recomputing each K-step
  // segment from its checkpoint (one extra forward pass in total).
  struct Rollout {
    int steps = 0, K = 0;
    double h = 0;
    DBuf<double> ckX, ckV;   // checkpoints, 3n each
    DBuf<double> seg;        // the K states of the segment being reversed
    DBuf<double> xN, vN;     // state after the rollout
    bool valid = false;
  } ro;
  DBuf<double> adjRhs, adjMu, adjR, adjZ, adjP, adjAp, adjTri, adjHin, adjTerms, adjLamX, adjLamV, adjAcc, adjOut;
  AdjStats adjStats{};
  int adjMaxIters = 2000;
  double adjTol = 1e-10;
  // Newton linear solve: 0 = the reference's (FD membrane HVP, PCG to 1e-3);
  // 1 = full FP64 Hessian (membrane with clamped compression, bending, frozen
  // contact) solved to newtonTol, for rollouts that must converge tightly.
  int newtonMode = 0;
  double newtonTol = 1e-8;
  // Exact-Newton mode starts Newton from x0 + h v rather than yHat (k_predict);
  // CLOSIM_DRIFT_GUESS=0 keeps yHat.
  bool driftGuess = [] {
    const char* e = std::getenv("CLOSIM_DRIFT_GUESS");
    return !(e && std::string(e) == "0");
  }();

  // Relative PCG tolerance the FP32 solve of the exact-Newton mode is held to
  // at the tightest (single precision cannot resolve residuals much below it).
  static constexpr double kMixedTolFloor = 1e-5;
  // Per-CTA lists for the resident phase A of the one-cluster PCG, when the
  // largest CTA's share fits in shared memory (CLOSIM_MX_RESIDENT=0 turns it off).
  void build_cluster_resident() {
    clRes[0] = clRes[1] = false;
    clPlan = ClPlan{};
    const char* env = std::getenv("CLOSIM_MX_RESIDENT");
    if (env && std::string(env) == "0") return;
    build_cluster_plan(mesh, mxCluster, kClWarps, clHost);
    if (!clHost.ok) return;
    // the shared memory left over holds contact records (up to 8192 per CTA)
    for (int k = 0; k < 2; k++) {
      const size_t base = k ? clHost.smemHinge : clHost.smemNoHinge;
      const long room = (long)kClMaxDynSmem - (long)base - 32;
      clCap[k] = room > 0 ? (int)std::min<long>(room / kClRecBytes, 8192) : 0;
      clSmem[k] = base + 32 + (size_t)clCap[k] * kClRecBytes;
    }
    clRes[1] = mx_cluster_resident_ok(mxCluster, clSmem[1]);
    clRes[0] = mx_cluster_resident_ok(mxCluster, clSmem[0]);
    if (!clRes[0] && !clRes[1]) return;
    auto up = [&](DBuf<int>& b, const std::vector<int>& v) {
      b.alloc(std::max<size_t>(v.size(), 1));
      b.upload(v.data(), v.size(), stream);
      return (const int*)b.p;
    };
    clPlan.vb = up(clVb, clHost.vb);
    clPlan.haloOff = up(clHaloOff, clHost.haloOff);
    clPlan.halo = up(clHalo, clHost.halo);
    clPlan.triOff = up(clTriOff, clHost.triOff);
    clPlan.triId = up(clTriId, clHost.triId);
    clPlan.hinOff = up(clHinOff, clHost.hinOff);
    clPlan.hinId = up(clHinId, clHost.hinId);
    clPlan.incOff = up(clIncOff, clHost.incOff);
    clPlan.incHin = up(clIncHin, clHost.incHin);
    clPlan.ownHalo = up(clOwnHalo, clHost.ownHalo);
    clPlan.vDst = up(clVDst, clHost.vDst);
    clTriLoc.alloc(std::max<size_t>(clHost.triLoc.size(), 4));
    clTriLoc.upload(clHost.triLoc.data(), clHost.triLoc.size(), stream);
    clHinLoc.alloc(std::max<size_t>(clHost.hinLoc.size(), 4));
    clHinLoc.upload(clHost.hinLoc.data(), clHost.hinLoc.size(), stream);
    clInc.alloc(std::max<size_t>(clHost.inc.size(), 1));
    clInc.upload(clHost.inc.data(), clHost.inc.size(), stream);
    clPlan.triLoc = reinterpret_cast<const ushort4*>(clTriLoc.p);
    clPlan.hinLoc = reinterpret_cast<const ushort4*>(clHinLoc.p);
    clPlan.inc = clInc.p;
  }
  // The plan for a launch: resident when this launch's lists fit.
  ClPlan cluster_plan_for(const MixBufs& m) const {
    ClPlan p = clPlan;
    const int k = m.hrec ? 1 : 0;
    p.resident = clRes[k] && clHost.nrank == mxCluster && d.precond >= 1 ? 1 : 0;
    p.smemBytes = p.resident ? (int)clSmem[k] : 0;
    p.cCap = p.resident ? clCap[k] : 0;
    return p;
  }

  // Schwarz assembly records of the mixed factor (MixBufs::asmRec): static
  // topology, built once per mesh.
  DBuf<uint32_t> asmOffBuf;
  DBuf<uint2> asmRecBuf;
  void build_schwarz_assembly() {
    mb.asmOff = nullptr;
    mb.asmRec = nullptr;
    if (mesh.D == 0 || mesh.maxDomain > 8) return;
    const int n = mesh.n;
    std::vector<int> domOf(n, -1), member(n, -1);
    for (int dm = 0; dm < mesh.D; dm++)
      for (int l = mesh.domStart[dm]; l < mesh.domStart[dm + 1]; l++) {
        domOf[mesh.domVerts[l]] = dm;
        member[mesh.domVerts[l]] = l - mesh.domStart[dm];
      }
    std::vector<uint32_t> off(n + 1, 0);
    std::vector<uint2> rec;
    rec.reserve(mesh.v2t.size());
    for (int v = 0; v < n; v++) {
      off[v] = (uint32_t)rec.size();
      for (uint32_t k = mesh.v2tOff[v]; k < mesh.v2tOff[v + 1]; k++) {
        const uint32_t t = mesh.v2t[k];
        const int c0 = (int)mesh.idx[3 * (size_t)t], c1 = (int)mesh.idx[3 * (size_t)t + 1],
                  c2 = (int)mesh.idx[3 * (size_t)t + 2];
        const int ci = c0 == v ? 0 : c1 == v ? 1 : 2;
        uint32_t lw = 0;
        const int cs3[3] = {c0, c1, c2};
        for (int cj = 0; cj < 3; cj++) {
          const int w = cs3[cj];
          const uint32_t m = domOf[w] == domOf[v] && domOf[v] >= 0 ? (uint32_t)member[w] : 15u;
          lw |= m << (4 * cj);
        }
        rec.push_back(make_uint2(t * 81u + (uint32_t)ci * 27u, lw));
      }
    }
    off[n] = (uint32_t)rec.size();
    asmOffBuf.upload(off.data(), off.size(), stream);
    asmRecBuf.alloc(std::max<size_t>(rec.size(), 1));
    asmRecBuf.upload(rec.data(), rec.size(), stream);
    mb.asmOff = asmOffBuf.p;
    mb.asmRec = asmRecBuf.p;
  }

  DBuf<float4> hrecBuf;
  float4* ensure_hrec() {
    if (hrecBuf.n < 4 * (size_t)mesh.hg) hrecBuf.alloc(4 * (size_t)mesh.hg);
    return hrecBuf.p;
  }

  void ensure_adj_buffers() {
    const size_t n3 = 3 * (size_t)mesh.n;
    const int stride = mesh.m + mesh.hg;
    for (DBuf<double>* b : {&adjRhs, &adjMu, &adjR, &adjZ, &adjP, &adjAp, &adjLamX, &adjLamV})
      if (b->n < n3) b->alloc(n3);
    if (adjTri.n < 9 * (size_t)std::max(mesh.m, 1)) adjTri.alloc(9 * (size_t)std::max(mesh.m, 1));
    if (adjHin.n < 12 * (size_t)std::max(mesh.hg, 1)) adjHin.alloc(12 * (size_t)std::max(mesh.hg, 1));
    if (adjTerms.n < 4 * (size_t)std::max(stride, 1)) adjTerms.alloc(4 * (size_t)std::max(stride, 1));
    if (adjAcc.n < 4) adjAcc.alloc(4);
    if (adjOut.n < 3) adjOut.alloc(3);
  }

  void forward(double h, int steps, int K) {
    if (!ready) throw std::logic_error("CpuSolver not initialized");
    if (steps <= 0 || K <= 0) throw std::invalid_argument("steps and checkpoint interval must be positive");
    const size_t n3 = 3 * (size_t)mesh.n;
    const int nck = (steps + K - 1) / K;
    ro.valid = false;
    ro.steps = steps; ro.K = K; ro.h = h;
    ro.ckX.alloc(nck * n3);
    ro.ckV.alloc(nck * n3);
    ro.seg.alloc((size_t)K * n3);
    ro.xN.alloc(n3);
    ro.vN.alloc(n3);
    int conv = 0;
    for (int st = 0; st < steps; st++) {
      if (st % K == 0) {
        const size_t c = st / K;
        CK(cudaMemcpyAsync(ro.ckX.p + c * n3, d.x, n3 * 8, cudaMemcpyDeviceToDevice, stream));
        CK(cudaMemcpyAsync(ro.ckV.p + c * n3, d.v, n3 * 8, cudaMemcpyDeviceToDevice, stream));
      }
      step(h);
      conv += stats.converged ? 1 : 0;
    }
    adjStats.forwardConverged = conv;
    CK(cudaMemcpyAsync(ro.xN.p, d.x, n3 * 8, cudaMemcpyDeviceToDevice, stream));
    CK(cudaMemcpyAsync(ro.vN.p, d.v, n3 * 8, cudaMemcpyDeviceToDevice, stream));
    CK(cudaStreamSynchronize(stream));
    ro.valid = true;
  }

  // dLdxN: host 3n; dtheta: host 4 (C00, C11, G, k_bend); dv0: host 3n (may be null).
  void backward(const double* dLdxN, double* dtheta, double* dv0, int maxIters, double tol) {
    if (!ro.valid) throw std::logic_error("backward needs a forward rollout");
    const size_t n3 = 3 * (size_t)mesh.n;
    ensure_adj_buffers();
    CK(cudaMemcpyAsync(adjLamX.p, dLdxN, n3 * 8, cudaMemcpyHostToDevice, stream));
    CK(cudaMemsetAsync(adjLamV.p, 0, n3 * 8, stream));
    CK(cudaMemsetAsync(adjAcc.p, 0, 4 * 8, stream));
    const double damp = 1 - std::min(std::max(mat.damping, 0.0), 0.1);
    const double beta = std::max(std::max(mat.stretch_warp, mat.stretch_weft), mat.shear) * mat.thickness * 0.1 + 1e-6;
    const int blocks = adj_grid_blocks(d);
    double* const xPrimary = d.x;
    double* const x0Primary = d.x0;
    const int fwdConv = adjStats.forwardConverged;
    adjStats = AdjStats{};
    adjStats.forwardConverged = fwdConv;
    const int nck = (ro.steps + ro.K - 1) / ro.K;
    std::vector<double> hout(3);
    for (int c = nck - 1; c >= 0; c--) {
      const int s0 = c * ro.K, s1 = std::min(ro.steps, s0 + ro.K);
      // recompute the segment from its checkpoint
      CK(cudaMemcpyAsync(d.x, ro.ckX.p + (size_t)c * n3, n3 * 8, cudaMemcpyDeviceToDevice, stream));
      CK(cudaMemcpyAsync(d.v, ro.ckV.p + (size_t)c * n3, n3 * 8, cudaMemcpyDeviceToDevice, stream));
      for (int st = s0; st < s1; st++) {
        step(ro.h);
        CK(cudaMemcpyAsync(ro.seg.p + (size_t)(st - s0) * n3, d.x, n3 * 8, cudaMemcpyDeviceToDevice, stream));
        adjStats.recomputedSteps++;
      }
      for (int st = s1 - 1; st >= s0; st--) {
        double* x1 = ro.seg.p + (size_t)(st - s0) * n3;
        double* x0 = st == s0 ? ro.ckX.p + (size_t)c * n3 : ro.seg.p + (size_t)(st - s0 - 1) * n3;
        d.x = x1;
        d.x0 = x0;
        d.h = ro.h;
        d.invH2 = 1 / (ro.h * ro.h);
        if (contact) {
          contact->begin_segment(*this);
          contact->fricOn = false;  // the adjoint holds friction constant
          contact->update_active_set(*this, x1);
        }
        launch_diag_init(d, beta, stream);
        if (d.precond >= 1) launch_schwarz_factor(d, stream);
        adj_rhs(d, adjLamX.p, adjLamV.p, damp, adjRhs.p, stream);
        AdjArgs a{d, adjRhs.p, adjMu.p, adjR.p, adjZ.p, adjP.p, adjAp.p, adjTri.p, adjHin.p, d.kb, 0, maxIters, tol,
                  adjOut.p};
        CK((cudaError_t)adj_launch_pcg(a, blocks, stream));
        adj_theta(d, adjMu.p, adjTerms.p, adjAcc.p, stream);
        adj_propagate(d, adjMu.p, adjLamX.p, adjLamV.p, damp, stream);
        CK(cudaMemcpyAsync(hout.data(), adjOut.p, 3 * 8, cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        adjStats.pcgIters += (long)hout[0];
        adjStats.maxRelResidual = std::max(adjStats.maxRelResidual, hout[2] > 0 ? hout[1] / hout[2] : 0.0);
        adjStats.solves++;
        d.x = xPrimary;
        d.x0 = x0Primary;
      }
    }
    // dL/dv0 is the velocity adjoint after the first step's propagation
    std::vector<double> acc(4);
    CK(cudaMemcpyAsync(acc.data(), adjAcc.p, 4 * 8, cudaMemcpyDeviceToHost, stream));
    if (dv0) CK(cudaMemcpyAsync(dv0, adjLamV.p, n3 * 8, cudaMemcpyDeviceToHost, stream));
    // restore the state after the rollout
    CK(cudaMemcpyAsync(d.x, ro.xN.p, n3 * 8, cudaMemcpyDeviceToDevice, stream));
    CK(cudaMemcpyAsync(d.v, ro.vN.p, n3 * 8, cudaMemcpyDeviceToDevice, stream));
    CK(cudaStreamSynchronize(stream));
    if (dtheta) for (int j = 0; j < 4; j++) dtheta[j] = acc[j];
    if (contact) contact->bind(*this);
  }

  // ---- SimulationSession hand-off (sim-session.ts:120-150) ----------------------
  DBuf<double> stableX;
  DBuf<int> nanFlag;
  int* hNan = nullptr;  // pinned mirror of nanFlag
  int stableStep = -1, sessionSteps = 0;

  void session_reset() {
    if (!ready) throw std::logic_error("CpuSolver not initialized");
    const size_t n3 = 3 * (size_t)mesh.n;
    if (stableX.n < n3) stableX.alloc(n3);
    if (nanFlag.n < 1) nanFlag.alloc(1);
    if (!hNan) CK(cudaMallocHost(&hNan, sizeof(int)));
    CK(cudaMemcpyAsync(stableX.p, d.x, n3 * 8, cudaMemcpyDeviceToDevice, stream));
    CK(cudaStreamSynchronize(stream));
    stableStep = 0;
    sessionSteps = 0;
  }

  // One step, the NaN check and the stable snapshot on the device, then the
  // positions into `out` (pinned host memory is fastest) with one sync.
  bool session_step(double h, double* out) {
    if (stableStep < 0) session_reset();
    step(h);
    sessionSteps++;
    const size_t n3 = 3 * (size_t)mesh.n;
    launch_session_check(d.x, stableX.p, (int)n3, nanFlag.p, stream);
    launch_counter() += 2;
    CK(cudaMemcpyAsync(hNan, nanFlag.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    if (out) CK(cudaMemcpyAsync(out, d.x, n3 * 8, cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    const bool finite = *hNan == 0;
    if (finite) stableStep = sessionSteps;
    return finite;
  }

  // restoreStable: positions <- the last NaN-free state, velocities <- 0.
  bool session_restore() {
    if (stableStep < 0) return false;
    const size_t n3 = 3 * (size_t)mesh.n;
    CK(cudaMemcpyAsync(d.x, stableX.p, n3 * 8, cudaMemcpyDeviceToDevice, stream));
    CK(cudaMemsetAsync(d.v, 0, n3 * 8, stream));
    CK(cudaStreamSynchronize(stream));
    return true;
  }

  void get(double* out, bool vel) {
    CK(cudaMemcpyAsync(out, vel ? d.v : d.x, 3 * (size_t)mesh.n * 8, cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
  }
  void set_state(const double* x, const double* v) {
    if (x) CK(cudaMemcpyAsync(d.x, x, 3 * (size_t)mesh.n * 8, cudaMemcpyHostToDevice, stream));
    if (v) CK(cudaMemcpyAsync(d.v, v, 3 * (size_t)mesh.n * 8, cudaMemcpyHostToDevice, stream));
    CK(cudaStreamSynchronize(stream));
  }
};

}  // namespace cs

