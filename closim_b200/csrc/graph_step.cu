// One implicit-Euler step (newton.ts:27-232) as a captured CUDA graph with the
// Newton / Armijo / trust-region control decided on the device.
//
// The host-driven step (Solver::step) reads a few scalars back at every
// decision: the active-set counts, the gradient norm, each Armijo trial's
// validity and energy. Here the step is captured once into a graph whose
// decisions are one-thread kernels setting conditional nodes:
//
//   predictor, superset, predictor check, bisection  WHILE (<= 8 probes)
//   active set, merit energy, Jacobi diagonal
//   Newton                                            WHILE (<= newtonIters)
//     active set + contact terms, gradient, [exact: friction potential, base energy]
//     convergence test                                IF (solve)
//       preconditioner, one-cluster PCG + descent safeguard + trust region
//       Armijo                                        WHILE (<= lineSearchIters)
//         trial x + alpha dx, CCD-gated validity, trial energy, accept / halve
//       accepted                                      IF: x <- trial, commit lags
//   velocity, restitution pass, pins
//
// and every broadphase query carries an IF node that rebuilds the pair
// superset when the query left it. A replay is one launch and one host read of
// the step's state. The arithmetic is the host-driven step's: the same kernels
// in the same order, the decisions restated on the device (compiled without
// FMA contraction, as the host compares). Buffer overflows are reported on the
// device; the step is then restored and repeated on the host-driven path with
// grown buffers. Scope: the mixed path's one-cluster PCG (sheets up to about
// 20,000 vertices); other configurations take the host-driven step.
#include <cstring>

#include "graph_ctx.hpp"
#include "solver.hpp"

namespace cs {

// Control state of a captured step (device), read by the host after a replay.
struct GState {
  double alpha, energy, gradNorm, maxStrain, rejections;
  double bisLo, bisHi;
  int ni, used, trials, li, accepted, stop, converged, nonfinite, pcgTotal, solves, accepts, bisIters;
  int valid0, bisected, lsIters, newtonIters;
  int haveTrial, pad;
};

__global__ void k_g_init(GState* g, int newtonIters, int lsIters, cudaGraphConditionalHandle hNewton) {
  GState z{};
  z.alpha = 1;
  z.gradNorm = INFINITY;
  z.newtonIters = newtonIters;
  z.lsIters = lsIters;
  *g = z;
  (void)hNewton;
}

// Bisection of the predictor (newton.ts:56-72): starts when the predictor is not CCD-valid.
__global__ void k_g_bis_init(GState* g, const int* cint, cudaGraphConditionalHandle hBis) {
  const int valid = cint[CI_VALID];
  g->valid0 = valid;
  g->bisLo = 0;
  g->bisHi = 1;
  g->bisected = valid ? 0 : 1;
  cudaGraphSetConditional(hBis, valid ? 0u : 1u);
}
__global__ void k_g_lerp_mid(double* out, const double* x0, const double* x, const GState* g, int n3) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double mid = 0.5 * (g->bisLo + g->bisHi);
  if (i < n3) out[i] = x0[i] + mid * (x[i] - x0[i]);
}
__global__ void k_g_bis_update(GState* g, const int* cint, cudaGraphConditionalHandle hBis) {
  const double mid = 0.5 * (g->bisLo + g->bisHi);
  if (cint[CI_VALID] == 1) g->bisLo = mid;
  else g->bisHi = mid;
  g->bisIters++;
  const bool more = g->bisIters < 8 && !(g->bisHi - g->bisLo < 1e-4);
  cudaGraphSetConditional(hBis, more ? 1u : 0u);
}
__global__ void k_g_lerp_lo(double* x, const double* x0, const GState* g, int n3) {
  if (!g->bisected) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double lo = g->bisLo;
  if (i < n3) x[i] = x0[i] + lo * (x[i] - x0[i]);
}
__global__ void k_g_pins_if_bisected(Dev d, const GState* g) {
  if (!g->bisected) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= d.npins) return;
  const int id = d.pinIds[k];
  d.x[id * 3] = d.pinPos[k * 3];
  d.x[id * 3 + 1] = d.pinPos[k * 3 + 1];
  d.x[id * 3 + 2] = d.pinPos[k * 3 + 2];
}

__global__ void k_g_energy0(GState* g, const double* scal, cudaGraphConditionalHandle hNewton) {
  g->energy = scal[S_ENERGY_TRIAL];
  cudaGraphSetConditional(hNewton, g->newtonIters > 0 ? 1u : 0u);
}

// Convergence test of a Newton iteration (newton.ts:126-130).
// meritAgain: the base energy was re-evaluated at x (exact-Newton mode).
__global__ void k_g_newton_check(GState* g, const double* scal, double gradTol, int meritAgain,
                                 cudaGraphConditionalHandle hSolve, cudaGraphConditionalHandle hNewton) {
  g->used = g->ni + 1;
  const double gn = scal[S_GRADNORM];
  g->gradNorm = gn;
  g->maxStrain = scal[S_MAXSTRAIN];
  if (meritAgain) g->energy = scal[S_ENERGY_TRIAL];
  bool solve = true;
  if (!isfinite(gn)) {
    g->nonfinite = 1;
    solve = false;
  } else if (gn < gradTol) {
    g->converged = 1;
    solve = false;
  }
  if (!solve) {
    g->stop = 1;
    cudaGraphSetConditional(hNewton, 0u);
  }
  cudaGraphSetConditional(hSolve, solve ? 1u : 0u);
}

__global__ void k_g_ls_init(GState* g, cudaGraphConditionalHandle hTrial, cudaGraphConditionalHandle hAccept) {
  g->alpha = 1;
  g->li = 0;
  g->accepted = 0;
  g->solves++;
  cudaGraphSetConditional(hTrial, g->lsIters > 0 ? 1u : 0u);
  cudaGraphSetConditional(hAccept, 0u);
}
__global__ void k_g_trial_x(Dev d, const GState* g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n * 3) return;
  d.xt[i] = d.x[i] + g->alpha * d.dx[i];
}
// One Armijo trial's decision (newton.ts:181-219): CCD validity, a finite
// energy, sufficient decrease c1 = 1e-4; else halve alpha.
__global__ void k_g_ls_decide(GState* g, const double* scal, const int* cint, int exactMode,
                              cudaGraphConditionalHandle hTrial, cudaGraphConditionalHandle hAccept) {
  g->trials++;
  g->li++;
  const double alpha = g->alpha;
  bool accept = false;
  if (cint[CI_VALID] == 1) {
    const double eNew = scal[S_ENERGY_TRIAL];
    if (isfinite(eNew)) {
      const bool nearConverged = exactMode && g->gradNorm < 1e-7 && alpha == 1;
      if (nearConverged || eNew <= g->energy + 1e-4 * alpha * scal[S_GTDX]) {
        accept = true;
        g->energy = eNew;
      }
    }
  }
  if (accept) {
    g->accepted = 1;
    g->accepts++;
  } else {
    g->rejections += 1;
    g->alpha = alpha * 0.5;
  }
  const bool more = !accept && g->li < g->lsIters;
  cudaGraphSetConditional(hTrial, more ? 1u : 0u);
  cudaGraphSetConditional(hAccept, accept ? 1u : 0u);
}
// End of a Newton iteration that solved (newton.ts:214-219).
__global__ void k_g_after(GState* g, const double* scal, cudaGraphConditionalHandle hNewton) {
  g->pcgTotal += (int)scal[S_PCG_ITERS];
  bool stop = !g->accepted || g->alpha < 1e-6;
  g->ni++;
  if (g->ni >= g->newtonIters) stop = true;
  if (stop) g->stop = 1;
  cudaGraphSetConditional(hNewton, stop ? 0u : 1u);
}

struct Solver::GraphStep {
  cudaGraphExec_t exec = nullptr;
  std::vector<double> key;
  GState* gs = nullptr;      // device
  GState* hgs = nullptr;     // pinned
  int* hacnt = nullptr;      // pinned AC_N
  double* v0 = nullptr;      // velocities at the step start (restored on fallback)
  size_t v0n = 0;
  // kernel launches per section, counted at capture, for the launch tally
  int64_t lTop = 0, lBis = 0, lNewton = 0, lSolve = 0, lTrial = 0, lAccept = 0;
  bool failed = false;       // capture or instantiation failed once: host-driven from then on
  GraphCtx ctx;
  ~GraphStep() {
    if (exec) cudaGraphExecDestroy(exec);
    if (gs) cudaFree(gs);
    if (hgs) cudaFreeHost(hgs);
    if (hacnt) cudaFreeHost(hacnt);
    if (v0) cudaFree(v0);
  }
};

void Solver::graph_release() {
  delete gstep;
  gstep = nullptr;
}

std::vector<double> Solver::graph_key(double h) const {
  std::vector<double> k = {h, (double)opts.newton_iters, (double)opts.pcg_max_iters, (double)opts.ls_iters,
                           (double)opts.precond, opts.grad_tol, (double)newtonMode, newtonTol, (double)mxCluster,
                           (double)d.npins, (double)(uintptr_t)d.pinIds, (double)(uintptr_t)d.pinPos,
                           (double)initEpoch, (double)(uintptr_t)hrecBuf.p, gravity[0], gravity[1], gravity[2],
                           (double)driftGuess};
  const double m[9] = {mat.areal_density, mat.thickness, mat.stretch_warp, mat.stretch_weft, mat.stretch_coupling,
                       mat.shear, mat.bend_warp, mat.bend_weft, mat.damping};
  k.insert(k.end(), m, m + 9);
  if (contact) {
    const ContactHost& c = *contact;
    const double cc[] = {(double)(uintptr_t)&c, (double)c.cand.cap, (double)c.actCap, (double)c.lagCap,
                         (double)c.pairCap, (double)c.spairCap, (double)c.supCap, (double)c.supSCap,
                         (double)c.flagCap};
    k.insert(k.end(), cc, cc + sizeof cc / sizeof cc[0]);
  }
  return k;
}

void Solver::graph_capture(double h) {
  GraphStep& G = *gstep;
  GraphCtx& g = G.ctx;
  int64_t& lc = launch_counter();
  const int64_t lc0 = lc;
  const int n3 = 3 * mesh.n;
  auto nb = [](long k) { return (int)((k + kThreads - 1) / kThreads); };
  // the Dev the captured launches see: primary buffers, this step's h
  d.h = h;
  d.invH2 = 1 / (h * h);
  for (int k = 0; k < 3; k++) d.gravity[k] = gravity[k];
  d.precond = precond_code();
  d.hasContact = contact ? 1 : 0;
  d.driftGuess = newtonMode == 1 && driftGuess ? 1 : 0;
  d.x = vx.p;
  d.xt = vxt.p;
  const bool exactMode = newtonMode == 1;
  mb.psd = exactMode ? 1 : 0;
  mb.hrec = exactMode && d.kb > 0 && d.hg > 0 ? ensure_hrec() : nullptr;
  mb.dcoarse = d.precond == 2 ? fdc.p : nullptr;
  const bool fricExact = exactMode && contact && contact->p.mu > 0;
  // Exact-Newton mode re-evaluates the Armijo base energy at x after each
  // active-set update (and friction freeze): contacts that enter the set while
  // Newton moves the sheet would otherwise be missing from the base energy but
  // present in every trial's, and the line search would reject every step.
  const bool meritAgain = exactMode && contact;
  const double beta = std::max(std::max(mat.stretch_warp, mat.stretch_weft), mat.shear) * mat.thickness * 0.1 + 1e-6;
  const double damp = 1 - std::min(std::max(mat.damping, 0.0), 0.1);
  const double pcgTol = exactMode ? std::max(newtonTol, kMixedTolFloor) : 1e-3;
  int* cint = contact ? contact->cint : nullptr;

  g.begin(stream);
  auto energy = [&](const double* x) {
    if (contact) contact->cap_merit_energy(*this, g, x);
    launch_energy_terms(d, x, g.cur());
    lc += 1;
    mx_energy_final(d, g.cur(), &lc);
  };
  cudaGraphConditionalHandle hNewton = g.handle(1);
  k_g_init<<<1, 1, 0, g.cur()>>>(G.gs, opts.newton_iters, opts.ls_iters, hNewton);
  GCK(cudaMemcpyAsync(G.v0, d.v, (size_t)n3 * 8, cudaMemcpyDeviceToDevice, g.cur()));
  launch_predict(d, g.cur());
  lc += 2 + (d.npins > 0);
  if (contact) {
    contact->cap_begin_step(*this, g);
    contact->cap_superset_step(*this, g, d.x);
    contact->cap_trial(*this, g, d.x);
    const cudaGraphConditionalHandle hBis = g.handle(0);
    k_g_bis_init<<<1, 1, 0, g.cur()>>>(G.gs, cint, hBis);
    lc++;
    const int64_t b0 = lc;
    g.push(hBis, cudaGraphCondTypeWhile);
    k_g_lerp_mid<<<nb(n3), kThreads, 0, g.cur()>>>(contact->probe, d.x0, d.x, G.gs, n3);
    launch_pins(d, contact->probe, g.cur());
    lc += 1 + (d.npins > 0);
    contact->cap_trial(*this, g, contact->probe);
    k_g_bis_update<<<1, 1, 0, g.cur()>>>(G.gs, cint, hBis);
    lc++;
    g.pop();
    G.lBis = lc - b0;
    k_g_lerp_lo<<<nb(n3), kThreads, 0, g.cur()>>>(d.x, d.x0, G.gs, n3);
    if (d.npins > 0) k_g_pins_if_bisected<<<nb(d.npins), kThreads, 0, g.cur()>>>(d, G.gs);
    lc += 1 + (d.npins > 0);
    contact->cap_update_active_set(*this, g, d.x);
  }
  energy(d.x);
  launch_diag_init(d, beta, g.cur());
  k_g_energy0<<<1, 1, 0, g.cur()>>>(G.gs, scal.p, hNewton);
  lc += 2;

  // ---- Newton -----------------------------------------------------------------------
  const int64_t n0 = lc;
  int64_t inner = 0;
  g.push(hNewton, cudaGraphCondTypeWhile);
  {
    if (contact) contact->cap_gradient_terms(*this, g);
    launch_grad_terms(d, g.cur(), true);
    lc += 2 + (d.kb > 0 && d.hg > 0);
    mx_grad_final(d, g.cur(), &lc);
    if (fricExact) contact->cap_friction_terms(*this, g);
    if (meritAgain) energy(d.x);
    const cudaGraphConditionalHandle hSolve = g.handle(0);
    k_g_newton_check<<<1, 1, 0, g.cur()>>>(G.gs, scal.p, opts.grad_tol, meritAgain ? 1 : 0, hSolve, hNewton);
    lc++;
    const int64_t s0 = lc;
    g.push(hSolve, cudaGraphCondTypeIf);
    {
      mx_prepare(d, mb, d.precond >= 1, g.cur(), &lc);
      GCK((cudaError_t)mx_launch_pcg_cluster(d, mb, cluster_plan_for(mb), fp.p, fp2.p, contact ? contact->dd : nullptr,
                                             opts.pcg_max_iters, pcgTol, mxCluster, g.cur()));
      lc++;
      const cudaGraphConditionalHandle hTrial = g.handle(0);
      const cudaGraphConditionalHandle hAccept = g.handle(0);
      k_g_ls_init<<<1, 1, 0, g.cur()>>>(G.gs, hTrial, hAccept);
      lc++;
      const int64_t t0 = lc;
      g.push(hTrial, cudaGraphCondTypeWhile);
      {
        k_g_trial_x<<<nb(n3), kThreads, 0, g.cur()>>>(d, G.gs);
        launch_pins(d, d.xt, g.cur());
        lc += 1 + (d.npins > 0);
        if (contact) contact->cap_trial(*this, g, d.xt);
        energy(d.xt);
        k_g_ls_decide<<<1, 1, 0, g.cur()>>>(G.gs, scal.p, cint ? cint : contact_free_valid(), exactMode ? 1 : 0,
                                            hTrial, hAccept);
        lc++;
      }
      g.pop();
      G.lTrial = lc - t0;
      const int64_t a0 = lc;
      g.push(hAccept, cudaGraphCondTypeIf);
      {
        GCK(cudaMemcpyAsync(d.x, d.xt, (size_t)n3 * 8, cudaMemcpyDeviceToDevice, g.cur()));
        if (contact) {
          contact->cap_commit(*this, g, d.x);
          contact->cap_mark_moved(g);
        }
      }
      g.pop();
      G.lAccept = lc - a0;
      k_g_after<<<1, 1, 0, g.cur()>>>(G.gs, scal.p, hNewton);
      lc++;
      inner = G.lTrial + G.lAccept;
    }
    g.pop();
    G.lSolve = lc - s0 - inner;
    inner += G.lSolve;
  }
  g.pop();
  G.lNewton = lc - n0 - inner;

  // ---- velocity, restitution, pins (newton.ts:221-232) -----------------------------------
  launch_velocity(d, damp, g.cur());
  lc++;
  if (contact) contact->cap_kill_approach_velocity(*this, g);
  launch_pins(d, d.x, g.cur());
  lc += (d.npins > 0);
  GCK(cudaMemcpyAsync(G.hgs, G.gs, sizeof(GState), cudaMemcpyDeviceToHost, g.cur()));
  if (contact) {
    GCK(cudaMemcpyAsync(G.hacnt, contact->acnt, AC_N * sizeof(int), cudaMemcpyDeviceToHost, g.cur()));
    GCK(cudaMemcpyAsync(contact->hint, contact->cint, CI_N * sizeof(int), cudaMemcpyDeviceToHost, g.cur()));
    GCK(cudaMemcpyAsync(contact->hdiag, contact->diag, sizeof(DevDiag), cudaMemcpyDeviceToHost, g.cur()));
  }
  cudaGraph_t graph = g.end();
  G.lTop = lc - lc0 - G.lNewton - G.lSolve - G.lTrial - G.lAccept - G.lBis;
  lc = lc0;  // capture launches nothing; replays are tallied from the section counts
  if (G.exec) {
    cudaGraphExecDestroy(G.exec);
    G.exec = nullptr;
  }
  const cudaError_t e = cudaGraphInstantiate(&G.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    G.exec = nullptr;
    throw GraphError(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  }
}

// Without contact the Armijo decision reads an always-valid flag.
const int* Solver::contact_free_valid() {
  if (!validOne.p) {
    validOne.alloc(CI_N);
    std::vector<int> one(CI_N, 0);
    one[CI_VALID] = 1;
    CK(cudaMemcpy(validOne.p, one.data(), CI_N * sizeof(int), cudaMemcpyHostToDevice));
  }
  return validOne.p;
}

bool Solver::step_graph(double h) {
  if (!graphMode || !mixed() || mxCluster <= 0 || prof || profPhases) return false;
  if (!gstep) gstep = new GraphStep();
  GraphStep& G = *gstep;
  if (G.failed) return false;
  const size_t n3 = 3 * (size_t)mesh.n;
  if (!G.gs) {
    CK(cudaMalloc(&G.gs, sizeof(GState)));
    CK(cudaMallocHost(&G.hgs, sizeof(GState)));
    CK(cudaMallocHost(&G.hacnt, AC_N * sizeof(int)));
  }
  if (G.v0n < n3) {
    if (G.v0) cudaFree(G.v0);
    CK(cudaMalloc(&G.v0, n3 * 8));
    G.v0n = n3;
  }
  if (newtonMode == 1 && d.kb > 0 && d.hg > 0) ensure_hrec();  // allocated before the key is taken
  if (!contact) contact_free_valid();                            // no allocation during a capture
  const std::vector<double> key = graph_key(h);
  if (!G.exec || key != G.key) {
    try {
      graph_capture(h);
      G.key = key;
    } catch (const GraphError&) {
      // capture failed: leave the stream out of capture mode and step on the host from now on
      cudaStreamCaptureStatus st;
      if (cudaStreamIsCapturing(stream, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(stream, &junk);
        if (junk) cudaGraphDestroy(junk);
      }
      cudaGetLastError();
      G.failed = true;
      if (contact) contact->bind(*this);
      return false;
    }
  }
  CK(cudaGraphLaunch(G.exec, stream));
  CK(cudaStreamSynchronize(stream));
  const GState& st = *G.hgs;
  int64_t& lc = launch_counter();
  lc += G.lTop + G.lBis * st.bisIters + G.lNewton * std::max(st.used, 0) + G.lSolve * st.solves +
        G.lTrial * st.trials + G.lAccept * st.accepts;
  if (contact && G.hacnt[AC_ERR]) {
    // a buffer was too small: restore the step's start and repeat it on the host path
    CK(cudaMemcpyAsync(d.x, d.x0, n3 * 8, cudaMemcpyDeviceToDevice, stream));
    CK(cudaMemcpyAsync(d.v, G.v0, n3 * 8, cudaMemcpyDeviceToDevice, stream));
    contact->cap_grow(*this, G.hacnt, contact->hint);
    contact->bind(*this);
    CK(cudaStreamSynchronize(stream));
    graphFallbacks++;
    return false;
  }
  if (st.nonfinite) throw NonFinite();
  stats = cs_step_stats{};
  stats.newton_iters = opts.newton_iters;
  stats.pcg_iters = st.pcgTotal;
  stats.grad_norm = st.gradNorm;
  stats.energy = st.energy;
  stats.max_strain = st.maxStrain;
  stats.converged = st.converged;
  stats.has_contact = contact ? 1 : 0;
  stats.newton_iters_used = st.used;
  stats.armijo_trials = st.trials;
  if (contact) {
    contact->cap_collect(G.hacnt, contact->hint, st.rejections);
    if (contact->hdiag->killStall != 0) throw std::runtime_error("restitution pass did not complete");
    stats.candidate_pairs = contact->candidatePairs;
    stats.active_pairs = contact->activePairs;
    stats.vt_pairs = contact->vtPairs;
    stats.ee_pairs = contact->eePairs;
    stats.floor_pairs = contact->floorPairs;
    stats.min_distance = contact->hdiag->minDistance;
    stats.min_toi = contact->hdiag->minTOI;
    stats.barrier_energy = contact->hdiag->barrierEnergy;
    stats.friction_work = contact->hdiag->frictionWork;
    stats.rejected_line_search_steps = st.rejections;
    stats.ccd_failures = contact->hdiag->ccdFailures;
    contact->bind(*this);  // host-driven view for calls between steps
  }
  haveStats = true;
  graphSteps++;
  return true;
}

}  // namespace cs
