// Host orchestration of the CUDA cloth step and the C ABI (include/closim_cuda.h).
//
// The Newton / Armijo control of src/solver/newton.ts:27-232 runs on the host
// over device-resident state (solver.hpp); each decision reads back a few
// scalars written by the kernels through pinned memory.
#include "solver.hpp"

// ---- C ABI -----------------------------------------------------------------------
struct cs_solver {
  cs::Solver s;
  std::string err;
};

template <class F>
static int guarded(cs_solver* h, F&& f) {
  if (!h) return CS_E_ARG;
  try {
    f();
    h->err.clear();
    return CS_OK;
  } catch (const cs::NonFinite& e) {
    h->err = e.what();
    return CS_E_NONFINITE;
  } catch (const cs::CudaError& e) {
    h->err = e.what();
    return CS_E_CUDA;
  } catch (const cs::CapacityError& e) {
    h->err = e.what();
    return CS_E_CAPACITY;
  } catch (const std::logic_error& e) {
    h->err = e.what();
    return std::string(e.what()).find("not initialized") != std::string::npos ? CS_E_UNINIT : CS_E_ARG;
  } catch (const std::exception& e) {
    h->err = e.what();
    return CS_E_ARG;
  }
}

extern "C" {

cs_solver* cs_create(int precision, int device) {
  if (precision != CS_PRECISION_FP64 && precision != CS_PRECISION_MIXED) return nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return nullptr;
  cs_solver* h = new cs_solver();
  try {
    h->s.create(precision, device);
  } catch (...) {
    delete h;
    return nullptr;
  }
  return h;
}
void cs_destroy(cs_solver* h) { delete h; }
const char* cs_last_error(cs_solver* h) { return h ? h->err.c_str() : "null handle"; }

int cs_initialize(cs_solver* h, const cs_mesh* mesh, const cs_material* mat, const double gravity[3],
                  const double* x, const double* v) {
  return guarded(h, [&] {
    if (!mesh || !mat || !x) throw std::invalid_argument("null argument");
    h->s.initialize(*mesh, *mat, gravity, x, v);
  });
}
int cs_set_contact(cs_solver* h, const cs_contact_params* p, int floor_on, double floor_y, const float* sp,
                   int32_t ns, const uint32_t* si, int32_t ms) {
  return guarded(h, [&] {
    if (!h->s.ready) throw std::logic_error("CpuSolver not initialized");
    cs::set_contact(h->s, p, floor_on, floor_y, sp, ns, si, ms);
  });
}
int cs_set_stepper_options(cs_solver* h, const cs_stepper_options* o) {
  return guarded(h, [&] {
    if (!o || o->newton_iters < 0 || o->pcg_max_iters < 0 || o->ls_iters < 0) throw std::invalid_argument("bad options");
    if (o->precond != CS_PRECOND_JACOBI && o->precond != CS_PRECOND_SCHWARZ && o->precond != CS_PRECOND_MAS2)
      throw std::invalid_argument("bad precond");
    h->s.opts = *o;
  });
}
int cs_set_material(cs_solver* h, const cs_material* m) {
  return guarded(h, [&] {
    if (!h->s.ready) throw std::logic_error("CpuSolver not initialized");
    if (!m) throw std::invalid_argument("null material");
    h->s.set_material(*m);
  });
}
int cs_set_pins(cs_solver* h, int32_t k, const int32_t* ids, const double* pos) {
  return guarded(h, [&] {
    if (k < 0 || (k > 0 && (!ids || !pos))) throw std::invalid_argument("bad pins");
    h->s.set_pins(k, ids, pos);
  });
}
int cs_step(cs_solver* h, double dt) {
  return guarded(h, [&] {
    if (!(dt > 0) || !std::isfinite(dt)) throw std::invalid_argument("dt must be positive");
    h->s.step(dt);
  });
}
int cs_step_n(cs_solver* h, double dt, int32_t nsteps) {
  return guarded(h, [&] {
    if (!(dt > 0)) throw std::invalid_argument("dt must be positive");
    for (int i = 0; i < nsteps; i++) h->s.step(dt);
  });
}
int cs_get_positions(cs_solver* h, double* out) {
  return guarded(h, [&] {
    if (!h->s.ready) throw std::logic_error("CpuSolver not initialized");
    h->s.get(out, false);
  });
}
int cs_get_velocities(cs_solver* h, double* out) {
  return guarded(h, [&] {
    if (!h->s.ready) throw std::logic_error("CpuSolver not initialized");
    h->s.get(out, true);
  });
}
int cs_set_state(cs_solver* h, const double* x, const double* v) {
  return guarded(h, [&] {
    if (!h->s.ready) throw std::logic_error("CpuSolver not initialized");
    h->s.set_state(x, v);
  });
}
int cs_membrane_hvp(cs_solver* h, const double* x, const double* p, double* out) {
  return guarded(h, [&] {
    if (!x || !p || !out) throw std::invalid_argument("null argument");
    h->s.membrane_hvp(x, p, out);
  });
}
int cs_internal_energy(cs_solver* h, const double* x, double* energy) {
  return guarded(h, [&] {
    if (!x || !energy) throw std::invalid_argument("null argument");
    h->s.internal_eval(x, energy, nullptr, nullptr);
  });
}
int cs_internal_gradient(cs_solver* h, const double* x, double* energy, double* grad, double* max_strain) {
  return guarded(h, [&] {
    if (!x || !grad) throw std::invalid_argument("null argument");
    h->s.internal_eval(x, energy, grad, max_strain);
  });
}
int cs_membrane_hvp_analytic(cs_solver* h, const double* x, const double* p, double* out) {
  return guarded(h, [&] {
    if (!x || !p || !out) throw std::invalid_argument("null argument");
    h->s.membrane_hvp_analytic(x, p, out);
  });
}
int cs_contact_active(cs_solver* h, int32_t cap, int32_t* count, int32_t* ids6, double* w7) {
  int rc = CS_OK;
  const int g = guarded(h, [&] {
    if (!count) throw std::invalid_argument("null argument");
    if (!h->s.ready) throw std::logic_error("CpuSolver not initialized");
    *count = h->s.contact ? h->s.contact->read_active(h->s, cap, ids6, w7) : 0;
    if (*count > cap && ids6) rc = CS_E_CAPACITY;
  });
  return g != CS_OK ? g : rc;
}
int cs_update_static_positions(cs_solver* h, const float* static_pos, int32_t ns) {
  return guarded(h, [&] {
    if (!static_pos) throw std::invalid_argument("null argument");
    if (!h->s.ready) throw std::logic_error("CpuSolver not initialized");
    if (!h->s.contact) throw std::invalid_argument("no contact system");
    h->s.contact->update_static_positions(h->s, static_pos, ns);
  });
}
int cs_set_graph_mode(cs_solver* h, int32_t enable) {
  return guarded(h, [&] {
    if (enable != 0 && enable != 1) throw std::invalid_argument("graph mode is 0 or 1");
    h->s.graphMode = enable;
  });
}
int cs_graph_info(cs_solver* h, int64_t* out2) {
  return guarded(h, [&] {
    if (!out2) throw std::invalid_argument("null argument");
    out2[0] = h->s.graphSteps;
    out2[1] = h->s.graphFallbacks;
  });
}
int cs_last_stats(cs_solver* h, cs_step_stats* out) {
  return guarded(h, [&] {
    if (!h->s.haveStats) throw std::logic_error("CpuSolver not initialized: no step taken");
    *out = h->s.stats;
  });
}
int cs_sync(cs_solver* h) {
  return guarded(h, [&] {
    cudaError_t e = cudaStreamSynchronize(h->s.stream);
    if (e != cudaSuccess) throw cs::CudaError(cudaGetErrorString(e));
  });
}
int64_t cs_kernel_launches(cs_solver* h) { return h ? cs::launch_counter() : 0; }
void* cs_stream(cs_solver* h) { return h ? (void*)h->s.stream : nullptr; }
int cs_profile(cs_solver* h, int enable) {
  return guarded(h, [&] {
    h->s.prof = enable != 0;
    h->s.profPhases = enable == 2;
    for (double& v : h->s.phaseMs) v = 0;
    h->s.profMs = h->s.profLaunches = h->s.profBytes = h->s.profIters = 0;
    h->s.profPending = false;
  });
}
int cs_profile_read(cs_solver* h, double* out) {
  return guarded(h, [&] {
    if (!out) throw std::invalid_argument("null output");
    out[0] = h->s.profMs;
    out[1] = h->s.profLaunches;
    out[2] = h->s.profBytes;
    out[3] = h->s.profIters;
    out[4] = h->s.profLaunches > 0 ? h->s.profMs / h->s.profLaunches : 0.0;
  });
}

int cs_forward(cs_solver* h, double dt, int32_t steps, int32_t checkpoint_every) {
  return guarded(h, [&] { h->s.forward(dt, steps, checkpoint_every); });
}

int cs_backward(cs_solver* h, const double* dL_dxN, double* dL_dtheta, double* dL_dv0) {
  return guarded(h, [&] {
    if (!dL_dxN) throw std::invalid_argument("null dL/dx_N");
    h->s.backward(dL_dxN, dL_dtheta, dL_dv0, h->s.adjMaxIters, h->s.adjTol);
  });
}

int cs_set_adjoint_options(cs_solver* h, int32_t max_iters, double tol) {
  return guarded(h, [&] {
    if (max_iters <= 0 || !(tol > 0)) throw std::invalid_argument("bad adjoint options");
    h->s.adjMaxIters = max_iters;
    h->s.adjTol = tol;
  });
}

int cs_set_newton_mode(cs_solver* h, int32_t mode, double tol) {
  return guarded(h, [&] {
    if ((mode != 0 && mode != 1) || !(tol > 0)) throw std::invalid_argument("bad Newton mode");
    h->s.newtonMode = mode;
    h->s.newtonTol = tol;
  });
}

int cs_adjoint_stats(cs_solver* h, double* out5) {
  return guarded(h, [&] {
    if (!out5) throw std::invalid_argument("null output");
    out5[0] = (double)h->s.adjStats.pcgIters;
    out5[1] = h->s.adjStats.solves;
    out5[2] = h->s.adjStats.recomputedSteps;
    out5[3] = h->s.adjStats.maxRelResidual;
    out5[4] = h->s.adjStats.forwardConverged;
  });
}

int cs_session_step(cs_solver* h, double dt, double* positions_out, int32_t* nan_free) {
  return guarded(h, [&] {
    const bool ok = h->s.session_step(dt, positions_out);
    if (nan_free) *nan_free = ok ? 1 : 0;
  });
}

int cs_session_restore_stable(cs_solver* h, int32_t* stable_step) {
  return guarded(h, [&] {
    const bool ok = h->s.session_restore();
    if (stable_step) *stable_step = ok ? h->s.stableStep : -1;
  });
}

int cs_session_reset(cs_solver* h) {
  return guarded(h, [&] { h->s.session_reset(); });
}

int cs_solver_info(cs_solver* h, int32_t* out, int32_t n) {
  return guarded(h, [&] {
    if (!out || n <= 0) throw std::invalid_argument("null output");
    const auto& S = h->s;
    const int32_t v[6] = {S.mxCluster, S.mxBlocks, S.pcgBlocks, S.mesh.D,
                          S.clRes[0] ? (int32_t)S.clSmem[0] : 0, S.clRes[1] ? (int32_t)S.clSmem[1] : 0};
    for (int i = 0; i < n; i++) out[i] = i < 6 ? v[i] : 0;
  });
}

int cs_profile_phases(cs_solver* h, double* out, int32_t n) {
  return guarded(h, [&] {
    if (!out || n <= 0) throw std::invalid_argument("null output");
    for (int i = 0; i < n; i++) out[i] = i < cs::PH_N ? h->s.phaseMs[i] : 0.0;
  });
}

int cs_build_grid(int32_t nx, int32_t ny, double w, double hh, float* pos, float* uv, uint32_t* idx) {
  if (nx <= 0 || ny <= 0 || !pos || !uv || !idx) return CS_E_ARG;
  std::vector<float> p, u;
  std::vector<uint32_t> ix;
  cs::grid_mesh(nx, ny, w, hh, p, u, ix);
  std::memcpy(pos, p.data(), p.size() * 4);
  std::memcpy(uv, u.data(), u.size() * 4);
  std::memcpy(idx, ix.data(), ix.size() * 4);
  return CS_OK;
}
int cs_preprocess(int32_t n, int32_t m, const float* pos, const float* uv, const uint32_t* idx, double density,
                  float* inv_dm, float* area, float* mass, int32_t* hg, int32_t* hinge, double* hinge_meta) {
  if (n <= 0 || m < 0 || !pos || !uv || !idx || !hg) return CS_E_ARG;
  try {
    std::vector<float> p(pos, pos + 3 * (size_t)n), u(uv, uv + 2 * (size_t)n);
    std::vector<uint32_t> ix(idx, idx + 3 * (size_t)m);
    for (uint32_t q : ix)
      if ((int)q >= n) return CS_E_ARG;
    cs::HostMesh me;
    cs::preprocess_mesh(p, u, ix, density, me);
    if (inv_dm) std::memcpy(inv_dm, me.inv.data(), me.inv.size() * 4);
    if (area) std::memcpy(area, me.area.data(), me.area.size() * 4);
    if (mass) std::memcpy(mass, me.mass.data(), me.mass.size() * 4);
    *hg = me.hg;
    if (hinge) std::memcpy(hinge, me.hinge.data(), me.hinge.size() * 4);
    if (hinge_meta) std::memcpy(hinge_meta, me.hmeta.data(), me.hmeta.size() * 8);
    return CS_OK;
  } catch (...) {
    return CS_E_ARG;
  }
}

}  // extern "C"
