// N-API addon over the C ABI of libclosim_cuda.so (include/closim_cuda.h).
//
// This is the binding the reference's Node host loads to reach the CUDA
// solver: host/ts/cuda-solver.ts calls every function exported here. Each
// export unwraps the solver handle (a JS external), reads typed arrays in
// place (no copies: the C ABI reads and writes host memory directly), calls
// one or two cs_* functions and turns a non-zero status into a JS Error
// carrying cs_last_error(). The messages of the reference's CpuSolver are kept:
// "CpuSolver not initialized" (cpu-solver.ts:16) and "non-finite gradient —
// blow up; reduce dt/stiffness" (newton.ts:129) come back verbatim.
//
// Exports (argument order as host/ts/cuda-solver.ts passes them):
//   create(precision: "fp64"|"mixed", device: number) -> handle
//   destroy(h)
//   initialize(h, mesh{count,triCount,indices,restPositions,invDm,areas,masses},
//              hinges: Int32Array(4hg), hingeMeta: Float64Array(3hg),
//              material, gravity: number[3], positions: Float64Array, velocities: Float64Array)
//   setContact(h, params|null, floorY: number|null, staticPos: Float32Array|null, staticIdx: Uint32Array|null)
//   setStepperOptions(h, {newtonIters, pcgMaxIters, lineSearchIters, gradTol, preconditioner})
//   setMaterial(h, material)
//   setPins(h, ids: Int32Array, pos: Float64Array)
//   setState(h, positions: Float64Array|null, velocities: Float64Array|null)
//   step(h, dt, positions: Float64Array, velocities: Float64Array)   // results written in place
//   lastStats(h) -> StepStats-shaped object
//   forward(h, dt, steps, checkpointEvery, positions: Float64Array)  // final positions written in place
//   backward(h, dLdxN: Float64Array, dLdTheta: Float64Array(4), dLdv0: Float64Array)
//   membraneHvp(h, x: Float64Array, p: Float64Array, out: Float64Array)
//   setNewtonMode(h, mode: "reference"|"exact", tol: number)
//   setGraphMode(h, on: boolean)
//   graphInfo(h) -> {graphSteps, repeats}
#include <node_api.h>

#include <cstdint>
#include <cstring>
#include <string>

#include "closim_cuda.h"

namespace {

// Throws a JS Error and returns false when `st` is not napi_ok.
bool ok(napi_env env, napi_status st, const char* what) {
  if (st == napi_ok) return true;
  bool pending = false;
  napi_is_exception_pending(env, &pending);
  if (!pending) napi_throw_error(env, nullptr, what);
  return false;
}

// Throws cs_last_error(h) (or a fixed text) for a non-zero cs_* status.
bool cs_ok(napi_env env, cs_solver* h, int rc) {
  if (rc == CS_OK) return true;
  std::string msg = h ? cs_last_error(h) : "closim_cuda: call failed";
  if (rc == CS_E_UNINIT) msg = "CpuSolver not initialized";
  napi_throw_error(env, nullptr, msg.c_str());
  return false;
}

bool is_nullish(napi_env env, napi_value v) {
  napi_valuetype t;
  if (napi_typeof(env, v, &t) != napi_ok) return true;
  return t == napi_null || t == napi_undefined;
}

// The JS handle is an external wrapping this box, so destroy() can release the
// solver early and the GC finalizer still runs exactly once.
struct Handle {
  cs_solver* h;
};

bool get_box(napi_env env, napi_value v, Handle** out) {
  void* p = nullptr;
  if (!ok(env, napi_get_value_external(env, v, &p), "expected a solver handle")) return false;
  if (!p) {
    napi_throw_type_error(env, nullptr, "expected a solver handle");
    return false;
  }
  *out = static_cast<Handle*>(p);
  return true;
}

bool get_handle(napi_env env, napi_value v, cs_solver** out) {
  Handle* b;
  if (!get_box(env, v, &b)) return false;
  if (!b->h) {
    napi_throw_error(env, nullptr, "solver handle was destroyed");
    return false;
  }
  *out = b->h;
  return true;
}

bool get_double(napi_env env, napi_value v, double* out) {
  return ok(env, napi_get_value_double(env, v, out), "expected a number");
}

bool get_int(napi_env env, napi_value v, int32_t* out) {
  return ok(env, napi_get_value_int32(env, v, out), "expected an integer");
}

bool prop(napi_env env, napi_value obj, const char* name, napi_value* out) {
  bool has = false;
  if (!ok(env, napi_has_named_property(env, obj, name, &has), "expected an object")) return false;
  if (!has) {
    napi_throw_type_error(env, nullptr, (std::string("missing property ") + name).c_str());
    return false;
  }
  return ok(env, napi_get_named_property(env, obj, name, out), name);
}

bool prop_double(napi_env env, napi_value obj, const char* name, double* out) {
  napi_value v;
  return prop(env, obj, name, &v) && get_double(env, v, out);
}

bool prop_int(napi_env env, napi_value obj, const char* name, int32_t* out) {
  napi_value v;
  return prop(env, obj, name, &v) && get_int(env, v, out);
}

// The element pointer and length of a typed array of the expected element type
// (the pointer already includes the view's byte offset).
template <class T>
bool typed(napi_env env, napi_value v, napi_typedarray_type want, T** data, size_t* len) {
  bool is = false;
  if (!ok(env, napi_is_typedarray(env, v, &is), "expected a typed array")) return false;
  if (!is) {
    napi_throw_type_error(env, nullptr, "expected a typed array");
    return false;
  }
  napi_typedarray_type t;
  void* p = nullptr;
  napi_value ab;
  size_t off = 0;
  if (!ok(env, napi_get_typedarray_info(env, v, &t, len, &p, &ab, &off), "typed array")) return false;
  if (t != want) {
    napi_throw_type_error(env, nullptr, "typed array of the wrong element type");
    return false;
  }
  *data = static_cast<T*>(p);
  return true;
}

template <class T>
bool typed_prop(napi_env env, napi_value obj, const char* name, napi_typedarray_type want, T** data, size_t* len) {
  napi_value v;
  return prop(env, obj, name, &v) && typed(env, v, want, data, len);
}

// ClothMaterial (src/physics/types.ts:1-12) -> cs_material.
bool material(napi_env env, napi_value o, cs_material* m) {
  return prop_double(env, o, "arealDensityKgM2", &m->areal_density) && prop_double(env, o, "thickness", &m->thickness) &&
         prop_double(env, o, "stretchWarp", &m->stretch_warp) && prop_double(env, o, "stretchWeft", &m->stretch_weft) &&
         prop_double(env, o, "stretchCoupling", &m->stretch_coupling) && prop_double(env, o, "shear", &m->shear) &&
         prop_double(env, o, "bendWarp", &m->bend_warp) && prop_double(env, o, "bendWeft", &m->bend_weft) &&
         prop_double(env, o, "damping", &m->damping);
}

template <size_t N>
bool args(napi_env env, napi_callback_info info, napi_value (&argv)[N], size_t need) {
  size_t argc = N;
  if (!ok(env, napi_get_cb_info(env, info, &argc, argv, nullptr, nullptr), "arguments")) return false;
  if (argc < need) {
    napi_throw_type_error(env, nullptr, "too few arguments");
    return false;
  }
  return true;
}

void finalize_handle(napi_env, void* data, void*) {
  Handle* b = static_cast<Handle*>(data);
  if (!b) return;
  if (b->h) cs_destroy(b->h);
  delete b;
}

napi_value Create(napi_env env, napi_callback_info info) {
  napi_value argv[2];
  if (!args(env, info, argv, 1)) return nullptr;
  char prec[16] = {0};
  size_t len = 0;
  if (!ok(env, napi_get_value_string_utf8(env, argv[0], prec, sizeof prec, &len), "precision must be a string"))
    return nullptr;
  int precision;
  if (std::strcmp(prec, "fp64") == 0) precision = CS_PRECISION_FP64;
  else if (std::strcmp(prec, "mixed") == 0) precision = CS_PRECISION_MIXED;
  else {
    napi_throw_range_error(env, nullptr, "precision must be \"fp64\" or \"mixed\"");
    return nullptr;
  }
  int32_t device = 0;
  if (!is_nullish(env, argv[1]) && !get_int(env, argv[1], &device)) return nullptr;
  cs_solver* h = cs_create(precision, device);
  if (!h) {
    napi_throw_error(env, nullptr, "cs_create failed: no CUDA device or unsupported precision");
    return nullptr;
  }
  Handle* b = new Handle{h};
  napi_value ext;
  if (!ok(env, napi_create_external(env, b, finalize_handle, nullptr, &ext), "handle")) {
    cs_destroy(h);
    delete b;
    return nullptr;
  }
  return ext;
}

// Releases the solver now (its device memory and stream); later calls with
// the handle throw, and the finalizer only frees the box.
napi_value Destroy(napi_env env, napi_callback_info info) {
  napi_value argv[1];
  if (!args(env, info, argv, 1)) return nullptr;
  Handle* b;
  if (!get_box(env, argv[0], &b)) return nullptr;
  if (b->h) cs_destroy(b->h);
  b->h = nullptr;
  return nullptr;
}

napi_value Initialize(napi_env env, napi_callback_info info) {
  napi_value argv[8];
  if (!args(env, info, argv, 8)) return nullptr;
  cs_solver* h;
  if (!get_handle(env, argv[0], &h)) return nullptr;
  napi_value me = argv[1];
  cs_mesh m{};
  size_t lidx = 0, lrest = 0, linv = 0, larea = 0, lmass = 0;
  uint32_t* idx;
  float *rest, *inv, *area, *mass;
  if (!prop_int(env, me, "count", &m.n) || !prop_int(env, me, "triCount", &m.m)) return nullptr;
  if (!typed_prop(env, me, "indices", napi_uint32_array, &idx, &lidx) ||
      !typed_prop(env, me, "restPositions", napi_float32_array, &rest, &lrest) ||
      !typed_prop(env, me, "invDm", napi_float32_array, &inv, &linv) ||
      !typed_prop(env, me, "areas", napi_float32_array, &area, &larea) ||
      !typed_prop(env, me, "masses", napi_float32_array, &mass, &lmass))
    return nullptr;
  if (lidx != 3 * (size_t)m.m || lrest != 3 * (size_t)m.n || linv != 4 * (size_t)m.m || larea != (size_t)m.m ||
      lmass != (size_t)m.n) {
    napi_throw_range_error(env, nullptr, "mesh array lengths do not match count / triCount");
    return nullptr;
  }
  int32_t* hinge;
  double* meta;
  size_t lh = 0, lm = 0;
  if (!typed(env, argv[2], napi_int32_array, &hinge, &lh) || !typed(env, argv[3], napi_float64_array, &meta, &lm))
    return nullptr;
  if (lh % 4 != 0 || lm != 3 * (lh / 4)) {
    napi_throw_range_error(env, nullptr, "hinges must hold 4 ids and hingeMeta 3 values per hinge");
    return nullptr;
  }
  m.hg = (int32_t)(lh / 4);
  m.indices = idx;
  m.rest = rest;
  m.inv_dm = inv;
  m.area = area;
  m.mass = mass;
  m.hinge = hinge;
  m.hinge_meta = meta;
  cs_material mat{};
  if (!material(env, argv[4], &mat)) return nullptr;
  double g[3];
  for (uint32_t k = 0; k < 3; k++) {
    napi_value e;
    if (!ok(env, napi_get_element(env, argv[5], k, &e), "gravity must be [gx, gy, gz]") || !get_double(env, e, &g[k]))
      return nullptr;
  }
  double *x, *v;
  size_t lx = 0, lv = 0;
  if (!typed(env, argv[6], napi_float64_array, &x, &lx) || !typed(env, argv[7], napi_float64_array, &v, &lv))
    return nullptr;
  if (lx != 3 * (size_t)m.n || lv != 3 * (size_t)m.n) {
    napi_throw_range_error(env, nullptr, "positions and velocities must hold 3n values");
    return nullptr;
  }
  cs_ok(env, h, cs_initialize(h, &m, &mat, g, x, v));
  return nullptr;
}

napi_value SetContact(napi_env env, napi_callback_info info) {
  napi_value argv[5];
  if (!args(env, info, argv, 5)) return nullptr;
  cs_solver* h;
  if (!get_handle(env, argv[0], &h)) return nullptr;
  if (is_nullish(env, argv[1])) {
    cs_ok(env, h, cs_set_contact(h, nullptr, 0, 0.0, nullptr, 0, nullptr, 0));
    return nullptr;
  }
  // ContactParams (src/collision/types.ts:27-47)
  cs_contact_params p{};
  if (!prop_double(env, argv[1], "dHatM", &p.dhat) || !prop_double(env, argv[1], "kappaJ", &p.kappa) ||
      !prop_double(env, argv[1], "dMinM", &p.dmin) || !prop_double(env, argv[1], "frictionMu", &p.mu) ||
      !prop_double(env, argv[1], "frictionEpsM", &p.eps))
    return nullptr;
  int floorOn = 0;
  double floorY = 0;
  if (!is_nullish(env, argv[2])) {
    if (!get_double(env, argv[2], &floorY)) return nullptr;
    floorOn = 1;
  }
  float* sp = nullptr;
  uint32_t* si = nullptr;
  size_t lsp = 0, lsi = 0;
  if (!is_nullish(env, argv[3]) && !typed(env, argv[3], napi_float32_array, &sp, &lsp)) return nullptr;
  if (!is_nullish(env, argv[4]) && !typed(env, argv[4], napi_uint32_array, &si, &lsi)) return nullptr;
  if (lsp % 3 != 0 || lsi % 3 != 0) {
    napi_throw_range_error(env, nullptr, "static mesh arrays must hold whole vertices / triangles");
    return nullptr;
  }
  cs_ok(env, h, cs_set_contact(h, &p, floorOn, floorY, sp, (int32_t)(lsp / 3), si, (int32_t)(lsi / 3)));
  return nullptr;
}

napi_value SetStepperOptions(napi_env env, napi_callback_info info) {
  napi_value argv[2];
  if (!args(env, info, argv, 2)) return nullptr;
  cs_solver* h;
  if (!get_handle(env, argv[0], &h)) return nullptr;
  cs_stepper_options o{};
  char pc[16] = {0};
  size_t len = 0;
  napi_value pv;
  if (!prop_int(env, argv[1], "newtonIters", &o.newton_iters) ||
      !prop_int(env, argv[1], "pcgMaxIters", &o.pcg_max_iters) ||
      !prop_int(env, argv[1], "lineSearchIters", &o.ls_iters) || !prop_double(env, argv[1], "gradTol", &o.grad_tol) ||
      !prop(env, argv[1], "preconditioner", &pv) ||
      !ok(env, napi_get_value_string_utf8(env, pv, pc, sizeof pc, &len), "preconditioner must be a string"))
    return nullptr;
  if (std::strcmp(pc, "jacobi") == 0) o.precond = CS_PRECOND_JACOBI;
  else if (std::strcmp(pc, "schwarz") == 0) o.precond = CS_PRECOND_SCHWARZ;
  else if (std::strcmp(pc, "mas2") == 0) o.precond = CS_PRECOND_MAS2;
  else {
    napi_throw_range_error(env, nullptr, "preconditioner must be \"jacobi\", \"schwarz\" or \"mas2\"");
    return nullptr;
  }
  cs_ok(env, h, cs_set_stepper_options(h, &o));
  return nullptr;
}

napi_value SetMaterial(napi_env env, napi_callback_info info) {
  napi_value argv[2];
  if (!args(env, info, argv, 2)) return nullptr;
  cs_solver* h;
  cs_material m{};
  if (!get_handle(env, argv[0], &h) || !material(env, argv[1], &m)) return nullptr;
  cs_ok(env, h, cs_set_material(h, &m));
  return nullptr;
}

napi_value SetPins(napi_env env, napi_callback_info info) {
  napi_value argv[3];
  if (!args(env, info, argv, 3)) return nullptr;
  cs_solver* h;
  if (!get_handle(env, argv[0], &h)) return nullptr;
  int32_t* ids;
  double* pos;
  size_t li = 0, lp = 0;
  if (!typed(env, argv[1], napi_int32_array, &ids, &li) || !typed(env, argv[2], napi_float64_array, &pos, &lp))
    return nullptr;
  if (lp != 3 * li) {
    napi_throw_range_error(env, nullptr, "pin positions must hold 3 values per id");
    return nullptr;
  }
  cs_ok(env, h, cs_set_pins(h, (int32_t)li, li ? ids : nullptr, li ? pos : nullptr));
  return nullptr;
}

napi_value SetState(napi_env env, napi_callback_info info) {
  napi_value argv[3];
  if (!args(env, info, argv, 3)) return nullptr;
  cs_solver* h;
  if (!get_handle(env, argv[0], &h)) return nullptr;
  double *x = nullptr, *v = nullptr;
  size_t lx = 0, lv = 0;
  if (!is_nullish(env, argv[1]) && !typed(env, argv[1], napi_float64_array, &x, &lx)) return nullptr;
  if (!is_nullish(env, argv[2]) && !typed(env, argv[2], napi_float64_array, &v, &lv)) return nullptr;
  cs_ok(env, h, cs_set_state(h, x, v));
  return nullptr;
}

// ClothSolver.step(dt): one step, then the new positions and velocities are
// written into the scene's own Float64Arrays (cpu-solver.ts:15-18 leaves them
// in scene.positions / scene.velocities).
napi_value Step(napi_env env, napi_callback_info info) {
  napi_value argv[4];
  if (!args(env, info, argv, 4)) return nullptr;
  cs_solver* h;
  double dt;
  if (!get_handle(env, argv[0], &h) || !get_double(env, argv[1], &dt)) return nullptr;
  double *x, *v;
  size_t lx = 0, lv = 0;
  if (!typed(env, argv[2], napi_float64_array, &x, &lx) || !typed(env, argv[3], napi_float64_array, &v, &lv))
    return nullptr;
  int rc = cs_step(h, dt);
  if (rc == CS_OK) rc = cs_get_positions(h, x);
  if (rc == CS_OK) rc = cs_get_velocities(h, v);
  cs_ok(env, h, rc);
  return nullptr;
}

bool set_num(napi_env env, napi_value o, const char* k, double val) {
  napi_value v;
  return ok(env, napi_create_double(env, val, &v), k) && ok(env, napi_set_named_property(env, o, k, v), k);
}

// Newton mode (no counterpart in the reference): "reference", the default, or
// "exact" with its relative PCG tolerance (cs_set_newton_mode).
napi_value SetNewtonMode(napi_env env, napi_callback_info info) {
  napi_value argv[3];
  if (!args(env, info, argv, 3)) return nullptr;
  cs_solver* h;
  double tol;
  if (!get_handle(env, argv[0], &h) || !get_double(env, argv[2], &tol)) return nullptr;
  char mode[16] = {0};
  size_t len = 0;
  if (!ok(env, napi_get_value_string_utf8(env, argv[1], mode, sizeof mode, &len), "mode must be a string"))
    return nullptr;
  int32_t m;
  if (std::strcmp(mode, "reference") == 0) m = 0;
  else if (std::strcmp(mode, "exact") == 0) m = 1;
  else {
    napi_throw_range_error(env, nullptr, "mode must be \"reference\" or \"exact\"");
    return nullptr;
  }
  cs_ok(env, h, cs_set_newton_mode(h, m, tol));
  return nullptr;
}

// Graph-captured steps on or off (cs_set_graph_mode).
napi_value SetGraphMode(napi_env env, napi_callback_info info) {
  napi_value argv[2];
  if (!args(env, info, argv, 2)) return nullptr;
  cs_solver* h;
  bool on = true;
  if (!get_handle(env, argv[0], &h) || !ok(env, napi_get_value_bool(env, argv[1], &on), "expected a boolean"))
    return nullptr;
  cs_ok(env, h, cs_set_graph_mode(h, on ? 1 : 0));
  return nullptr;
}

// Steps taken as graph replays and steps repeated host-driven (cs_graph_info).
napi_value GraphInfo(napi_env env, napi_callback_info info) {
  napi_value argv[1];
  if (!args(env, info, argv, 1)) return nullptr;
  cs_solver* h;
  if (!get_handle(env, argv[0], &h)) return nullptr;
  int64_t o[2] = {0, 0};
  if (!cs_ok(env, h, cs_graph_info(h, o))) return nullptr;
  napi_value r;
  if (!ok(env, napi_create_object(env, &r), "graphInfo") || !set_num(env, r, "graphSteps", (double)o[0]) ||
      !set_num(env, r, "repeats", (double)o[1]))
    return nullptr;
  return r;
}

// StepStats (src/solver/newton.ts:10-18) with ContactDiagnostics
// (src/collision/types.ts:49-62) under `contact` (null without contact).
napi_value LastStats(napi_env env, napi_callback_info info) {
  napi_value argv[1];
  if (!args(env, info, argv, 1)) return nullptr;
  cs_solver* h;
  if (!get_handle(env, argv[0], &h)) return nullptr;
  cs_step_stats s{};
  if (!cs_ok(env, h, cs_last_stats(h, &s))) return nullptr;
  napi_value o, conv, con;
  if (!ok(env, napi_create_object(env, &o), "stats")) return nullptr;
  if (!set_num(env, o, "newtonIters", s.newton_iters) || !set_num(env, o, "pcgIters", s.pcg_iters) ||
      !set_num(env, o, "gradNorm", s.grad_norm) || !set_num(env, o, "energy", s.energy) ||
      !set_num(env, o, "maxStrain", s.max_strain) || !set_num(env, o, "newtonItersUsed", s.newton_iters_used) ||
      !set_num(env, o, "armijoTrials", s.armijo_trials))
    return nullptr;
  if (!ok(env, napi_get_boolean(env, s.converged != 0, &conv), "stats") ||
      !ok(env, napi_set_named_property(env, o, "converged", conv), "stats"))
    return nullptr;
  if (s.has_contact) {
    if (!ok(env, napi_create_object(env, &con), "stats")) return nullptr;
    if (!set_num(env, con, "candidatePairs", s.candidate_pairs) || !set_num(env, con, "activePairs", s.active_pairs) ||
        !set_num(env, con, "vtPairs", s.vt_pairs) || !set_num(env, con, "eePairs", s.ee_pairs) ||
        !set_num(env, con, "floorPairs", s.floor_pairs) || !set_num(env, con, "minDistance", s.min_distance) ||
        !set_num(env, con, "minTOI", s.min_toi) || !set_num(env, con, "barrierEnergy", s.barrier_energy) ||
        !set_num(env, con, "frictionWork", s.friction_work) ||
        !set_num(env, con, "rejectedLineSearchSteps", s.rejected_line_search_steps) ||
        !set_num(env, con, "ccdFailures", s.ccd_failures))
      return nullptr;
  } else if (!ok(env, napi_get_null(env, &con), "stats")) {
    return nullptr;
  }
  if (!ok(env, napi_set_named_property(env, o, "contact", con), "stats")) return nullptr;
  return o;
}

// Differentiable rollout (no counterpart in the reference): forward keeps
// checkpoints on the device and writes the final positions into `positions`.
napi_value Forward(napi_env env, napi_callback_info info) {
  napi_value argv[5];
  if (!args(env, info, argv, 5)) return nullptr;
  cs_solver* h;
  double dt;
  int32_t steps, every;
  if (!get_handle(env, argv[0], &h) || !get_double(env, argv[1], &dt) || !get_int(env, argv[2], &steps) ||
      !get_int(env, argv[3], &every))
    return nullptr;
  double* x;
  size_t lx = 0;
  if (!typed(env, argv[4], napi_float64_array, &x, &lx)) return nullptr;
  int rc = cs_forward(h, dt, steps, every);
  if (rc == CS_OK) rc = cs_get_positions(h, x);
  cs_ok(env, h, rc);
  return nullptr;
}

napi_value Backward(napi_env env, napi_callback_info info) {
  napi_value argv[4];
  if (!args(env, info, argv, 4)) return nullptr;
  cs_solver* h;
  if (!get_handle(env, argv[0], &h)) return nullptr;
  double *g, *th, *dv = nullptr;
  size_t lg = 0, lt = 0, ld = 0;
  if (!typed(env, argv[1], napi_float64_array, &g, &lg) || !typed(env, argv[2], napi_float64_array, &th, &lt))
    return nullptr;
  if (!is_nullish(env, argv[3]) && !typed(env, argv[3], napi_float64_array, &dv, &ld)) return nullptr;
  if (lt != 4 || (dv && ld != lg)) {
    napi_throw_range_error(env, nullptr, "dLdTheta holds 4 values and dLdv0 as many as dLdxN");
    return nullptr;
  }
  cs_ok(env, h, cs_backward(h, g, th, dv));
  return nullptr;
}

napi_value MembraneHvp(napi_env env, napi_callback_info info) {
  napi_value argv[4];
  if (!args(env, info, argv, 4)) return nullptr;
  cs_solver* h;
  if (!get_handle(env, argv[0], &h)) return nullptr;
  double *x, *p, *out;
  size_t lx = 0, lp = 0, lo = 0;
  if (!typed(env, argv[1], napi_float64_array, &x, &lx) || !typed(env, argv[2], napi_float64_array, &p, &lp) ||
      !typed(env, argv[3], napi_float64_array, &out, &lo))
    return nullptr;
  if (lx != lp || lx != lo) {
    napi_throw_range_error(env, nullptr, "x, p and out must have the same length");
    return nullptr;
  }
  cs_ok(env, h, cs_membrane_hvp(h, x, p, out));
  return nullptr;
}

}  // namespace

NAPI_MODULE_INIT() {
  const napi_property_descriptor fns[] = {
      {"create", nullptr, Create, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"destroy", nullptr, Destroy, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"initialize", nullptr, Initialize, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setContact", nullptr, SetContact, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setStepperOptions", nullptr, SetStepperOptions, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setMaterial", nullptr, SetMaterial, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setPins", nullptr, SetPins, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setState", nullptr, SetState, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"step", nullptr, Step, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"lastStats", nullptr, LastStats, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"forward", nullptr, Forward, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"backward", nullptr, Backward, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"membraneHvp", nullptr, MembraneHvp, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setNewtonMode", nullptr, SetNewtonMode, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"setGraphMode", nullptr, SetGraphMode, nullptr, nullptr, nullptr, napi_default, nullptr},
      {"graphInfo", nullptr, GraphInfo, nullptr, nullptr, nullptr, napi_default, nullptr},
  };
  if (napi_define_properties(env, exports, sizeof fns / sizeof fns[0], fns) != napi_ok) return nullptr;
  return exports;
}
