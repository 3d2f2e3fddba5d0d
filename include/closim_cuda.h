/*
 * closim_cuda.h - C ABI of the B200 CUDA cloth solver (libclosim_cuda.so).
 *
 * Drop-in replacement for the reference's ClothSolver backend
 * (mohdabraralikhan/closim src/backend/solver.ts:5-13, implemented on the CPU
 * by src/backend/cpu-solver.ts). A host binding (N-API addon, ctypes, ...)
 * wraps one cs_solver per ClothScene. Plain pointers and sizes only.
 *
 * Frame: y-up, as the reference (gravity defaults to {0,-9.81,0}, the floor is
 * a y = const plane).
 *
 * Errors: every call returns CS_OK (0) or a CS_E_* code; cs_last_error()
 * returns a message. A handle is synchronous and single-threaded; separate
 * handles are independent.
 */
#ifndef CLOSIM_CUDA_H
#define CLOSIM_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  CS_OK = 0,
  CS_E_UNINIT = 1,     /* "CpuSolver not initialized" (cpu-solver.ts:16,21,26,41,46) */
  CS_E_NONFINITE = 2,  /* "non-finite gradient - blow up; reduce dt/stiffness" (newton.ts:129) */
  CS_E_CAPACITY = 3,   /* a device buffer was too small; the call was not applied */
  CS_E_CUDA = 4,       /* CUDA runtime error */
  CS_E_ARG = 5         /* invalid argument */
};

enum { CS_PRECISION_FP64 = 0, CS_PRECISION_MIXED = 1 };
/* Preconditioners: Jacobi; one-level additive Schwarz on <= 8-vertex domains
 * (src/solver/schwarz.ts); two-level additive Schwarz with the damped-Jacobi
 * coarse correction over the same domains (src/solver/mas.ts, omega = 0.5). */
enum { CS_PRECOND_JACOBI = 0, CS_PRECOND_SCHWARZ = 1, CS_PRECOND_MAS2 = 2 };

/* ClothMaterial (src/physics/types.ts:1-12). */
typedef struct cs_material {
  double areal_density;   /* kg/m^2, lumped mass only */
  double thickness;       /* m, scales the elastic energy */
  double stretch_warp;    /* C00 */
  double stretch_weft;    /* C11 */
  double stretch_coupling;/* C01 */
  double shear;           /* G */
  double bend_warp;
  double bend_weft;
  double damping;         /* 0..0.1 velocity damping */
} cs_material;

/* ContactParams (src/collision/types.ts:27-47). */
typedef struct cs_contact_params {
  double dhat;            /* barrier activation distance, m */
  double kappa;           /* barrier energy scale, J */
  double dmin;            /* minimum admissible distance, m */
  double mu;              /* Coulomb coefficient */
  double eps;             /* friction regularization, m */
} cs_contact_params;

/* Preprocessed ClothMeshData (src/mesh/mesh.ts:3-14). */
typedef struct cs_mesh {
  int32_t n, m, hg;           /* vertices, triangles, hinges */
  const uint32_t* indices;    /* 3m */
  const float* rest;          /* 3n rest positions (Schwarz domain seeding) */
  const float* inv_dm;        /* 4m: a,b,c,d */
  const float* area;          /* m */
  const float* mass;          /* n lumped */
  const int32_t* hinge;       /* 4hg: v0,v1 (shared edge), v2, v3 */
  const double* hinge_meta;   /* 3hg: restAngle, edgeLen, areaSum */
} cs_mesh;

/* StepperOptions (src/solver/newton.ts:20-25) + preconditioner choice. */
typedef struct cs_stepper_options {
  int32_t newton_iters;   /* default 10 */
  int32_t pcg_max_iters;  /* default 60 */
  int32_t ls_iters;       /* default 10 */
  int32_t precond;        /* CS_PRECOND_* (Schwarz domains: target 8, min 1) */
  double grad_tol;        /* default 1e-5 */
} cs_stepper_options;

/* StepStats (src/solver/newton.ts:10-18) + ContactDiagnostics
 * (src/collision/types.ts:49-62) + counters of this implementation. */
typedef struct cs_step_stats {
  int32_t newton_iters;       /* the configured budget, as the reference reports */
  int32_t pcg_iters;          /* summed over Newton iterations */
  double grad_norm, energy, max_strain;
  int32_t converged;
  int32_t has_contact;
  double candidate_pairs, active_pairs, vt_pairs, ee_pairs, floor_pairs;
  double min_distance, min_toi, barrier_energy, friction_work;
  double rejected_line_search_steps, ccd_failures;
  int32_t newton_iters_used;  /* iterations actually run */
  int32_t armijo_trials;      /* line-search trials run */
} cs_step_stats;

typedef struct cs_solver cs_solver;

/* Creates a solver on CUDA device `device` (precision: CS_PRECISION_*). */
cs_solver* cs_create(int precision, int device);
void cs_destroy(cs_solver* s);
const char* cs_last_error(cs_solver* s);

/* ClothSolver.initialize(scene) (solver.ts:6): uploads mesh, material,
 * gravity, positions x (3n f64) and velocities v (3n f64; NULL = zero). */
int cs_initialize(cs_solver* s, const cs_mesh* mesh, const cs_material* mat,
                  const double gravity[3], const double* x, const double* v);
/* scene.contact = new ContactSystem(params, indices) + setFloor + setStaticMesh
 * (contact-assembly.ts:63-73). params NULL disables contact. */
int cs_set_contact(cs_solver* s, const cs_contact_params* params, int floor_on, double floor_y,
                   const float* static_pos, int32_t ns, const uint32_t* static_idx, int32_t ms);
int cs_set_stepper_options(cs_solver* s, const cs_stepper_options* opts);
/* ClothSolver.setMaterial (solver.ts:8). */
int cs_set_material(cs_solver* s, const cs_material* mat);
/* Replaces the pin map (scene.pinned, solver.ts:9-10): k ids and 3k positions. */
int cs_set_pins(cs_solver* s, int32_t k, const int32_t* ids, const double* pos);
/* ClothSolver.step(dt) (solver.ts:7; cpu-solver.ts:15-18). */
int cs_step(cs_solver* s, double dt);
/* getPositions / getVelocities (solver.ts:11-12): copy 3n f64 out. */
int cs_get_positions(cs_solver* s, double* out);
int cs_get_velocities(cs_solver* s, double* out);
/* Overwrites positions and/or velocities (either may be NULL). */
int cs_set_state(cs_solver* s, const double* x, const double* v);
/* CpuSolver.lastStats (cpu-solver.ts:6). */
int cs_last_stats(cs_solver* s, cs_step_stats* out);

/* membraneHvp(x, p) (src/physics/fem.ts:108-130): the central-difference
 * membrane Hessian-vector product the FP64 path's PCG applies, h = 1e-8 (1 + |p|),
 * on the initialized mesh and current material. Host arrays of 3n doubles. */
int cs_membrane_hvp(cs_solver* s, const double* x, const double* p, double* out);

/* A collider that moves between steps: replaces the static mesh's ns vertex
 * positions (f32, the same triangles as cs_set_contact gave), as
 * ContactSystem.setStaticMesh with a collider's sampled pose does
 * (src/collision/avatar-collider.ts:205-237, attachCollisionObject). Within a
 * step the static mesh stays where it was put, as in the reference. */
int cs_update_static_positions(cs_solver* s, const float* static_pos, int32_t ns);

/* ContactSystem.active (contact-assembly.ts:50): the frozen active set of the
 * last update (after cs_step: the one its restitution pass used), in
 * active-list order. *count receives its size; when ids6 (6 per record: kind
 * 0 VT / 1 EE / 2 floor, p, a, b, c, d; static ids are -(i + 2)) and w7 (7 per
 * record: w0..w3, nx, ny, nz) are given and cap >= *count they are filled,
 * else CS_E_CAPACITY. */
int cs_contact_active(cs_solver* s, int32_t cap, int32_t* count, int32_t* ids6, double* w7);

/* Graph-captured steps (no counterpart in the reference): with enable = 1 (the
 * default) a step of the mixed path whose PCG fits one thread-block cluster is
 * a replay of a CUDA graph captured once per configuration, with the Newton,
 * Armijo and trust-region decisions taken on the device (conditional graph
 * nodes) and one host synchronization per step; its results equal the
 * host-driven step's. A step whose buffers overflow is restored and repeated
 * host-driven with grown buffers. enable = 0 forces the host-driven step.
 * cs_graph_info: out2[0] steps taken as graph replays, out2[1] repeats. */
int cs_set_graph_mode(cs_solver* s, int32_t enable);
int cs_graph_info(cs_solver* s, int64_t* out2);

/* ---- material model (src/physics/material-model.ts:232-296) ----
 * ClothMaterialModel.energy / gradient / hessianVector of the orthotropic StVK
 * model on the GPU, for the handle's mesh and current material (cs_set_material),
 * at positions x (host, 3n doubles): no inertia, pins or contact.
 * cs_internal_energy: internalEnergyOnly (src/physics/fem.ts:56-75).
 * cs_internal_gradient: evalInternal (fem.ts:15-54): energy, gradient (3n),
 *   max |Green strain|; energy and max_strain may be NULL.
 * cs_membrane_hvp_analytic: evalMembraneHvp (src/physics/membrane-hvp.ts:80-108),
 *   the analytic membrane Hessian-vector product along p (bending excluded). */
int cs_internal_energy(cs_solver* s, const double* x, double* energy);
int cs_internal_gradient(cs_solver* s, const double* x, double* energy, double* grad, double* max_strain);
int cs_membrane_hvp_analytic(cs_solver* s, const double* x, const double* p, double* out);

/* ---- device-resident helpers (no reference counterpart needed by a drop-in) ---- */
/* Runs `nsteps` steps back to back without copying state to the host. */
int cs_step_n(cs_solver* s, double dt, int32_t nsteps);
/* Synchronizes the solver's stream; returns CS_E_CUDA on a pending error. */
int cs_sync(cs_solver* s);
/* Number of this library's kernel launches since creation. */
int64_t cs_kernel_launches(cs_solver* s);
/* The solver's CUDA stream (cudaStream_t), for recording events around calls. */
void* cs_stream(cs_solver* s);
/* Per-launch timing of the linear-solve kernel (the dominant kernel): when
 * enabled, each launch is bracketed by CUDA events on the solver's stream.
 * cs_profile_read fills out[5]: total ms, launches, algorithmic bytes, PCG
 * iterations, and the flush-free mean ms per launch. */
int cs_profile(cs_solver* s, int enable);
int cs_profile_read(cs_solver* s, double* out5);
/* Wall-time breakdown of the step (diagnostic, no counterpart in the
 * reference): after cs_profile(s, 2) the stream is synchronized at every
 * phase boundary, which slows the step. Fills out[0..n) with milliseconds
 * accumulated per phase since cs_profile: other, broadphase, active set,
 * gradient, preconditioner, PCG, trial check, trial energy, commit. */
int cs_profile_phases(cs_solver* s, double* out, int32_t n);
/* Launch shapes chosen at cs_initialize (diagnostic): out[0] CTAs of the
 * one-cluster mixed PCG (0 = the grid-wide kernel is used), out[1] CTAs of the
 * grid-wide mixed PCG, out[2] CTAs of the FP64 PCG, out[3] Schwarz domains,
 * out[4] / out[5] dynamic shared memory per CTA (bytes) of the one-cluster
 * PCG's resident element lists without / with the Gauss-Newton bending term
 * (0 = they do not fit and the kernel gathers from global memory). */
int cs_solver_info(cs_solver* s, int32_t* out, int32_t n);

/* ---- SimulationSession.doStep hand-off (src/view/sim-session.ts:132-150) ----
 * cs_session_step: one step, then on the device the NaN scan of the new
 * positions and, when they are finite, a device copy into the stable
 * snapshot; the positions land in positions_out (3n doubles; pinned host
 * memory avoids a staging copy; may be NULL) and *nan_free tells whether they
 * are finite -- one stream synchronization per step, where the reference
 * scans and copies on the host. cs_session_reset makes the current positions
 * the stable snapshot (SimulationSession.attach); cs_session_restore_stable
 * puts the snapshot back with zero velocities (restoreStable) and reports the
 * session step it was taken at (-1 when there is none). */
int cs_session_step(cs_solver* s, double dt, double* positions_out, int32_t* nan_free);
int cs_session_reset(cs_solver* s);
int cs_session_restore_stable(cs_solver* s, int32_t* stable_step);

/* ---- differentiable rollout (no counterpart in the reference) ----
 * cs_forward runs `steps` implicit steps of size dt from the current state
 * (pins held fixed) and keeps (x, v) at every checkpoint_every-th step start.
 * cs_backward takes dL/dx_N (host, 3n doubles) for a loss on the final
 * positions and returns dL/d(C00, C11, G, k_bend) in dL_dtheta[4] (k_bend sets
 * bendWarp = bendWeft) and dL/dv_0 in dL_dv0 (3n, may be NULL), through the
 * implicit-function theorem on every step (one FP64 solve of H mu = lambda per
 * step, H the Newton Hessian at the step's end state with membrane, bending
 * and frozen barrier terms; friction and the restitution filter are held
 * constant). Each checkpoint segment is recomputed from its checkpoint; the
 * state after cs_forward is restored on return. The gradient is that of the
 * converged step map: give cs_set_stepper_options a budget under which every
 * step converges. */
int cs_forward(cs_solver* s, double dt, int32_t steps, int32_t checkpoint_every);
int cs_backward(cs_solver* s, const double* dL_dxN, double* dL_dtheta, double* dL_dv0);
/* Newton linear solve (no counterpart in the reference). mode 0 (default) is
 * the reference's: matrix-free FD membrane HVP, PCG to relative 1e-3, Newton
 * from the inertial target x0 + h v + h^2 g. mode 1 (exact-Newton) solves with
 * the full Hessian (analytic membrane HVP with compressed principal stresses
 * clamped to zero, exact bending HVP (Gauss-Newton on the mixed path), frozen
 * contact, lagged friction as a frozen potential) to the relative PCG
 * tolerance tol, takes the analytic hinge gradient, and starts Newton from
 * x0 + h v; it keeps the reference's descent safeguard, trust region and
 * Armijo search, with the Armijo base energy re-evaluated at every Newton
 * iterate (its active set and friction potential) and a CCD-valid full step
 * taken once the gradient norm is below 1e-7, where the energy decrease falls
 * below the rounding of the energy sum. The converged step is the same,
 * reached in far fewer iterations, as the converged comparisons and the
 * adjoint's implicit-function theorem need. The exception is friction between
 * two cloth sides (VT, EE): the reference's friction term there is not the
 * gradient of any potential, and the line search can stall as in mode 0. cs_set_stepper_options' budgets apply to both. */
int cs_set_newton_mode(cs_solver* s, int32_t mode, double tol);
/* Adjoint PCG budget (default 2000 iterations, relative residual 1e-10). */
int cs_set_adjoint_options(cs_solver* s, int32_t max_iters, double tol);
/* out[5]: adjoint PCG iterations, solves, recomputed steps and largest final
 * relative residual of the last cs_backward; steps of the last cs_forward
 * that converged (reached gradTol). */
int cs_adjoint_stats(cs_solver* s, double* out5);

/* ---- allocation-free membrane HVP (no counterpart in the reference) ----
 * For callers that may not call cudaMalloc while stepping: a frame recorded into
 * a CUDA graph (no allocation during stream capture), a real-time loop that
 * cannot absorb cudaMalloc's device-wide synchronization, or a plugin whose
 * device memory belongs to another runtime. Computes exactly what
 * cs_membrane_hvp computes, without a solver handle: every argument is a
 * device pointer the caller owns (inv_dm 16-byte aligned), `stream` is a
 * cudaStream_t (NULL = the legacy default stream), and the kernels' scratch
 * (18 doubles per triangle plus 3 per vertex, about 11 MB) is a fixed array
 * inside this library that every GPU loading the library holds until exit.
 * inc_offsets (n+1) and inc_records (3m) are the membrane incidence as a CSR
 * over vertices: the records of vertex v are inc_records[inc_offsets[v] ..
 * inc_offsets[v+1]), each the value triangle * 4 + corner, listed in ascending
 * triangle order. Limits: n <= CS_STATIC_HVP_MAX_VERTICES and
 * m <= CS_STATIC_HVP_MAX_TRIANGLES, else CS_E_CAPACITY. The first call on a
 * device resolves the array's address (cudaGetSymbolAddress): make that call
 * before any stream capture. The address is cached per device index for the
 * life of the process: after cudaDeviceReset the cache is stale, so do not call
 * this entry point again in that process. All calls share the array: calls that overlap on
 * the GPU race, so serialize them. Returns CS_OK, CS_E_ARG, CS_E_CAPACITY or
 * CS_E_CUDA. */
#define CS_STATIC_HVP_MAX_VERTICES 65536
#define CS_STATIC_HVP_MAX_TRIANGLES 65536
int cs_membrane_hvp_static(int32_t n, int32_t m, const uint32_t* indices, const float* inv_dm,
                           const float* area, const uint32_t* inc_offsets, const uint32_t* inc_records,
                           const cs_material* mat, const double* x, const double* p, double* out,
                           void* stream);

/* ---- mesh preprocessing (src/mesh/mesh.ts:17-126), host side ---- */
/* buildGrid(nx, ny, w, h): pos 3n f32, uv 2n f32, idx 6*nx*ny u32. */
int cs_build_grid(int32_t nx, int32_t ny, double w, double h, float* pos, float* uv, uint32_t* idx);
/* preprocess(positions, uv, indices, density): inv_dm 4m, area m, mass n; the
 * hinge count is returned through *hg and hinge / hinge_meta receive 4hg / 3hg
 * values. Any output pointer may be NULL (a first call with NULLs sizes hg). */
int cs_preprocess(int32_t n, int32_t m, const float* pos, const float* uv, const uint32_t* idx,
                  double density, float* inv_dm, float* area, float* mass, int32_t* hg,
                  int32_t* hinge, double* hinge_meta);

#ifdef __cplusplus
}
#endif
#endif /* CLOSIM_CUDA_H */
