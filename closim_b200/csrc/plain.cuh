// Device-side data of one solver instance and the kernel launchers of the
// FP64 path. All arrays live in HBM for the lifetime of the solver.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "elem.cuh"

namespace cs {

// Slots of the device scalar array (double).
enum ScalarSlot {
  S_GRADNORM = 0, S_MAXSTRAIN, S_ENERGY_TRIAL, S_GTDX, S_PCG_ITERS, S_PCG_RES, S_E_INERTIA,
  S_E_TRI, S_E_MERIT, S_E_HINGE, S_FALLBACK, S_MAXDX, S_VALID, S_MINDIST, S_MINTOI, S_CCDFAIL,
  S_BARRIER_E, S_FWORK, S_ENERGY_BASE, S_CH0 = 24, S_CH1, S_CH2, S_CH3, S_NSCALARS = 32
};

// Active contacts as seen by a kernel: the device count in a graph-captured
// step, else the host's.
struct Contact;
__device__ __forceinline__ int n_active(const Contact& c);

// One frozen contact (contact-assembly.ts:22-30): kind 0 VT, 1 EE, 2 floor.
// Ids < 0 other than -1 are static vertices -(i + 2).
struct Frozen {
  int kind, p, a, b, c, d;
  double w0, w1, w2, w3, nx, ny, nz;
};

// Frozen active set and its per-vertex gather structure, as seen by kernels.
struct Contact {
  double dHat, kappa, dMin, mu, eps, floorY;
  int hasFloor;
  int ns;                  // static vertices
  const float* spos;       // 3 ns
  int nActive;             // active records (VT/EE first, then floor)
  const int* nActiveD;     // graph-captured steps: the device's count (else null)
  const Frozen* active;
  double* dd;              // per-contact scalar (HVP coefficient, diag curvature, ...)
  double* cg;              // 4 per contact: barrier dE/dd, friction force args (-f)
  const uint32_t* cOff;    // n+1: vertex -> records (contact << 2 | slot), contact order
  const uint32_t* cRec;
  double* recScratch;      // 6 per record: per-record contact shares, summed per vertex in record order
  // Exact-Newton mode only (fric = 1): lagged friction as the potential
  // D = mu lambda sqrt(|P u|^2 + eps^2) of the relative slip u, with lambda and
  // the normal frozen for the Newton iteration. fh (8 per contact: mu lambda,
  // s = mu lambda / |.|, t = P u / |.|, n) feeds its Hessian s (P - t t^T) to the
  // HVP and D to the merit; fdd (3 per contact) holds the HVP's per-contact
  // friction share. The reference mode keeps friction out of both (as
  // contact-assembly.ts:371-428 does).
  int fric;
  const double* fh;
  double* fdd;
};

__device__ __forceinline__ int n_active(const Contact& c) { return c.nActiveD ? *c.nActiveD : c.nActive; }

// Everything a kernel of the FP64 path needs, passed by value.
struct Dev {
  int n, m, hg, npins;
  // mesh constants (Float32, as the reference stores them)
  const uint32_t* idx;     // 3m
  const float4* inv;       // m: Dm^-1 (a,b,c,d)
  const float* area;       // m
  const float* mass;       // n
  const int4* hinge;       // hg: v0,v1,v2,v3
  const double* hmeta;     // 3hg: restAngle, edgeLen, areaSum
  // CSR incidence, element-ordered (record = elem << 2 | corner)
  const uint32_t* memOff;  // n+1
  const uint32_t* memRec;  // 3m
  const uint32_t* hinOff;  // n+1
  const uint32_t* hinRec;  // 4hg (distinct corners)
  // pins
  const uint8_t* pinned;   // n
  const int* pinIds;       // npins
  const double* pinPos;    // 3 npins
  // state and work vectors (3n doubles each)
  double *x, *v, *x0, *yHat, *g, *diag, *dx, *r, *z, *p, *Ap, *xt, *cgrad, *cHp;
  double* elem;            // 18m element-local scratch
  double* helem;           // 12hg
  double* part;            // partial sums: NPART rows x maxBlocks
  int partStride;
  // Per-element terms of the reductions. The FP64 path adds them one by one in
  // index order (the reference's sequential loops), one thread per chain.
  double *T0, *T1, *T2, *T3; // max(3n, m + hg) each
  double* Tc;              // per-contact terms (contact capacity)
  double* scal;            // S_NSCALARS
  // material
  Mat<double> mat;
  double kb, h, invH2;
  double gravity[3];
  // one-level additive Schwarz (<= 8 vertices per domain)
  int D;
  const int* domStart;     // D+1
  const int* domVerts;     // n (members, ascending per domain)
  const int* v2tOff;       // n+1 vertex -> incident triangles (ascending)
  const int* v2t;          // 3m
  double* L;               // D x 576 (24x24 row-major), Cholesky or inverse diagonal
  uint8_t* domFlag;        // D
  double* dcoarse;         // 3D: coarse diagonal of the two-level Schwarz (precond 2)
  int precond;             // 0 Jacobi, 1 one-level Schwarz, 2 two-level Schwarz (mas2)
  int driftGuess;          // 1: Newton starts from x0 + h v (exact-Newton mode), 0: from yHat (newton.ts:41-50)
  int hasContact;
  Contact c;               // valid when hasContact
};

constexpr int kThreads = 256;
constexpr int NPART = 8;

// Launchers (plain.cu).
void launch_predict(const Dev& d, cudaStream_t s);
void launch_pins(const Dev& d, double* x, cudaStream_t s);
// g, gradNorm, maxStrain; analyticBend: the analytic hinge gradient instead of
// the reference's central differences (see launch_grad_terms).
void launch_grad(const Dev& d, cudaStream_t s, bool analyticBend = false);
// g and its squared terms, strain partials; analyticBend (mixed path) takes the
// analytic hinge gradient instead of the reference's central differences.
void launch_grad_terms(const Dev& d, cudaStream_t s, bool analyticBend = false);
void launch_energy_terms(const Dev& d, const double* x, cudaStream_t s);
void launch_energy(const Dev& d, const double* x, cudaStream_t s);  // S_ENERGY_TRIAL
void launch_diag_init(const Dev& d, double beta, cudaStream_t s);
void launch_schwarz_factor(const Dev& d, cudaStream_t s);
int launch_pcg(const Dev& d, int maxIters, double tol, int gridBlocks, cudaStream_t s);
void launch_trial(const Dev& d, double alpha, cudaStream_t s);   // xt = x + alpha dx, pins
void launch_velocity(const Dev& d, double damp, cudaStream_t s);
// SimulationSession.doStep hand-off (sim-session.ts:132-150) on the device:
// flag = any non-finite coordinate; stable <- x when finite.
void launch_session_check(const double* x, double* stable, int n3, int* flag, cudaStream_t s);
// Material-model evaluation over the mesh at x (no inertia, pins or contact):
// out2[0] = internalEnergyOnly, out2[1] = max strain (when grad is given);
// grad (3n, may be null) = evalInternal's gradient.
void launch_internal_eval(const Dev& d, const double* x, double* grad, double* out2, cudaStream_t s);
// evalMembraneHvp: analytic membrane Hessian-vector product at x along p.
void launch_membrane_hvp_analytic(const Dev& d, const double* x, const double* p, double* out, cudaStream_t s);
int pcg_grid_blocks(const Dev& d);
// FD membrane HVP over device arrays (T: 3n terms, h: 1 double, elem: 18m scratch).
void launch_membrane_hvp(const uint32_t* idx, const float4* inv, const float* area, const Mat<double>& mat, int n,
                         int m, const uint32_t* memOff, const uint32_t* memRec, const double* x, const double* p,
                         double* out, double* T, double* h, double* elem, cudaStream_t s);

}  // namespace cs
