// ContactSystem on the device (reference src/collision/contact-assembly.ts),
// FP64 path (compiled with -fmad=false).
//
// Per Newton iteration the frozen active set is rebuilt from the broadphase
// candidates (sorted by (kind, p, a, b, c, d), contact-assembly.ts:118) and the
// floor vertices; per-contact kernels evaluate the barrier, lagged friction,
// frozen HVP and diagonal terms, and per-vertex kernels gather them through a
// vertex -> (contact, slot) CSR built by a stable sort, so every vertex adds its
// contact terms in active-list order as the reference's scatter does. Chained
// sums (barrier energy, friction work, merit energy) are evaluated left to
// right by one thread.
#include <climits>

#include "broadphase.cuh"
#include "contact.cuh"
#include "contact_host.hpp"
#include "graph_ctx.hpp"
#include "solver.hpp"

namespace cs {

constexpr int kCT = 256;
static inline int cnb(long n) { return (int)((n + kCT - 1) / kCT); }

struct CView {  // kernel view of the contact host buffers
  Contact c;
  int nCand, nFloor, n;
  const double* x0;  // xStep
  // Candidate pairs of the current query (counts in ccnt): self triangle
  // pairs and (cloth triangle, static triangle) pairs, and the index buffers.
  const int2* selfPairs;
  const int2* staticPairs;
  const uint32_t* idx;
  const uint32_t* sidx;
  int ns, idBits;              // static vertex count, bits per id in the order key
  unsigned long long* badKey;  // [hi, lo] smallest (key, status) of a failing CCD candidate
  // Minima as order-preserving 64-bit images of doubles (ord_of):
  // [0] trial distance, [1] trial TOI, [2] active-set distance.
  unsigned long long* omin;
  int* badList;                // indices of failing trial candidates (first kBadCap)
  // A trial enqueued before its Newton iteration's gradient norm was read
  // records nothing unless *gradGate >= gradTol (null: always records).
  const double* gradGate;
  double gradTol;
  const uint32_t* ccnt;        // [self pairs, static pairs] of the current query (device)
  uint32_t* cflag;
  uint32_t* fflag;
  Frozen* active;
  double* dd;
  double* cg;
  double* tc;
  double* tf;
  double* lagFloor;
  uint8_t* lagFloorOk;
  const Key<6>* lagKeys;
  const double4* lagVals;
  int lagCount;
  int* cint;
  DevDiag* diag;
  // Graph-captured steps: the frozen-set and lag-table counts on the device
  // (ACnt); every count below is then read from here, and launches are sized
  // for capacities. Null on the host-driven path.
  int* acnt;
};

__device__ __forceinline__ int v_ncand(const CView& v) { return v.acnt ? v.acnt[AC_NCAND] : v.nCand; }
__device__ __forceinline__ int v_lag(const CView& v) { return v.acnt ? v.acnt[AC_LAG] : v.lagCount; }
// A contact count passed by the host, or (negative) read from the device.
__device__ __forceinline__ int v_na(const CView& v, int na) { return na >= 0 ? na : v.acnt[AC_NA]; }

__device__ __forceinline__ double seq_sum(const double* t, int n) {
  double s = 0.0;
  for (int i = 0; i < n; i++) s = s + t[i];
  return s;
}

// Order-preserving map of a non-NaN double onto an unsigned 64-bit integer
// (negative values bit-flipped, non-negative ones with the sign bit set), so
// that an atomicMin on the image is a minimum of the doubles.
__device__ __forceinline__ unsigned long long ord_of(double d) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(d);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dbl_of(unsigned long long o) {
  return __longlong_as_double((long long)((o >> 63) ? (o & 0x7fffffffffffffffull) : ~o));
}
constexpr unsigned long long kOrdInf = 0xfff0000000000000ull;  // ord_of(+inf)

// Block minima of two per-thread values (NaN-free: callers keep a value only
// when it is below the running +inf start, the reference's `if (d < m) m = d`)
// folded into dst0 / dst1 with one atomicMin each. Every thread of the block calls it.
__device__ __forceinline__ void block_min_into(double a, double b, unsigned long long* dst0,
                                               unsigned long long* dst1) {
  __shared__ double sa[32], sb[32];
  for (int o = 16; o > 0; o >>= 1) {
    const double ta = __shfl_down_sync(0xffffffffu, a, o), tb = __shfl_down_sync(0xffffffffu, b, o);
    if (ta < a) a = ta;
    if (tb < b) b = tb;
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sa[w] = a; sb[w] = b; }
  __syncthreads();
  if (w == 0) {
    const int nw = (int)(blockDim.x >> 5);
    a = l < nw ? sa[l] : INFINITY;
    b = l < nw ? sb[l] : INFINITY;
    for (int o = 16; o > 0; o >>= 1) {
      const double ta = __shfl_down_sync(0xffffffffu, a, o), tb = __shfl_down_sync(0xffffffffu, b, o);
      if (ta < a) a = ta;
      if (tb < b) b = tb;
    }
    if (l == 0) {
      if (a < INFINITY) atomicMin(dst0, ord_of(a));
      if (dst1 && b < INFINITY) atomicMin(dst1, ord_of(b));
    }
  }
}

// cint[CI_MOVED] = 1 when some coordinate moved more than `travel` from base.
__global__ void k_moved(const double* x, const double* base, int n3, double travel, int* cint) {
  int bad = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x)
    if (!(fabs(x[i] - base[i]) <= travel)) bad = 1;
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&cint[CI_MOVED], 1);
}

__global__ void k_lerp(double* out, const double* x0, const double* x, double t, int n3) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) out[i] = x0[i] + t * (x[i] - x0[i]);
}

// ---- active set (contact-assembly.ts:164-220) -------------------------------------
__device__ __forceinline__ void cand_closest(const CView& v, const double* x, const int* r, Closest& cp) {
  double P[3], A[3], B[3], C[3];
  if (r[0] == 0) {
    cpos(v.c, x, r[1], P); cpos(v.c, x, r[2], A); cpos(v.c, x, r[3], B); cpos(v.c, x, r[4], C);
    cp = closest_vt(P, A, B, C);
  } else {
    cpos(v.c, x, r[2], A); cpos(v.c, x, r[3], B); cpos(v.c, x, r[4], C); cpos(v.c, x, r[5], P);
    cp = closest_ee(A, B, C, P);
  }
}

// Candidates of the current query: 15 per self pair, 12 per static pair.
__device__ __forceinline__ int cand_count(const CView& v) { return 15 * (int)v.ccnt[0] + 12 * (int)v.ccnt[1]; }

// Record (kind, p, a, b, c, d) of candidate i, decoded from its pair
// (expandTriPair, contact-assembly.ts:91-115). Candidates are slot-major: slot s
// of self pair k is s * P + k, slot s of static pair k is 15 P + s * Q + k (P self
// pairs, Q static pairs), so a warp evaluates one kind for 32 pairs. Self slots
// 0-2: VT of A's vertices against B, 3-5: VT of B's vertices against A, 6-14:
// EE of edge ea of A against edge eb of B (void, kind 3, when the edges share a
// vertex). Static slots 0-2: VT of A's vertices against the static triangle,
// 3-11: EE. Static ids are stored as -(id + 2). The order of the records is
// free: every consumer orders them by key.
__device__ __forceinline__ void cand_rec(const CView& v, int i, int* r) {
  const int P = (int)v.ccnt[0];
  const int e0[3] = {0, 1, 2}, e1[3] = {1, 2, 0};
  if (i < 15 * P) {
    const int slot = i / P, k = i - slot * P;
    const int2 pr = v.selfPairs[k];
    const int A[3] = {(int)v.idx[pr.x * 3], (int)v.idx[pr.x * 3 + 1], (int)v.idx[pr.x * 3 + 2]};
    const int B[3] = {(int)v.idx[pr.y * 3], (int)v.idx[pr.y * 3 + 1], (int)v.idx[pr.y * 3 + 2]};
    if (slot < 3) {
      r[0] = 0; r[1] = A[slot]; r[2] = B[0]; r[3] = B[1]; r[4] = B[2]; r[5] = -1;
    } else if (slot < 6) {
      r[0] = 0; r[1] = B[slot - 3]; r[2] = A[0]; r[3] = A[1]; r[4] = A[2]; r[5] = -1;
    } else {
      const int ea = (slot - 6) / 3, eb = (slot - 6) - 3 * ea;
      const int a = A[e0[ea]], b = A[e1[ea]], c = B[e0[eb]], d = B[e1[eb]];
      if (a == c || a == d || b == c || b == d) {
        r[0] = 3; r[1] = r[2] = r[3] = r[4] = r[5] = 0;
      } else {
        r[0] = 1; r[1] = -1; r[2] = a; r[3] = b; r[4] = c; r[5] = d;
      }
    }
    return;
  }
  const int Q = (int)v.ccnt[1];
  const int j = i - 15 * P, slot = j / Q, k = j - slot * Q;
  const int2 pr = v.staticPairs[k];
  const int A[3] = {(int)v.idx[pr.x * 3], (int)v.idx[pr.x * 3 + 1], (int)v.idx[pr.x * 3 + 2]};
  const int B[3] = {-((int)v.sidx[pr.y * 3] + 2), -((int)v.sidx[pr.y * 3 + 1] + 2), -((int)v.sidx[pr.y * 3 + 2] + 2)};
  if (slot < 3) {
    r[0] = 0; r[1] = A[slot]; r[2] = B[0]; r[3] = B[1]; r[4] = B[2]; r[5] = -2;
  } else {
    const int ea = (slot - 3) / 3, eb = (slot - 3) - 3 * ea;
    r[0] = 1; r[1] = -1; r[2] = A[e0[ea]]; r[3] = A[e1[ea]]; r[4] = B[e0[eb]]; r[5] = B[e1[eb]];
  }
}

// Distance of every candidate (for the minima) and the order keys of the active
// ones, appended through a warp-aggregated counter (cint[CI_NCAND]): their
// positions are arbitrary, the radix sort that follows imposes the reference's
// (kind, p, a, b, c, d) order, and equal keys are identical records. The grid
// strides over the candidate count on the device; keys past `cap` are counted
// but not stored (the host grows the buffers and repeats the query).
__global__ void __launch_bounds__(kCT) k_cand_flags(CView v, const double* x, int cap, Key<4>* keys, uint32_t* pay) {
  const int total = cand_count(v);
  double dmin = INFINITY;
  for (int base = blockIdx.x * blockDim.x; base < total; base += gridDim.x * blockDim.x) {
    const int i = base + threadIdx.x;
    bool act = false;
    CandKey k{0, 0};
    if (i < total) {
      int r[6];
      cand_rec(v, i, r);
      if (r[0] != 3) {
        Closest cp;
        cand_closest(v, x, r, cp);
        act = !(cp.dist >= v.c.dHat || cp.dist < 1e-12);
        if (cp.dist < dmin) dmin = cp.dist;
        if (act) {
          k = cand_key(r, v.ns, v.idBits, 0, 0);
          if (r[0] == 0) atomicAdd(&v.cint[CI_NVT], 1);
        }
      }
    }
    const uint32_t mask = __ballot_sync(0xffffffffu, act);
    if (!mask) continue;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    uint32_t pbase = 0;
    if (lane == leader) pbase = atomicAdd((uint32_t*)&v.cint[CI_NCAND], (uint32_t)__popc(mask));
    pbase = __shfl_sync(0xffffffffu, pbase, leader);
    if (act) {
      const uint32_t pos = pbase + __popc(mask & ((1u << lane) - 1u));
      if (pos < (uint32_t)cap) {
        keys[pos].w[0] = (uint32_t)(k.hi >> 32);
        keys[pos].w[1] = (uint32_t)k.hi;
        keys[pos].w[2] = (uint32_t)(k.lo >> 32);
        keys[pos].w[3] = (uint32_t)k.lo;
        pay[pos] = (uint32_t)i;
      }
    }
  }
  block_min_into(dmin, INFINITY, &v.omin[2], nullptr);
}

// Floor flags, and the floor distances folded into the active-set minimum
// (contact-assembly.ts:200-215).
__global__ void k_floor_flags(CView v, const double* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double dmin = INFINITY;
  if (i < v.n) {
    if (!v.c.hasFloor) {
      v.fflag[i] = 0;
    } else {
      const double d = x[i * 3 + 1] - v.c.floorY;
      if (d < dmin) dmin = d;
      v.fflag[i] = d >= v.c.dHat ? 0u : 1u;
    }
  }
  block_min_into(dmin, INFINITY, &v.omin[2], nullptr);
}

// Frozen record j of the active set from the j-th candidate in key order
// (updateActiveSet, contact-assembly.ts:164-220).
__global__ void k_cand_active(CView v, const double* x, const uint32_t* order, int nAct) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (nAct < 0) nAct = v.acnt[AC_NCAND];
  if (j >= nAct) return;
  int r[6];
  cand_rec(v, (int)order[j], r);
  Closest cp;
  cand_closest(v, x, r, cp);
  Frozen f;
  f.kind = r[0]; f.p = r[1]; f.a = r[2]; f.b = r[3]; f.c = r[4]; f.d = r[5];
  f.nx = cp.rx / cp.dist; f.ny = cp.ry / cp.dist; f.nz = cp.rz / cp.dist;
  if (r[0] == 0) {
    f.d = -1;
    f.w1 = cp.s; f.w2 = cp.t; f.w0 = 1 - cp.s - cp.t; f.w3 = 0;
  } else {
    f.p = -1;
    f.w0 = 1 - cp.s; f.w1 = cp.s; f.w2 = -(1 - cp.t); f.w3 = -cp.t;
  }
  v.active[j] = f;
}

__global__ void k_floor_compact(CView v, const double* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n || !v.c.hasFloor) return;
  const double d = x[i * 3 + 1] - v.c.floorY;
  if (d >= v.c.dHat) return;
  Frozen f;
  f.kind = 2; f.p = i; f.a = f.b = f.c = f.d = -1;
  f.w0 = f.w1 = f.w2 = f.w3 = 0;
  f.nx = 0; f.ny = 1; f.nz = 0;
  v.active[v_ncand(v) + v.fflag[i]] = f;
}

__global__ void k_active_reset(CView v) {
  v.cint[CI_NVT] = 0;
  v.cint[CI_NCAND] = 0;
  v.omin[2] = kOrdInf;
}
__global__ void k_active_min(CView v) {
  if (v.cint[CI_MOVED]) return;  // the query is repeated on a rebuilt superset
  const double m = dbl_of(v.omin[2]);
  if (m < v.diag->minDistance) v.diag->minDistance = m;
}

// CSR records: one per (contact, slot) whose vertex is a cloth vertex.
__global__ void k_csr_records(CView v, Key<1>* k, uint32_t* p, int na) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  na = v_na(v, na);
  if (i >= na * 4) return;
  const int c = i >> 2, slot = i & 3;
  const Frozen f = v.active[c];
  int vert = -1;
  if (f.kind == 2) vert = slot == 0 ? f.p : -1;
  else if (f.kind == 0) vert = slot == 0 ? f.p : slot == 1 ? f.a : slot == 2 ? f.b : f.c;
  else vert = slot == 0 ? f.a : slot == 1 ? f.b : slot == 2 ? f.c : f.d;
  // unused slots sort after every vertex (key n): with keys below 2^16 the
  // sort skips its two high byte passes
  k[i].w[0] = vert >= 0 ? (uint32_t)vert : (uint32_t)v.n;
  p[i] = (uint32_t)i;
}

__global__ void k_csr_offsets(const Key<1>* k, int nrec, uint32_t* off, int n, const int* dna = nullptr) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (dna) nrec = 4 * *dna;
  if (v > n) return;
  int lo = 0, hi = nrec;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (k[mid].w[0] < (uint32_t)v) lo = mid + 1;
    else hi = mid;
  }
  off[v] = (uint32_t)lo;
}

// ---- barrier + lagged friction (contact-assembly.ts:262-285) -----------------------
__device__ __forceinline__ void lag_key(const Frozen& f, int ns, Key<6>& k) {
  const uint32_t off = (uint32_t)(ns + 2);
  k.w[0] = (uint32_t)f.kind;
  if (f.kind == 0) {
    int t0 = f.a, t1 = f.b, t2 = f.c, tmp;
    if (t1 < t0) { tmp = t0; t0 = t1; t1 = tmp; }
    if (t2 < t1) { tmp = t1; t1 = t2; t2 = tmp; }
    if (t1 < t0) { tmp = t0; t0 = t1; t1 = tmp; }
    k.w[1] = (uint32_t)f.p + off; k.w[2] = (uint32_t)t0 + off; k.w[3] = (uint32_t)t1 + off;
    k.w[4] = (uint32_t)t2 + off;
  } else {
    int e1a = min(f.a, f.b), e1b = max(f.a, f.b), e2a = min(f.c, f.d), e2b = max(f.c, f.d);
    if (e2a < e1a || (e2a == e1a && e2b < e1b)) {
      int t = e1a; e1a = e2a; e2a = t;
      t = e1b; e1b = e2b; e2b = t;
    }
    k.w[1] = (uint32_t)e1a + off; k.w[2] = (uint32_t)e1b + off; k.w[3] = (uint32_t)e2a + off;
    k.w[4] = (uint32_t)e2b + off;
  }
  k.w[5] = 0;
}

// Latest committed (n, lambdaN) for a VT/EE key; false when never committed.
__device__ __forceinline__ bool lag_find(const CView& v, const Key<6>& k, double4& out) {
  int lo = 0, hi = v_lag(v);  // first entry whose key words exceed k (seq ignored)
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const Key<6>& e = v.lagKeys[mid];
    bool le = true;
    for (int w = 0; w < 5; w++) {
      if (e.w[w] != k.w[w]) { le = e.w[w] < k.w[w]; break; }
    }
    if (le) lo = mid + 1;
    else hi = mid;
  }
  if (lo == 0) return false;
  const Key<6>& e = v.lagKeys[lo - 1];
  for (int w = 0; w < 5; w++)
    if (e.w[w] != k.w[w]) return false;
  out = v.lagVals[lo - 1];
  return true;
}

__device__ __forceinline__ void relative_slip(const CView& v, const double* x, const Frozen& f, double u[3]) {
  auto D = [&](int q, double o[3]) {
    if (q < 0) { o[0] = o[1] = o[2] = 0; return; }
    o[0] = x[q * 3] - v.x0[q * 3]; o[1] = x[q * 3 + 1] - v.x0[q * 3 + 1]; o[2] = x[q * 3 + 2] - v.x0[q * 3 + 2];
  };
  if (f.kind == 2) { D(f.p, u); return; }
  if (f.kind == 0) {
    // the third triangle vertex reads D(c.d), a negative id (reference behaviour)
    double dp[3], da[3], db[3], dc[3];
    D(f.p, dp); D(f.a, da); D(f.b, db); D(f.d, dc);
    for (int i = 0; i < 3; i++) u[i] = dp[i] - (f.w0 * da[i] + f.w1 * db[i] + f.w2 * dc[i]);
    return;
  }
  double da[3], db[3], dc[3], dd[3];
  D(f.a, da); D(f.b, db); D(f.c, dc); D(f.d, dd);
  for (int i = 0; i < 3; i++) u[i] = f.w0 * da[i] + f.w1 * db[i] + f.w2 * dc[i] + f.w3 * dd[i];
}

// Lagged normal and normal force of a contact at distance d: the committed
// (n, lambdaN) of its key, else the frozen normal and the barrier's normal force
// at d (energyGrad, contact-assembly.ts:262-285).
__device__ __forceinline__ void fric_lagged(const CView& v, const Frozen& f, double d, double& nx, double& ny,
                                            double& nz, double& lam) {
  const Contact& c = v.c;
  nx = f.nx; ny = f.ny; nz = f.nz;
  bool has = false;
  double4 lv;
  if (f.kind == 2) {
    if (v.lagFloorOk[f.p]) { has = true; lv = make_double4(0, 1, 0, v.lagFloor[f.p]); }
  } else {
    Key<6> k;
    lag_key(f, c.ns, k);
    has = lag_find(v, k, lv);
  }
  if (has) { nx = lv.x; ny = lv.y; nz = lv.z; lam = lv.w; }
  else lam = barrier_normal_force(d, c.dHat, c.kappa, 1);
}

// Per contact: active flag (dd), barrier dE/dd and friction args (cg), the
// energy and friction-work chain terms (tc, tf).
__global__ void k_contact_prep(CView v, const double* x, int na) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v_na(v, na)) return;
  const Frozen f = v.active[i];
  const Contact& c = v.c;
  const double d = js_max(frozen_dist(c, x, f), 1e-12);
  if (d >= c.dHat) {
    v.dd[i] = 0; v.tc[i] = 0; v.tf[i] = 0;
    return;
  }
  v.dd[i] = 1;
  v.tc[i] = c.kappa * barrier_value(d, c.dHat);
  const double g = barrier_grad_scalar(d, c.dHat, c.kappa, 1);
  double nx, ny, nz, lam;
  fric_lagged(v, f, d, nx, ny, nz, lam);
  double u[3], fr[3];
  relative_slip(v, x, f, u);
  coulomb_force(u, nx, ny, nz, lam, c.mu, c.eps, fr);
  v.cg[i * 4] = g;
  v.cg[i * 4 + 1] = -fr[0];
  v.cg[i * 4 + 2] = -fr[1];
  v.cg[i * 4 + 3] = -fr[2];
  v.tf[i] = fr[0] * u[0] + fr[1] * u[1] + fr[2] * u[2];
}

// Barrier energy and friction work of the step's diagnostics. The FP64 path
// adds the terms left to right like the reference; the mixed path (tree = 1)
// uses a fixed-order block tree: each of the 1024 threads adds a strided
// subset, then warp and block trees (same bits on every run).
__global__ void __launch_bounds__(1024) k_contact_chains(CView v, int na, int tree) {
  if (na < 0) na = v.acnt ? v.acnt[AC_NA] : 0;
  if (!tree) {
    if (threadIdx.x == 0) v.diag->barrierEnergy = seq_sum(v.tc, na);
    if (threadIdx.x == 32) v.diag->frictionWork = v.diag->frictionWork + seq_sum(v.tf, na);
    return;
  }
  __shared__ double ws[2][32];
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < na; i += blockDim.x) {
    a += v.tc[i];
    b += v.tf[i];
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) { ws[0][w] = a; ws[1][w] = b; }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    a = lane < nw ? ws[0][lane] : 0.0;
    b = lane < nw ? ws[1][lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if (lane == 0) {
      v.diag->barrierEnergy = a;
      v.diag->frictionWork = v.diag->frictionWork + b;
    }
  }
}

// The contact gradient in two passes: one thread per (contact, slot) record
// computes the record's barrier and friction shares (a vertex may sit in many
// contacts); each vertex then adds its records' shares in record order, the
// order and the operations of a per-vertex walk (contact-assembly.ts:298-341).
__global__ void k_contact_grad_rec(CView v, int nrec) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nrec || q >= (int)v.c.cOff[v.n]) return;
  const uint32_t rec = v.c.cRec[q];
  const int ci = rec >> 2, slot = rec & 3;
  double a[3] = {0, 0, 0}, b[3] = {0, 0, 0};
  if (v.dd[ci] != 0) {
    const Frozen f = v.active[ci];
    dist_grad_slot(f, slot, v.cg[ci * 4], a);
    friction_slot(f, slot, v.cg + ci * 4 + 1, b);
  }
  double* o = v.c.recScratch + (size_t)q * 6;
  o[0] = a[0]; o[1] = a[1]; o[2] = a[2]; o[3] = b[0]; o[4] = b[1]; o[5] = b[2];
}
__global__ void k_contact_grad_gather(CView v, double* cgrad) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= v.n) return;
  double o[3] = {0, 0, 0};
  for (uint32_t k = v.c.cOff[q]; k < v.c.cOff[q + 1]; k++) {
    const double* r = v.c.recScratch + (size_t)k * 6;
    o[0] += r[0]; o[1] += r[1]; o[2] += r[2];
    o[0] += r[3]; o[1] += r[4]; o[2] += r[5];
  }
  cgrad[q * 3] = o[0]; cgrad[q * 3 + 1] = o[1]; cgrad[q * 3 + 2] = o[2];
}

// addDiagEstimate (contact-assembly.ts:436-471): dd = kappa max(b'', 0).
__global__ void k_contact_curv(CView v, const double* x, int na) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v_na(v, na)) return;
  const double d = js_max(frozen_dist(v.c, x, v.active[i]), 1e-12);
  v.dd[i] = d >= v.c.dHat ? 0.0 : barrier_curvature(d, v.c.dHat, v.c.kappa);
}

// The diagonal estimate in the same two passes (addDiagEstimate,
// contact-assembly.ts:436-471).
__global__ void k_contact_diag_rec(CView v, int nrec) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nrec || q >= (int)v.c.cOff[v.n]) return;
  const uint32_t rec = v.c.cRec[q];
  const int ci = rec >> 2, slot = rec & 3;
  double c[3] = {0, 0, 0};
  const double kk = v.dd[ci];
  if (kk != 0) {
    const Frozen f = v.active[ci];
    if (f.kind == 2) {
      c[1] = kk;
    } else {
      const double n2[3] = {f.nx * f.nx, f.ny * f.ny, f.nz * f.nz};
      if (f.kind == 0 && slot == 0) {
        for (int a = 0; a < 3; a++) c[a] = kk * n2[a];
      } else {
        const double w = f.kind == 0 ? (slot == 1 ? f.w0 : slot == 2 ? f.w1 : f.w2)
                                     : (slot == 0 ? f.w0 : slot == 1 ? f.w1 : slot == 2 ? f.w2 : f.w3);
        for (int a = 0; a < 3; a++) c[a] = kk * w * w * n2[a];
      }
    }
  }
  double* o = v.c.recScratch + (size_t)q * 6;
  o[0] = c[0]; o[1] = c[1]; o[2] = c[2];
}
__global__ void k_contact_diag_gather(CView v, double* diag) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= v.n) return;
  double o[3] = {diag[q * 3], diag[q * 3 + 1], diag[q * 3 + 2]};
  for (uint32_t k = v.c.cOff[q]; k < v.c.cOff[q + 1]; k++) {
    const double* r = v.c.recScratch + (size_t)k * 6;
    o[0] += r[0]; o[1] += r[1]; o[2] += r[2];
  }
  diag[q * 3] = o[0]; diag[q * 3 + 1] = o[1]; diag[q * 3 + 2] = o[2];
}

// Exact-Newton mode: the friction potential's data at x for this Newton
// iteration (fh, see Contact): mu lambda and the lagged normal of every contact
// inside dHat (as its gradient term in k_contact_prep), s = mu lambda / m and
// t = P u / m with m = sqrt(|P u|^2 + eps^2), the gradient's own magnitude.
__global__ void k_contact_fric(CView v, const double* x, int na, double* fh) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v_na(v, na)) return;
  double* o = fh + (size_t)i * 8;
  const Frozen f = v.active[i];
  const Contact& c = v.c;
  const double d = js_max(frozen_dist(c, x, f), 1e-12);
  if (d >= c.dHat) {
    for (int k = 0; k < 8; k++) o[k] = 0;
    return;
  }
  double nx, ny, nz, lam;
  fric_lagged(v, f, d, nx, ny, nz, lam);
  double u[3];
  relative_slip(v, x, f, u);
  const double un = u[0] * nx + u[1] * ny + u[2] * nz;
  const double t[3] = {u[0] - un * nx, u[1] - un * ny, u[2] - un * nz};
  const double mag = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2] + c.eps * c.eps);
  const double ml = c.mu * fmax(0.0, lam);
  o[0] = ml;
  o[1] = ml / mag;
  o[2] = t[0] / mag; o[3] = t[1] / mag; o[4] = t[2] / mag;
  o[5] = nx; o[6] = ny; o[7] = nz;
}

// meritEnergy terms (contact-assembly.ts:419-428); in exact-Newton mode plus
// the friction potential mu lambda sqrt(|P u|^2 + eps^2) with this iteration's
// frozen mu lambda and normal.
__global__ void k_contact_merit(CView v, const double* x, int na) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v_na(v, na)) return;
  const Frozen f = v.active[i];
  const double d = js_max(frozen_dist(v.c, x, f), 1e-12);
  double e = d >= v.c.dHat ? 0.0 : v.c.kappa * barrier_value(d, v.c.dHat);
  if (v.c.fric) {
    const double* fh = v.c.fh + (size_t)i * 8;
    if (fh[0] != 0) {
      double u[3];
      relative_slip(v, x, f, u);
      const double un = u[0] * fh[5] + u[1] * fh[6] + u[2] * fh[7];
      const double t[3] = {u[0] - un * fh[5], u[1] - un * fh[6], u[2] - un * fh[7]};
      e += fh[0] * sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2] + v.c.eps * v.c.eps);
    }
  }
  v.tc[i] = e;
}

// commit (contact-assembly.ts:475-485): floor multipliers in a per-vertex
// table; VT/EE entries appended to the lag table (key, commit sequence).
__global__ void k_contact_commit(CView v, const double* x, int na, Key<6>* lk, uint32_t* lp, double4* lval,
                                 int base, int commitNo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (v.acnt) {
    na = v.acnt[AC_NA];
    base = v.acnt[AC_LAG];
    commitNo = v.acnt[AC_COMMIT];
  }
  if (i >= na) return;
  const Frozen f = v.active[i];
  const double d = js_max(frozen_dist(v.c, x, f), 1e-12);
  const bool ok = d < v.c.dHat;
  const double lam = ok ? barrier_normal_force(d, v.c.dHat, v.c.kappa, 1) : 0.0;
  if (f.kind == 2) {
    if (ok) { v.lagFloor[f.p] = lam; v.lagFloorOk[f.p] = 1; }
    return;
  }
  if (i >= v_ncand(v)) return;
  const int e = base + i;
  Key<6> k;
  if (ok) {
    lag_key(f, v.c.ns, k);
    k.w[5] = ((uint32_t)commitNo << 24) | (uint32_t)i;
  } else {
    for (int w = 0; w < 6; w++) k.w[w] = 0xffffffffu;
  }
  lk[e] = k;
  lp[e] = (uint32_t)e;
  lval[e] = make_double4(f.nx, f.ny, f.nz, lam);
}

__global__ void k_iota(uint32_t* p, int n, const int* dn = nullptr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (dn) n = min(n, *dn);
  if (i < n) p[i] = (uint32_t)i;
}

// dn (optional): n read on the device.
__global__ void k_gather_vals(const double4* src, const uint32_t* order, int n, double4* dst,
                              const int* dn = nullptr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (dn) n = min(n, *dn);
  if (i < n) dst[i] = src[order[i]];
}

// ---- trial validation (contact-assembly.ts:489-553) ----------------------------------
__global__ void k_trial_reset(CView v) {
  v.cint[CI_FIRSTNF] = INT_MAX;
  v.cint[CI_FLOORBAD] = 0;
  v.cint[CI_VALID] = 0;
  v.cint[CI_NBAD] = 0;
  v.badKey[0] = ~0ull;
  v.badKey[1] = ~0ull;
  v.omin[0] = kOrdInf;
  v.omin[1] = kOrdInf;
}

// Trial distance and CCD of candidate i; returns its distance and TOI for the
// minima (+inf when it has none).
__device__ __forceinline__ void trial_one(const CView& v, const double* xt, int i, double dMin, double& dOut,
                                          double& tOut) {
  v.cflag[i] = 0;
  int r[6];
  cand_rec(v, i, r);
  if (r[0] == 3) return;
  Closest cp;
  cand_closest(v, xt, r, cp);
  dOut = cp.dist;
  if (!isfinite(cp.dist)) atomicMin(&v.cint[CI_FIRSTNF], i);
  int ids[4];
  if (r[0] == 0) {
    if (r[1] < 0 && r[2] < 0) return;
    ids[0] = r[1]; ids[1] = r[2]; ids[2] = r[3]; ids[3] = r[4];
  } else {
    if (r[2] < 0 && r[3] < 0 && r[4] < 0 && r[5] < 0) return;
    ids[0] = r[2]; ids[1] = r[3]; ids[2] = r[4]; ids[3] = r[5];
  }
  double P0[12], P1[12];
  for (int k = 0; k < 4; k++) {
    cpos(v.c, v.x0, ids[k], P0 + k * 3);
    cpos(v.c, xt, ids[k], P1 + k * 3);
  }
  const double toi = trial_ccd(r[0] == 0 ? 0 : 1, P0, P1, cp.dist, dMin);
  tOut = toi;
  uint32_t st = 0;
  if (isnan(toi)) st = 2;
  else if (toi > 0 && toi < 1 - 1e-9) st = 1;
  if (!st) return;
  v.cflag[i] = st;
  // The reference stops at the first failing candidate in key order; its
  // status (NaN or crossing) is the low two bits of the smallest (key, status).
  atomicMin(&v.badKey[0], (unsigned long long)cand_key(r, v.ns, v.idBits, 2, st).hi);
  const int j = atomicAdd(&v.cint[CI_NBAD], 1);
  if (j < kBadCap) v.badList[j] = i;
}

// checkTrial's candidate loops (contact-assembly.ts:498-535): exact distances at
// the trial, CCD of the segment, and their minima.
__global__ void __launch_bounds__(kCT) k_trial_cand(CView v, const double* xt, double dMin) {
  const int total = cand_count(v);
  double d = INFINITY, t = INFINITY;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    double dOut = INFINITY, tOut = INFINITY;
    trial_one(v, xt, i, dMin, dOut, tOut);
    if (dOut < d) d = dOut;
    if (tOut < t) t = tOut;
  }
  block_min_into(d, t, &v.omin[0], &v.omin[1]);
}

// Second half of the smallest failing (key, status): the low word among the
// failing candidates whose high word is the minimum. Walks the list of failing
// indices, or every candidate when more failed than the list holds.
__global__ void k_trial_bad_lo(CView v) {
  const int nbad = v.cint[CI_NBAD];
  if (nbad == 0) return;
  const bool listed = nbad <= kBadCap;
  const int cnt = listed ? nbad : cand_count(v);
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < cnt; j += gridDim.x * blockDim.x) {
    const int i = listed ? v.badList[j] : j;
    const uint32_t st = v.cflag[i];
    if (!st) continue;
    int r[6];
    cand_rec(v, i, r);
    const CandKey k = cand_key(r, v.ns, v.idBits, 2, st);
    if (k.hi == v.badKey[0]) atomicMin(&v.badKey[1], (unsigned long long)k.lo);
  }
}

__global__ void k_trial_floor(CView v, const double* xt, double dMin) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  double d = INFINITY, t = INFINITY;
  if (q < v.n && v.c.hasFloor) {
    const double dd = xt[q * 3 + 1] - v.c.floorY;
    if (dd < d) d = dd;
    const double y0 = v.x0[q * 3 + 1] - v.c.floorY;
    const double yT = xt[q * 3 + 1] - v.c.floorY;
    if (!(y0 - fabs(yT - y0) > dMin) && y0 > dMin && yT <= dMin && y0 > yT) {
      const double toi = (y0 - dMin) / (y0 - yT);
      if (toi < t) t = toi;
      if (toi < 1 - 1e-9) atomicOr(&v.cint[CI_FLOORBAD], 1);
    }
  }
  block_min_into(d, t, &v.omin[0], &v.omin[1]);
}

__global__ void k_trial_final(CView v, double dMin) {
  const double minDist = dbl_of(v.omin[0]);
  const double minTOI = dbl_of(v.omin[1]);
  if (v.gradGate && !(v.gradGate[0] >= v.gradTol)) {  // the iteration ends at its convergence test
    v.cint[CI_VALID] = 0;
    return;
  }
  if (v.cint[CI_MOVED]) {  // the query is repeated on a rebuilt superset
    v.cint[CI_VALID] = -1;
    return;
  }
  int valid = 0;
  DevDiag* dg = v.diag;
  if (v.cint[CI_FIRSTNF] != INT_MAX) {
    dg->ccdFailures += 1;
  } else if (minDist <= dMin) {
  } else if (v.badKey[0] != ~0ull) {
    if ((v.badKey[1] & 3ull) == 2) dg->ccdFailures += 1;
  } else if (v.cint[CI_FLOORBAD]) {
  } else {
    valid = 1;
    if (minDist < dg->minDistance) dg->minDistance = minDist;
    if (minTOI < dg->minTOI) dg->minTOI = minTOI;
  }
  dg->trialMinDist = minDist;
  dg->trialMinTOI = minTOI;
  v.cint[CI_VALID] = valid;
}

// ---- restitution-0 filter (newton.ts:238-303) -----------------------------------------
// Restitution-0 impulse of one VT or EE contact (newton.ts:246-301).
__device__ __forceinline__ void kill_one(const Frozen& c, double* vel) {
  if (c.kind == 0) {
    const double vp[3] = {vel[c.p * 3], vel[c.p * 3 + 1], vel[c.p * 3 + 2]};
    double tx = 0, ty = 0, tz = 0;
    const double ws[3] = {c.w0, c.w1, c.w2};
    const int vs[3] = {c.a, c.b, c.c};
    for (int k = 0; k < 3; k++) {
      if (vs[k] < 0) continue;
      tx += ws[k] * vel[vs[k] * 3];
      ty += ws[k] * vel[vs[k] * 3 + 1];
      tz += ws[k] * vel[vs[k] * 3 + 2];
    }
    const double rel = (vp[0] - tx) * c.nx + (vp[1] - ty) * c.ny + (vp[2] - tz) * c.nz;
    if (rel < 0) {
      const double j = -0.5 * rel;
      vel[c.p * 3] += j * c.nx;
      vel[c.p * 3 + 1] += j * c.ny;
      vel[c.p * 3 + 2] += j * c.nz;
      for (int k = 0; k < 3; k++) {
        if (vs[k] < 0) continue;
        vel[vs[k] * 3] -= j * ws[k] * c.nx;
        vel[vs[k] * 3 + 1] -= j * ws[k] * c.ny;
        vel[vs[k] * 3 + 2] -= j * ws[k] * c.nz;
      }
    }
    return;
  }
  double A[3] = {0, 0, 0}, B[3] = {0, 0, 0};
  {
    double xa[3] = {0, 0, 0}, xb[3] = {0, 0, 0};
    if (c.a >= 0) for (int k = 0; k < 3; k++) xa[k] = vel[c.a * 3 + k];
    if (c.b >= 0) for (int k = 0; k < 3; k++) xb[k] = vel[c.b * 3 + k];
    for (int k = 0; k < 3; k++) A[k] = (xa[k] + xb[k]) / 2;
    double xc[3] = {0, 0, 0}, xd[3] = {0, 0, 0};
    if (c.c >= 0) for (int k = 0; k < 3; k++) xc[k] = vel[c.c * 3 + k];
    if (c.d >= 0) for (int k = 0; k < 3; k++) xd[k] = vel[c.d * 3 + k];
    for (int k = 0; k < 3; k++) B[k] = (xc[k] + xd[k]) / 2;
  }
  const double rel = (A[0] - B[0]) * c.nx + (A[1] - B[1]) * c.ny + (A[2] - B[2]) * c.nz;
  if (rel < 0) {
    const double j = -0.25 * rel;
    const int up[2] = {c.a, c.b}, dn[2] = {c.c, c.d};
    for (int q = 0; q < 2; q++) {
      if (up[q] < 0) continue;
      vel[up[q] * 3] += j * c.nx; vel[up[q] * 3 + 1] += j * c.ny; vel[up[q] * 3 + 2] += j * c.nz;
    }
    for (int q = 0; q < 2; q++) {
      if (dn[q] < 0) continue;
      vel[dn[q] * 3] -= j * c.nx; vel[dn[q] * 3 + 1] -= j * c.ny; vel[dn[q] * 3 + 2] -= j * c.nz;
    }
  }
}

constexpr int kKillRoundsMax = 48 * 1024 * 8;  // contacts whose done bits fit 48 KB of shared memory

// VT/EE impulses in list order by one thread (each sees the earlier updates).
__global__ void k_kill_vtee(CView v, double* vel, int nve) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  if (v.acnt) {
    nve = v.acnt[AC_NCAND];
    if (nve <= kKillRoundsMax) return;  // the rounds kernel handled it
  }
  for (int i = 0; i < nve; i++) kill_one(v.active[i], vel);
}

// Predecessor of each VT/EE contact on each of its cloth vertices: the previous
// contact in that vertex's list (the vertex -> (contact, slot) CSR is in contact
// order), -1 for none or a static vertex.
__global__ void k_kill_pred(CView v, const Key<1>* rk, const uint32_t* rp, const uint32_t* off, int nrec, int nve,
                            int* pred) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (v.acnt) {
    nrec = 4 * v.acnt[AC_NA];
    nve = v.acnt[AC_NCAND];
  }
  if (q >= nrec) return;
  const uint32_t vert = rk[q].w[0];
  const uint32_t pay = rp[q];
  const int c = (int)(pay >> 2), slot = (int)(pay & 3);
  if (c >= nve) return;
  pred[c * 4 + slot] = (vert != 0xffffffffu && q > (int)off[vert]) ? (int)(rp[q - 1] >> 2) : -1;
}

// The same pass by one block in rounds: a contact is applied once its
// predecessor on each of its vertices has been. Contacts applied in one round
// share no vertex, and every vertex receives its contacts' impulses in list
// order, so the velocities equal the one-thread pass bit for bit. The smallest
// pending contact is always ready, so each round applies at least one and
// nve + 1 rounds bound the loop; diag->killStall is set if it ever runs out.
constexpr int kKillThreads = 1024;
__global__ void __launch_bounds__(kKillThreads) k_kill_vtee_rounds(CView v, double* vel, int nve,
                                                                   const int* pred) {
  extern __shared__ uint32_t doneBits[];
  if (v.acnt) {
    // graph-captured step: launched with the largest bitset; longer lists take
    // the one-thread pass (k_kill_vtee) instead
    nve = v.acnt[AC_NCAND];
    if (nve > kKillRoundsMax) return;
  }
  const int words = (nve + 31) >> 5;
  for (int w = threadIdx.x; w < words; w += blockDim.x) doneBits[w] = 0;
  __syncthreads();
  int cur = threadIdx.x;
  auto done = [&](int c) { return c < 0 || c == cur || ((doneBits[c >> 5] >> (c & 31)) & 1u); };
  bool pending = cur < nve;
  for (int round = 0; round <= nve; round++) {
    bool ready = false;
    if (pending) {
      const int4 pr = reinterpret_cast<const int4*>(pred)[cur];
      ready = done(pr.x) && done(pr.y) && done(pr.z) && done(pr.w);
      if (ready) kill_one(v.active[cur], vel);
    }
    __syncthreads();
    if (ready) {
      atomicOr(&doneBits[cur >> 5], 1u << (cur & 31));
      cur += blockDim.x;
      pending = cur < nve;
    }
    if (!__syncthreads_or(pending)) return;
  }
  if (threadIdx.x == 0) v.diag->killStall = 1;
}

__global__ void k_kill_floor(CView v, double* vel, int base, int nf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (v.acnt) {
    base = v.acnt[AC_NCAND];
    nf = v.acnt[AC_NFLOOR];
  }
  if (i >= nf) return;
  const int p = v.active[base + i].p;
  if (vel[p * 3 + 1] < 0) vel[p * 3 + 1] = 0;
}

// ---- host side --------------------------------------------------------------------------
template <class T>
static void dalloc(T*& p, size_t n) {
  if (p) cudaFree(p);
  p = nullptr;
  if (n) CK(cudaMalloc(&p, n * sizeof(T)));
}
template <class T>
static void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

static CView view(ContactHost& h, Solver& s) {
  CView v;
  v.c = s.d.c;
  v.nCand = h.nCand;
  v.nFloor = h.nFloor;
  v.n = h.n;
  v.x0 = s.d.x0;
  v.selfPairs = h.bvh.pairs;
  v.staticPairs = h.spairs;
  v.idx = s.idx.p;
  v.sidx = h.sidx;
  v.ns = h.ns;
  v.idBits = h.idBits;
  v.badKey = h.badKey;
  v.ccnt = (const uint32_t*)(h.cint + CI_SELF);
  v.cflag = h.cflag;
  v.fflag = h.fflag;
  v.omin = h.omin;
  v.badList = h.badList;
  v.gradGate = nullptr;
  v.gradTol = 0;
  v.active = h.active;
  v.dd = h.dd;
  v.cg = h.cg;
  v.tc = h.tc;
  v.tf = h.tf;
  v.lagFloor = h.lagFloor;
  v.lagFloorOk = h.lagFloorOk;
  v.lagKeys = h.lk0;
  v.lagVals = h.lsorted;
  v.lagCount = h.lagCount;
  v.cint = h.cint;
  v.diag = h.diag;
  v.acnt = nullptr;
  return v;
}
// The view of a graph-captured step: device counts, capacity-sized launches.
static CView cview(ContactHost& h, Solver& s) {
  CView v = view(h, s);
  v.acnt = h.acnt;
  v.nCand = 0;
  v.nFloor = 0;
  v.lagCount = 0;
  return v;
}

ContactHost::~ContactHost() {
  for (void** q : {(void**)&spos, (void**)&sidx, (void**)&bvh.box64, (void**)&bvh.boxc, (void**)&bvh.boxr,
                   (void**)&bvh.cent, (void**)&bvh.scene, (void**)&bvh.k0, (void**)&bvh.k1, (void**)&bvh.p0,
                   (void**)&bvh.p1, (void**)&bvh.hist, (void**)&bvh.left, (void**)&bvh.right, (void**)&bvh.parent,
                   (void**)&bvh.depth, (void**)&bvh.nbox, (void**)&bvh.rec, (void**)&bvh.visit, (void**)&bvh.root,
                   (void**)&bvh.pairs, (void**)&badKey, (void**)&spairs,
                   (void**)&cand.k0, (void**)&cand.k1, (void**)&cand.p0, (void**)&cand.p1, (void**)&cand.hist,
                   (void**)&cflag, (void**)&fflag, (void**)&omin, (void**)&badList, (void**)&active, (void**)&dd,
                   (void**)&cg, (void**)&tc, (void**)&tf, (void**)&rk0, (void**)&rk1, (void**)&rp0, (void**)&rp1,
                   (void**)&rhist, (void**)&kpred, (void**)&recScratch, (void**)&fh, (void**)&fdd, (void**)&cOff, (void**)&lagFloor, (void**)&lagFloorOk, (void**)&lk0,
                   (void**)&lk1, (void**)&lp0, (void**)&lp1, (void**)&lhist, (void**)&lval, (void**)&lsorted,
                   (void**)&probe, (void**)&diag, (void**)&cint, (void**)&acnt, (void**)&supPairs,
                   (void**)&supSPairs, (void**)&supBase})
    if (*q) cudaFree(*q);
  if (hint) cudaFreeHost(hint);
  if (hdiag) cudaFreeHost(hdiag);
}

void ContactHost::init(Solver& s, const cs_contact_params* prm, int floor_on, double floor_y, const float* sp,
                       int nsv, const uint32_t* si, int msv) {
  p = *prm;
  hasFloor = floor_on != 0;
  floorY = floor_y;
  n = s.mesh.n;
  m = s.mesh.m;
  ns = nsv;
  ms = msv;
  if ((long)n + ns + 2 >= (1l << 24)) throw std::invalid_argument("too many vertices for the candidate key");
  idBits = cand_id_bits(n, ns);
  if (ms > 0) {
    for (int i = 0; i < 3 * ms; i++)
      if ((int)si[i] >= ns) throw std::invalid_argument("static index out of range");
    dalloc(spos, 3 * (size_t)ns);
    dalloc(sidx, 3 * (size_t)ms);
    CK(cudaMemcpy(spos, sp, 12 * (size_t)ns, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(sidx, si, 12 * (size_t)ms, cudaMemcpyHostToDevice));
  }
  bvh.m = m;
  bvh.ns = ns;
  bvh.ms = ms;
  bvh.idx = s.idx.p;
  bvh.spos = spos;
  bvh.sidx = sidx;
  const size_t nn = std::max(1, 2 * m - 1);
  dalloc(bvh.box64, 6 * (size_t)m);
  dalloc(bvh.boxc, 6 * (size_t)m);
  dalloc(bvh.boxr, 6 * (size_t)m);
  dalloc(bvh.cent, 3 * (size_t)m);
  dalloc(bvh.scene, 6);
  dalloc(bvh.k0, (size_t)m);
  dalloc(bvh.k1, (size_t)m);
  dalloc(bvh.p0, (size_t)m);
  dalloc(bvh.p1, (size_t)m);
  dalloc(bvh.hist, 256 * (size_t)((m + kSortTile - 1) / kSortTile) + 1);
  dalloc(bvh.left, nn);
  dalloc(bvh.right, nn);
  dalloc(bvh.parent, nn);
  dalloc(bvh.depth, nn);
  dalloc(bvh.nbox, 6 * nn);
  dalloc(bvh.rec, 4 * (size_t)std::max(1, m - 1));
  dalloc(bvh.visit, nn);
  dalloc(bvh.root, 1);
  dalloc(badKey, 2);
  dalloc(omin, 3);
  dalloc(badList, kBadCap);
  dalloc(supBase, 3 * (size_t)n);
  dalloc(fflag, (size_t)n + 1);
  dalloc(cOff, (size_t)n + 1);
  dalloc(lagFloor, (size_t)n);
  dalloc(lagFloorOk, (size_t)n);
  dalloc(probe, 3 * (size_t)n);
  dalloc(diag, 1);
  dalloc(cint, CI_N);
  dalloc(acnt, AC_N);
  CK(cudaMemset(acnt, 0, AC_N * sizeof(int)));
  dalloc(csrMemo, 2);
  CK(cudaMemset(csrMemo, 0xff, 2 * sizeof(int)));
  dalloc(supMemo, 4);
  CK(cudaMemset(supMemo, 0, 4 * sizeof(int)));
  dalloc(actDirty, 1);
  CK(cudaMemset(actDirty, 0, sizeof(int)));
  CK(cudaMallocHost(&hint, CI_N * sizeof(int)));
  CK(cudaMallocHost(&hdiag, sizeof(DevDiag)));
  // Capacities sized from the mesh up front: a buffer that grows mid-run costs
  // a cudaFree (a device-wide synchronization) and a cudaMalloc inside a step,
  // measured at 10-70 ms per event. Sixteen pairs per triangle covers the
  // drapes here with room for folds; growth past it still works (doubling).
  const size_t pairs0 = std::max<size_t>(1024, 16 * (size_t)m);
  ensure_pairs(pairs0, ms > 0 ? pairs0 : 64);
  supCap = pairCap;
  supSCap = spairCap;
  dalloc(supPairs, supCap);
  dalloc(supSPairs, supSCap);
  ensure_cands(std::max<size_t>(1024, (size_t)m));
  ensure_flags(15 * pairs0 + (ms > 0 ? 12 * pairs0 : 0));
  {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, dev));
  }
  ensure_active(s, std::max<size_t>(1024, (size_t)n + 2 * (size_t)m));
  ensure_lag(std::max<size_t>(1024, 4 * ((size_t)n + (size_t)m)));
  bvh.flags = cint + CI_OVERFLOW;
  bind(s);
}

void ContactHost::ensure_pairs(size_t np, size_t nsp) {
  if (np > pairCap) { pairCap = 2 * np + 64; dalloc(bvh.pairs, pairCap); }
  if (nsp > spairCap) { spairCap = 2 * nsp + 64; dalloc(spairs, spairCap); }
}
void ContactHost::ensure_cands(size_t nc) {
  if ((int)nc <= cand.cap) return;
  const size_t c = nc + nc / 2 + 256;
  cand.cap = (int)c;
  dalloc(cand.k0, c);
  dalloc(cand.k1, c);
  dalloc(cand.p0, c);
  dalloc(cand.p1, c);
  dalloc(cand.hist, 256 * ((c + kSortTile - 1) / kSortTile) + 1);
}
void ContactHost::ensure_flags(size_t nc) {
  if (nc + 1 <= flagCap) return;
  flagCap = nc + nc / 2 + 256;
  dalloc(cflag, flagCap);
}
void ContactHost::ensure_active(Solver& s, size_t na) {
  if (na <= actCap) return;
  const size_t c = 2 * na + 256;
  actCap = c;
  dalloc(active, c);
  dalloc(dd, c);
  dalloc(cg, 4 * c);
  dalloc(tc, c);
  dalloc(tf, c);
  dalloc(rk0, 4 * c);
  dalloc(rk1, 4 * c);
  dalloc(rp0, 4 * c);
  dalloc(rp1, 4 * c);
  dalloc(rhist, 256 * ((4 * c + kSortTile - 1) / kSortTile) + 1);
  dalloc(kpred, 4 * c);
  dalloc(recScratch, 24 * c);
  dalloc(fh, 8 * c);
  dalloc(fdd, 3 * c);
  dalloc(csrIds, 5 * c);
  if (csrMemo) CK(cudaMemsetAsync(csrMemo, 0xff, 2 * sizeof(int), s.stream));  // the saved list is gone
}
void ContactHost::ensure_lag(size_t nl) {
  if (nl <= lagCap) return;
  const size_t c = 2 * nl + 256;
  // keep existing sorted entries
  Key<6>* ok = nullptr;
  double4* ov = nullptr;
  if (lagCount > 0) {
    CK(cudaMalloc(&ok, lagCount * sizeof(Key<6>)));
    CK(cudaMalloc(&ov, lagCount * sizeof(double4)));
    CK(cudaMemcpy(ok, lk0, lagCount * sizeof(Key<6>), cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(ov, lsorted, lagCount * sizeof(double4), cudaMemcpyDeviceToDevice));
  }
  lagCap = c;
  dalloc(lk0, c);
  dalloc(lk1, c);
  dalloc(lp0, c);
  dalloc(lp1, c);
  dalloc(lhist, 256 * ((c + kSortTile - 1) / kSortTile) + 1);
  dalloc(lval, c);
  dalloc(lsorted, c);
  if (lagCount > 0) {
    CK(cudaMemcpy(lk0, ok, lagCount * sizeof(Key<6>), cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(lsorted, ov, lagCount * sizeof(double4), cudaMemcpyDeviceToDevice));
    cudaFree(ok);
    cudaFree(ov);
  }
}

void ContactHost::bind(Solver& s) {
  Contact& c = s.d.c;
  c.dHat = p.dhat; c.kappa = p.kappa; c.dMin = p.dmin; c.mu = p.mu; c.eps = p.eps;
  c.floorY = floorY;
  c.hasFloor = hasFloor ? 1 : 0;
  c.ns = ns;
  c.spos = spos;
  c.nActive = nCand + nFloor;
  c.nActiveD = nullptr;
  c.active = active;
  c.dd = dd;
  c.cg = cg;
  c.cOff = cOff;
  c.cRec = rp0;
  c.recScratch = recScratch;
  c.fric = fricOn ? 1 : 0;
  c.fh = fh;
  c.fdd = fdd;
  s.d.Tc = tc;
  s.d.hasContact = 1;
}

void ContactHost::read_ints(Solver& s) {
  CK(cudaMemcpyAsync(hint, cint, CI_N * sizeof(int), cudaMemcpyDeviceToHost, s.stream));
  CK(cudaStreamSynchronize(s.stream));
}

void ContactHost::build_superset(Solver& s, const double* x, double padSup) {
  cudaStream_t st = s.stream;
  int64_t& lc = launch_counter();
  CK(cudaMemsetAsync(supMemo, 0, sizeof(int), st));  // captured steps rebuild their own
  CK(cudaMemcpyAsync(supBase, x, 3 * (size_t)n * 8, cudaMemcpyDeviceToDevice, st));
  bvh_build(bvh, s.d.x0, x, padSup, false, st, &lc);
  topoValid = true;
  if (supCap == 0) { supCap = std::max<size_t>(pairCap, 1024); dalloc(supPairs, supCap); }
  if (supSCap == 0) { supSCap = std::max<size_t>(spairCap, 64); dalloc(supSPairs, supSCap); }
  for (int attempt = 0; attempt < 2; attempt++) {
    CK(cudaMemsetAsync(cint, 0, CI_N * sizeof(int), st));
    BvhBufs sb = bvh;
    sb.cnt = (uint32_t*)(cint + CI_SELF);
    sb.pairs = supPairs;
    sb.pairCap = (uint32_t)supCap;
    bvh_append_self(sb, st, &lc);
    if (ms > 0) bvh_append_static(bvh, padSup, supSPairs, (uint32_t)supSCap, (uint32_t*)(cint + CI_STATIC), st, &lc);
    read_ints(s);
    if (hint[CI_OVERFLOW]) throw CapacityError("broadphase traversal aborted (stack deeper than 64 or malformed tree)");
    const size_t P = (uint32_t)hint[CI_SELF], S = ms > 0 ? (uint32_t)hint[CI_STATIC] : 0u;
    nSup = (int)P;
    nSupS = (int)S;
    if (P <= supCap && S <= supSCap) break;
    if (attempt == 1) throw CapacityError("broadphase superset changed between identical traversals");
    if (P > supCap) { supCap = 2 * P + 64; dalloc(supPairs, supCap); }
    if (S > supSCap) { supSCap = 2 * S + 64; dalloc(supSPairs, supSCap); }
  }
  ensure_pairs((size_t)nSup, (size_t)nSupS);
  const size_t bound = 15 * (size_t)nSup + 12 * (size_t)nSupS;
  if (bound > (size_t)INT_MAX / 8) throw CapacityError("too many contact candidates");
  ensure_flags(bound);
  CK(cudaMemsetAsync(cint, 0, CI_N * sizeof(int), st));
}

// Launches one broadphase query (no host synchronization): the pairs of the
// segment xStep -> x padded by `pad`, counted on the device (cint[CI_SELF],
// cint[CI_STATIC]). Queries filter a superset of pairs built for the segment
// x0 -> xBase with the pad widened by kSupTravel: a query whose positions all
// stay within kSupTravel (max norm) of xBase has its swept boxes inside the
// superset's, so filtering the superset by the query's own f64 boxes gives
// exactly the pairs a traversal would. A query that moved further raises
// cint[CI_MOVED]; the kernels that follow then leave no trace, and the caller
// rebuilds the superset around the query and repeats it.
void ContactHost::launch_query(Solver& s, const double* x, double pad) {
  struct Restore {
    Solver& s;
    int prev;
    ~Restore() {
      try {
        s.phase(prev);
      } catch (...) {
      }
    }
  } restore{s, s.phase(PH_BROADPHASE)};
  cudaStream_t st = s.stream;
  int64_t& lc = launch_counter();
  if (!supValid) {
    build_superset(s, x, sup_pad());
    supValid = true;
  }
  CK(cudaMemsetAsync(cint, 0, CI_N * sizeof(int), st));
  const int n3 = 3 * n;
  k_moved<<<std::min(1184, (n3 + 255) / 256), 256, 0, st>>>(x, supBase, n3, kSupTravel, cint);
  bvh_boxes(bvh, s.d.x0, x, pad, st, &lc);
  filter_pairs(bvh, supPairs, nSup, bvh.pairs, (uint32_t)pairCap, (uint32_t*)(cint + CI_SELF), supSPairs, nSupS,
               pad, spairs, (uint32_t)spairCap, (uint32_t*)(cint + CI_STATIC), st, &lc);
  lc++;
}

// Blocks for the grid-stride candidate kernels: enough for the superset's
// bound, at most 8 per SM.
int ContactHost::cand_blocks() const {
  const long bound = 15l * nSup + 12l * nSupS;
  return (int)std::max(1l, std::min((bound + kCT - 1) / kCT, 8l * smCount));
}

void ContactHost::update_active_set(Solver& s, double* x) {
  cudaStream_t st = s.stream;
  int64_t& lc = launch_counter();
  // One host read per query: the counts, and whether the superset covered it.
  for (int attempt = 0;; attempt++) {
    launch_query(s, x, p.dhat);
    CView v = view(*this, s);
    k_active_reset<<<1, 1, 0, st>>>(v);
    k_cand_flags<<<cand_blocks(), kCT, 0, st>>>(v, x, cand.cap, cand.k0, cand.p0);
    k_floor_flags<<<cnb(n), kCT, 0, st>>>(v, x);
    k_active_min<<<1, 1, 0, st>>>(v);
    lc += 4;
    scan_counts(fflag, n, (uint32_t*)(cint + CI_NFLOOR), st, &lc);
    read_ints(s);
    const bool moved = hint[CI_MOVED] != 0, overflow = hint[CI_NCAND] > cand.cap;
    if (!moved && !overflow) break;
    if (attempt >= 2) throw CapacityError("active-set query repeated without settling");
    if (moved) build_superset(s, x, sup_pad());
    if (overflow) ensure_cands((size_t)hint[CI_NCAND]);
  }
  candidatePairs = 15.0 * (uint32_t)hint[CI_SELF] + 12.0 * (uint32_t)(ms > 0 ? hint[CI_STATIC] : 0);
  nCand = hint[CI_NCAND];
  nFloor = hint[CI_NFLOOR];
  nVT = hint[CI_NVT];
  const int na = nCand + nFloor;
  ensure_active(s, na);
  CView v = view(*this, s);
  if (nCand > 0) {
    // Only the active candidates are put in the reference's (kind, p, a, b, c, d) order.
    const bool flip = radix_sort<4>(cand.k0, cand.p0, cand.k1, cand.p1, nCand, cand_key_bits(idBits, 0), cand.hist,
                                    st, &lc);
    k_cand_active<<<cnb(nCand), kCT, 0, st>>>(v, x, flip ? cand.p1 : cand.p0, nCand);
    lc++;
  }
  k_floor_compact<<<cnb(n), kCT, 0, st>>>(v, x);
  lc++;
  activePairs = na;
  vtPairs = nVT;
  eePairs = nCand - nVT;
  floorPairs = nFloor;
  // vertex -> (contact, slot) CSR in contact order
  if (na > 0) {
    k_csr_records<<<cnb(4l * na), kCT, 0, st>>>(v, rk0, rp0, na);
    lc++;
    const bool flip = radix_sort<1>(rk0, rp0, rk1, rp1, 4 * na, 32, rhist, st, &lc);
    if (flip) {
      CK(cudaMemcpyAsync(rk0, rk1, 4 * (size_t)na * sizeof(Key<1>), cudaMemcpyDeviceToDevice, st));
      CK(cudaMemcpyAsync(rp0, rp1, 4 * (size_t)na * 4, cudaMemcpyDeviceToDevice, st));
    }
    k_csr_offsets<<<cnb(n + 1), kCT, 0, st>>>(rk0, 4 * na, cOff, n);
    lc++;
    CK(cudaMemsetAsync(csrMemo, 0xff, 2 * sizeof(int), st));  // captured steps must rebuild
  } else {
    CK(cudaMemsetAsync(csrMemo, 0xff, 2 * sizeof(int), st));
    CK(cudaMemsetAsync(cOff, 0, ((size_t)n + 1) * 4, st));
  }
  bind(s);
}

void ContactHost::gradient_terms(Solver& s) {
  cudaStream_t st = s.stream;
  int64_t& lc = launch_counter();
  update_active_set(s, s.d.x);
  const int na = nCand + nFloor;
  CView v = view(*this, s);
  if (na > 0) {
    k_contact_prep<<<cnb(na), kCT, 0, st>>>(v, s.d.x, na);
    k_contact_chains<<<1, s.mixed() ? 1024 : 64, 0, st>>>(v, na, s.mixed() ? 1 : 0);
    lc += 2;
  } else {
    k_contact_chains<<<1, 64, 0, st>>>(v, 0, 0);
    lc++;
  }
  if (na > 0) {
    k_contact_grad_rec<<<cnb(4l * na), kCT, 0, st>>>(v, 4 * na);
    lc++;
  }
  k_contact_grad_gather<<<cnb(n), kCT, 0, st>>>(v, s.d.cgrad);
  lc++;
  if (na > 0) {
    k_contact_curv<<<cnb(na), kCT, 0, st>>>(v, s.d.x, na);
    k_contact_diag_rec<<<cnb(4l * na), kCT, 0, st>>>(v, 4 * na);
    k_contact_diag_gather<<<cnb(n), kCT, 0, st>>>(v, s.d.diag);
    lc += 3;
  }
}

void ContactHost::friction_terms(Solver& s) {
  const int na = nCand + nFloor;
  fricOn = true;
  bind(s);
  if (na <= 0) return;
  CView v = view(*this, s);
  k_contact_fric<<<cnb(na), kCT, 0, s.stream>>>(v, s.d.x, na, fh);
  launch_counter()++;
}

void ContactHost::merit_energy(Solver& s, const double* x) {
  const int na = nCand + nFloor;
  if (na <= 0) return;
  CView v = view(*this, s);
  k_contact_merit<<<cnb(na), kCT, 0, s.stream>>>(v, x, na);
  launch_counter()++;
}

// checkTrial (contact-assembly.ts:489-553) launched without a host read: the
// candidate and floor kernels, then an asynchronous copy of the counters that
// trial_result reads after the caller's next synchronization.
void ContactHost::trial_launch(Solver& s, const double* xt, const double* gradGate, double gradTol) {
  cudaStream_t st = s.stream;
  int64_t& lc = launch_counter();
  launch_query(s, xt, p.dmin);
  CView v = view(*this, s);
  v.gradGate = gradGate;
  v.gradTol = gradTol;
  k_trial_reset<<<1, 1, 0, st>>>(v);
  k_trial_cand<<<cand_blocks(), kCT, 0, st>>>(v, xt, p.dmin);
  k_trial_bad_lo<<<4 * smCount, kCT, 0, st>>>(v);
  k_trial_floor<<<cnb(n), kCT, 0, st>>>(v, xt, p.dmin);
  k_trial_final<<<1, 1, 0, st>>>(v, p.dmin);
  lc += 5;
  CK(cudaMemcpyAsync(hint, cint, CI_N * sizeof(int), cudaMemcpyDeviceToHost, st));
}

// After a synchronization: 1 valid, 0 invalid, -1 when the query fell outside
// the superset (nothing was recorded; rebuild and repeat).
int ContactHost::trial_result() {
  candidatePairs = 15.0 * (uint32_t)hint[CI_SELF] + 12.0 * (uint32_t)(ms > 0 ? hint[CI_STATIC] : 0);
  return hint[CI_VALID];
}

// A trial whose query fell outside the superset: rebuild around it and check again.
bool ContactHost::trial_redo(Solver& s, const double* xt) {
  build_superset(s, xt, sup_pad());
  trial_launch(s, xt);
  CK(cudaStreamSynchronize(s.stream));
  const int r = trial_result();
  if (r < 0) throw CapacityError("broadphase superset rebuilt around the query does not cover it");
  return r != 0;
}

bool ContactHost::check_trial(Solver& s, const double* xt) {
  for (int attempt = 0;; attempt++) {
    trial_launch(s, xt);
    CK(cudaStreamSynchronize(s.stream));
    const int r = trial_result();
    if (r >= 0) return r != 0;
    if (attempt >= 1) throw CapacityError("broadphase superset rebuilt around the query does not cover it");
    build_superset(s, xt, sup_pad());
  }
}

void ContactHost::commit(Solver& s, const double* x) {
  cudaStream_t st = s.stream;
  int64_t& lc = launch_counter();
  const int na = nCand + nFloor;
  if (na <= 0) return;
  ensure_lag((size_t)lagCount + nCand + 1);
  if (nCand > 0 && lagCount > 0) {
    // the sorted prefix becomes entries 0..lagCount-1 with their values in place
    CK(cudaMemcpyAsync(lval, lsorted, (size_t)lagCount * sizeof(double4), cudaMemcpyDeviceToDevice, st));
    k_iota<<<cnb(lagCount), kCT, 0, st>>>(lp0, lagCount);
    lc++;
  }
  CView v = view(*this, s);
  k_contact_commit<<<cnb(na), kCT, 0, st>>>(v, x, na, lk0, lp0, lval, lagCount, commitNo);
  lc++;
  commitNo++;
  if (nCand > 0) {
    const int total = lagCount + nCand;
    const bool flip = radix_sort<6>(lk0, lp0, lk1, lp1, total, 192, lhist, st, &lc);
    const uint32_t* sp = flip ? lp1 : lp0;
    k_gather_vals<<<cnb(total), kCT, 0, st>>>(lval, sp, total, lsorted);
    lc++;
    if (flip) CK(cudaMemcpyAsync(lk0, lk1, (size_t)total * sizeof(Key<6>), cudaMemcpyDeviceToDevice, st));
    lagCount = total;
  }
}

void ContactHost::kill_approach_velocity(Solver& s) {
  update_active_set(s, s.d.x);
  CView v = view(*this, s);
  if (nCand > 0) {
    const size_t smem = 4 * (((size_t)nCand + 31) / 32);
    if (smem <= 48 * 1024) {
      // The vertex -> (contact, slot) CSR of update_active_set gives each
      // contact's predecessors; the rounds kernel applies them in parallel.
      k_kill_pred<<<cnb(4l * (nCand + nFloor)), kCT, 0, s.stream>>>(v, rk0, rp0, cOff, 4 * (nCand + nFloor), nCand,
                                                                     kpred);
      k_kill_vtee_rounds<<<1, kKillThreads, smem, s.stream>>>(v, s.d.v, nCand, kpred);
      launch_counter() += 2;
    } else {
      k_kill_vtee<<<1, 1, 0, s.stream>>>(v, s.d.v, nCand);
      launch_counter()++;
    }
  }
  if (nFloor > 0) {
    k_kill_floor<<<cnb(nFloor), kCT, 0, s.stream>>>(v, s.d.v, nCand, nFloor);
    launch_counter()++;
  }
}

void ContactHost::begin_step_and_bisect(Solver& s) {
  cudaStream_t st = s.stream;
  DevDiag z{};
  z.minDistance = INFINITY;
  z.minTOI = INFINITY;
  CK(cudaMemcpyAsync(diag, &z, sizeof z, cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(lagFloorOk, 0, (size_t)n, st));
  lagCount = 0;
  commitNo = 0;
  rejections = 0;
  fricOn = false;
  topoValid = false;
  supValid = false;
  candidatePairs = activePairs = vtPairs = eePairs = floorPairs = 0;
  nCand = nFloor = nVT = 0;
  bind(s);
  CK(cudaStreamSynchronize(st));  // z is a host temporary
  if (check_trial(s, s.d.x)) return;
  double lo = 0, hi = 1;
  const int n3 = 3 * n;
  for (int b = 0; b < 8; b++) {
    const double mid = 0.5 * (lo + hi);
    k_lerp<<<cnb(n3), kCT, 0, st>>>(probe, s.d.x0, s.d.x, mid, n3);
    launch_counter()++;
    launch_pins(s.d, probe, st);
    if (check_trial(s, probe)) lo = mid;
    else hi = mid;
    if (hi - lo < 1e-4) break;
  }
  k_lerp<<<cnb(n3), kCT, 0, st>>>(s.d.x, s.d.x0, s.d.x, lo, n3);
  launch_counter()++;
  launch_pins(s.d, s.d.x, st);
}

void ContactHost::fill_stats(Solver& s, cs_step_stats& out) {
  CK(cudaMemcpyAsync(hdiag, diag, sizeof(DevDiag), cudaMemcpyDeviceToHost, s.stream));
  CK(cudaStreamSynchronize(s.stream));
  if (hdiag->killStall != 0) throw std::runtime_error("restitution pass did not complete");
  out.candidate_pairs = candidatePairs;
  out.active_pairs = activePairs;
  out.vt_pairs = vtPairs;
  out.ee_pairs = eePairs;
  out.floor_pairs = floorPairs;
  out.min_distance = hdiag->minDistance;
  out.min_toi = hdiag->minTOI;
  out.barrier_energy = hdiag->barrierEnergy;
  out.friction_work = hdiag->frictionWork;
  out.rejected_line_search_steps = rejections;
  out.ccd_failures = hdiag->ccdFailures;
}

void ContactHost::update_static_positions(Solver& s, const float* sp, int nsv) {
  if (ms <= 0 || nsv != ns) throw std::invalid_argument("static positions must match the static mesh's vertex count");
  for (int i = 0; i < 3 * nsv; i++)
    if (!std::isfinite(sp[i])) throw std::invalid_argument("static positions must be finite");
  CK(cudaMemcpyAsync(spos, sp, 12 * (size_t)ns, cudaMemcpyHostToDevice, s.stream));
  CK(cudaMemsetAsync(supMemo, 0, sizeof(int), s.stream));  // the static pairs moved
  CK(cudaStreamSynchronize(s.stream));  // sp is the caller's
  supValid = false;
  topoValid = false;
}

int ContactHost::read_active(Solver& s, int cap, int32_t* ids6, double* w7) {
  const int na = nCand + nFloor;
  if (na > 0 && ids6 && w7 && cap >= na) {
    std::vector<Frozen> h((size_t)na);
    CK(cudaMemcpyAsync(h.data(), active, (size_t)na * sizeof(Frozen), cudaMemcpyDeviceToHost, s.stream));
    CK(cudaStreamSynchronize(s.stream));
    for (int i = 0; i < na; i++) {
      const Frozen& f = h[i];
      int32_t* o = ids6 + (size_t)i * 6;
      o[0] = f.kind; o[1] = f.p; o[2] = f.a; o[3] = f.b; o[4] = f.c; o[5] = f.d;
      double* w = w7 + (size_t)i * 7;
      w[0] = f.w0; w[1] = f.w1; w[2] = f.w2; w[3] = f.w3; w[4] = f.nx; w[5] = f.ny; w[6] = f.nz;
    }
  }
  return na;
}

// ---- graph-captured step ------------------------------------------------------------
// The host-driven methods above read counts back to size launches and sorts and
// to grow buffers. Their captured counterparts below read every count on the
// device (acnt), size launches for capacities and report overflow in
// acnt[AC_ERR]; the solver then repeats the step on the host-driven path with
// grown buffers. Kernels and their arithmetic are the same, so a captured step
// computes what the host-driven one does.

__global__ void k_cap_begin(DevDiag* diag, int* acnt, int* actDirty) {
  DevDiag z{};
  z.minDistance = INFINITY;
  z.minTOI = INFINITY;
  *diag = z;
  for (int k = 0; k < AC_N; k++) acnt[k] = 0;
  *actDirty = 1;
}
__global__ void k_cap_set_flag(int* f, int v) { *f = v; }
__global__ void k_cap_act_decide(const int* actDirty, cudaGraphConditionalHandle h) {
  cudaGraphSetConditional(h, *actDirty ? 1u : 0u);
}
__global__ void k_cap_save_query(const int* cint, int* acnt) {
  acnt[AC_QSELF] = cint[CI_SELF];
  acnt[AC_QSTATIC] = cint[CI_STATIC];
}
// Superset sizes of a traversal into acnt, with the checks build_superset makes.
__global__ void k_cap_sup_counts(const int* cint, int* acnt, long supCap, long supSCap, long pairCap,
                                 long spairCap, long flagCap, int hasStatic) {
  const long P = (uint32_t)cint[CI_SELF], S = hasStatic ? (uint32_t)cint[CI_STATIC] : 0;
  acnt[AC_NSUP] = (int)min(P, supCap);
  acnt[AC_NSUPS] = (int)min(S, supSCap);
  if (cint[CI_OVERFLOW] || P > supCap || S > supSCap || P > pairCap || S > spairCap || 15 * P + 12 * S > flagCap)
    acnt[AC_ERR] |= ACE_CAPACITY;
}
__global__ void k_cap_cond_moved(const int* cint, cudaGraphConditionalHandle h) {
  cudaGraphSetConditional(h, cint[CI_MOVED] ? 1u : 0u);
}
// A query repeated on a superset rebuilt around it must be covered.
__global__ void k_cap_err_moved(const int* cint, int* acnt) {
  if (cint[CI_MOVED]) acnt[AC_ERR] |= ACE_SUPERSET;
}
// Frozen-set layout of the query just made (update_active_set's host reads).
__global__ void k_cap_active_counts(const int* cint, int* acnt, int candCap, int actCap) {
  const int nc = cint[CI_NCAND], nf = cint[CI_NFLOOR];
  if (nc > candCap || (long)nc + nf > actCap) acnt[AC_ERR] |= ACE_CAPACITY;
  const int c = min(nc, candCap), na = min(c + nf, actCap);
  acnt[AC_NCAND] = c;
  acnt[AC_NFLOOR] = na - c;
  acnt[AC_NVT] = cint[CI_NVT];
  acnt[AC_NA] = na;
  acnt[AC_NREC] = 4 * na;
}
// commit's host bookkeeping: the lag table grows by the candidates when there
// are any, the commit sequence advances when there is any contact.
__global__ void k_cap_lag_total(int* acnt) { acnt[AC_NTOT] = acnt[AC_LAG] + acnt[AC_NCAND]; }
// After a captured superset build: its counts and validity for later steps.
__global__ void k_cap_sup_save(const int* acnt, int* memo) {
  memo[0] = (acnt[AC_ERR] & ACE_CAPACITY) ? 0 : 1;
  memo[1] = acnt[AC_NSUP];
  memo[2] = acnt[AC_NSUPS];
}
// Step start of a captured step: rebuild the superset unless the saved one is
// valid and neither the step start nor the first iterate left its travel.
__global__ void k_cap_sup_decide(const int* cint, const int* memo, int* acnt, cudaGraphConditionalHandle h) {
  const bool rebuild = memo[0] != 1 || cint[CI_MOVED] != 0;
  if (!rebuild) {
    acnt[AC_NSUP] = memo[1];
    acnt[AC_NSUPS] = memo[2];
  }
  cudaGraphSetConditional(h, rebuild ? 1u : 0u);
}
// The vertex of record slot `slot` of a frozen contact (-1: unused), as k_csr_records.
__device__ __forceinline__ int slot_vertex(const Frozen& f, int slot) {
  if (f.kind == 2) return slot == 0 ? f.p : -1;
  if (f.kind == 0) return slot == 0 ? f.p : slot == 1 ? f.a : slot == 2 ? f.b : f.c;
  return slot == 0 ? f.a : slot == 1 ? f.b : slot == 2 ? f.c : f.d;
}
__global__ void k_cap_csr_same(CView v, const int* ids, int* memo, const int* acnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int na = acnt[AC_NA];
  if (i >= na || memo[0] != na) return;  // a different count is decided below
  const Frozen f = v.active[i];
  const int* q = ids + (size_t)i * 5;
  bool same = q[0] == f.kind;
#pragma unroll
  for (int sl = 0; sl < 4; sl++) same = same && q[1 + sl] == slot_vertex(f, sl);
  if (!same) atomicOr(memo + 1, 1);
}
__global__ void k_cap_csr_decide(int* memo, const int* acnt, cudaGraphConditionalHandle h) {
  const bool rebuild = memo[1] != 0 || memo[0] != acnt[AC_NA];
  memo[1] = 0;
  cudaGraphSetConditional(h, rebuild ? 1u : 0u);
}
__global__ void k_cap_csr_save(CView v, int* ids, int* memo, const int* acnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int na = acnt[AC_NA];
  if (i == 0) memo[0] = na;
  if (i >= na) return;
  const Frozen f = v.active[i];
  int* q = ids + (size_t)i * 5;
  q[0] = f.kind;
#pragma unroll
  for (int sl = 0; sl < 4; sl++) q[1 + sl] = slot_vertex(f, sl);
}
__global__ void k_cap_lag_advance(int* acnt, int lagCap) {
  if (acnt[AC_NCAND] > 0) {
    if (acnt[AC_NTOT] > lagCap) acnt[AC_ERR] |= ACE_CAPACITY;
    else acnt[AC_LAG] = acnt[AC_NTOT];
  }
  if (acnt[AC_NA] > 0) acnt[AC_COMMIT] += 1;
}
__global__ void k_cap_copy_vals(double4* dst, const double4* src, int cap, const int* dn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < min(cap, *dn)) dst[i] = src[i];
}

void ContactHost::cap_bind(Solver& s) {
  bind(s);
  Contact& c = s.d.c;
  c.nActive = (int)actCap;      // launch sizes
  c.nActiveD = acnt + AC_NA;    // the count kernels use
}

int ContactHost::cand_blocks_cap() const {
  const long bound = 15l * (long)supCap + 12l * (long)(ms > 0 ? supSCap : 0);
  return (int)std::max(1l, std::min((bound + kCT - 1) / kCT, 8l * smCount));
}

void ContactHost::cap_begin_step(Solver& s, GraphCtx& g) {
  cudaStream_t st = g.cur();
  k_cap_begin<<<1, 1, 0, st>>>(diag, acnt, actDirty);
  CK(cudaMemsetAsync(lagFloorOk, 0, (size_t)n, st));
  launch_counter()++;
  fricOn = false;
  cap_bind(s);
}

void ContactHost::cap_superset(Solver& s, GraphCtx& g, const double* x) {
  cudaStream_t st = g.cur();
  int64_t& lc = launch_counter();
  const double padSup = sup_pad();
  CK(cudaMemcpyAsync(supBase, x, 3 * (size_t)n * 8, cudaMemcpyDeviceToDevice, st));
  bvh_build(bvh, s.d.x0, x, padSup, false, st, &lc);
  CK(cudaMemsetAsync(cint, 0, CI_N * sizeof(int), st));
  BvhBufs sb = bvh;
  sb.cnt = (uint32_t*)(cint + CI_SELF);
  sb.pairs = supPairs;
  sb.pairCap = (uint32_t)supCap;
  bvh_append_self(sb, st, &lc);
  if (ms > 0) bvh_append_static(bvh, padSup, supSPairs, (uint32_t)supSCap, (uint32_t*)(cint + CI_STATIC), st, &lc);
  k_cap_sup_counts<<<1, 1, 0, st>>>(cint, acnt, (long)supCap, (long)supSCap, (long)pairCap, (long)spairCap,
                                    (long)flagCap, ms > 0 ? 1 : 0);
  k_cap_sup_save<<<1, 1, 0, st>>>(acnt, supMemo);
  lc += 2;
}

// A superset swept x0 -> base with the pad widened by kSupTravel contains every
// pair of a later query swept x0' -> x' when x0' and x' both stay within
// kSupTravel (max norm) of base, whatever step the query belongs to. So a
// captured step reuses the previous step's superset when its start x0 and its
// first iterate x pass that test, and rebuilds it around x otherwise.
void ContactHost::cap_superset_step(Solver& s, GraphCtx& g, const double* x) {
  int64_t& lc = launch_counter();
  cudaStream_t st = g.cur();
  const int n3 = 3 * n;
  CK(cudaMemsetAsync(cint, 0, CI_N * sizeof(int), st));
  k_moved<<<std::min(1184, (n3 + 255) / 256), 256, 0, st>>>(s.d.x0, supBase, n3, kSupTravel, cint);
  k_moved<<<std::min(1184, (n3 + 255) / 256), 256, 0, st>>>(x, supBase, n3, kSupTravel, cint);
  const cudaGraphConditionalHandle h = g.handle(1);
  k_cap_sup_decide<<<1, 1, 0, st>>>(cint, supMemo, acnt, h);
  lc += 3;
  g.push(h, cudaGraphCondTypeIf);
  cap_superset(s, g, x);
  g.pop();
}

// launch_query, then (conditional node) the superset rebuilt around x and the
// query repeated when x left the superset's 4 mm travel.
void ContactHost::cap_query(Solver& s, GraphCtx& g, const double* x, double pad) {
  int64_t& lc = launch_counter();
  auto query = [&](cudaStream_t st) {
    CK(cudaMemsetAsync(cint, 0, CI_N * sizeof(int), st));
    const int n3 = 3 * n;
    k_moved<<<std::min(1184, (n3 + 255) / 256), 256, 0, st>>>(x, supBase, n3, kSupTravel, cint);
    bvh_boxes(bvh, s.d.x0, x, pad, st, &lc);
    filter_pairs_dev(bvh, supPairs, (int)supCap, bvh.pairs, (uint32_t)pairCap, (uint32_t*)(cint + CI_SELF), supSPairs,
                     ms > 0 ? (int)supSCap : 0, pad, spairs, (uint32_t)spairCap, (uint32_t*)(cint + CI_STATIC),
                     acnt + AC_NSUP, st, &lc);
    lc++;
  };
  query(g.cur());
  const cudaGraphConditionalHandle h = g.handle(0);
  k_cap_cond_moved<<<1, 1, 0, g.cur()>>>(cint, h);
  lc++;
  g.push(h, cudaGraphCondTypeIf);
  cap_superset(s, g, x);
  query(g.cur());
  k_cap_err_moved<<<1, 1, 0, g.cur()>>>(cint, acnt);
  lc++;
  g.pop();
}

void ContactHost::cap_mark_moved(GraphCtx& g) {
  k_cap_set_flag<<<1, 1, 0, g.cur()>>>(actDirty, 1);
  launch_counter()++;
}

// The active set at x, as update_active_set. Positions that did not change
// since the last update (the first Newton iteration after the step start's
// update, the restitution pass after a converged Newton check) give the same
// active set, CSR and diagnostics, so the update runs in an IF node on actDirty.
void ContactHost::cap_update_active_set(Solver& s, GraphCtx& g, const double* x) {
  int64_t& lc = launch_counter();
  const cudaGraphConditionalHandle hAct = g.handle(1);
  k_cap_act_decide<<<1, 1, 0, g.cur()>>>(actDirty, hAct);
  lc++;
  g.push(hAct, cudaGraphCondTypeIf);
  cap_update_active_set_body(s, g, x);
  k_cap_set_flag<<<1, 1, 0, g.cur()>>>(actDirty, 0);
  lc++;
  g.pop();
  cap_bind(s);
}

void ContactHost::cap_update_active_set_body(Solver& s, GraphCtx& g, const double* x) {
  cap_query(s, g, x, p.dhat);
  cudaStream_t st = g.cur();
  int64_t& lc = launch_counter();
  k_cap_save_query<<<1, 1, 0, st>>>(cint, acnt);
  lc++;
  CView v = cview(*this, s);
  k_active_reset<<<1, 1, 0, st>>>(v);
  k_cand_flags<<<cand_blocks_cap(), kCT, 0, st>>>(v, x, cand.cap, cand.k0, cand.p0);
  k_floor_flags<<<cnb(n), kCT, 0, st>>>(v, x);
  k_active_min<<<1, 1, 0, st>>>(v);
  lc += 4;
  scan_counts(fflag, n, (uint32_t*)(cint + CI_NFLOOR), st, &lc);
  k_cap_active_counts<<<1, 1, 0, st>>>(cint, acnt, cand.cap, (int)actCap);
  lc++;
  const bool flip = radix_sort_dev<4>(cand.k0, cand.p0, cand.k1, cand.p1, acnt + AC_NCAND, cand.cap,
                                      cand_key_bits(idBits, 0), cand.hist, st, &lc);
  k_cand_active<<<cnb(cand.cap), kCT, 0, st>>>(v, x, flip ? cand.p1 : cand.p0, -1);
  k_floor_compact<<<cnb(n), kCT, 0, st>>>(v, x);
  lc += 2;
  // the vertex -> record CSR depends only on each contact's kind and slot
  // vertices: rebuild it only when those changed since the last build (a
  // sheet at rest keeps the same floor contacts step after step)
  k_cap_csr_same<<<cnb((long)actCap), kCT, 0, st>>>(v, csrIds, csrMemo, acnt);
  const cudaGraphConditionalHandle h = g.handle(1);
  k_cap_csr_decide<<<1, 1, 0, st>>>(csrMemo, acnt, h);
  lc += 2;
  g.push(h, cudaGraphCondTypeIf);
  {
    cudaStream_t sb = g.cur();
    k_csr_records<<<cnb(4l * (long)actCap), kCT, 0, sb>>>(v, rk0, rp0, -1);
    lc++;
    // 32-bit keys: an even number of passes leaves the result in (rk0, rp0)
    radix_sort_dev<1>(rk0, rp0, rk1, rp1, acnt + AC_NREC, 4 * (int)actCap, 32, rhist, sb, &lc);
    k_csr_offsets<<<cnb(n + 1), kCT, 0, sb>>>(rk0, 0, cOff, n, acnt + AC_NA);
    k_cap_csr_save<<<cnb((long)actCap), kCT, 0, sb>>>(v, csrIds, csrMemo, acnt);
    lc += 2;
  }
  g.pop();
}

void ContactHost::cap_gradient_terms(Solver& s, GraphCtx& g) {
  cap_update_active_set(s, g, s.d.x);
  cudaStream_t st = g.cur();
  CView v = cview(*this, s);
  const long cap = (long)actCap;
  k_contact_prep<<<cnb(cap), kCT, 0, st>>>(v, s.d.x, -1);
  k_contact_chains<<<1, s.mixed() ? 1024 : 64, 0, st>>>(v, -1, s.mixed() ? 1 : 0);
  k_contact_grad_rec<<<cnb(4 * cap), kCT, 0, st>>>(v, (int)(4 * cap));
  k_contact_grad_gather<<<cnb(n), kCT, 0, st>>>(v, s.d.cgrad);
  k_contact_curv<<<cnb(cap), kCT, 0, st>>>(v, s.d.x, -1);
  k_contact_diag_rec<<<cnb(4 * cap), kCT, 0, st>>>(v, (int)(4 * cap));
  k_contact_diag_gather<<<cnb(n), kCT, 0, st>>>(v, s.d.diag);
  launch_counter() += 7;
}

void ContactHost::cap_friction_terms(Solver& s, GraphCtx& g) {
  fricOn = true;
  cap_bind(s);
  CView v = cview(*this, s);
  k_contact_fric<<<cnb((long)actCap), kCT, 0, g.cur()>>>(v, s.d.x, -1, fh);
  launch_counter()++;
}

void ContactHost::cap_merit_energy(Solver& s, GraphCtx& g, const double* x) {
  CView v = cview(*this, s);
  k_contact_merit<<<cnb((long)actCap), kCT, 0, g.cur()>>>(v, x, -1);
  launch_counter()++;
}

void ContactHost::cap_trial(Solver& s, GraphCtx& g, const double* xt) {
  cap_query(s, g, xt, p.dmin);
  cudaStream_t st = g.cur();
  CView v = cview(*this, s);
  k_trial_reset<<<1, 1, 0, st>>>(v);
  k_trial_cand<<<cand_blocks_cap(), kCT, 0, st>>>(v, xt, p.dmin);
  k_trial_bad_lo<<<4 * smCount, kCT, 0, st>>>(v);
  k_trial_floor<<<cnb(n), kCT, 0, st>>>(v, xt, p.dmin);
  k_trial_final<<<1, 1, 0, st>>>(v, p.dmin);
  launch_counter() += 5;
}

void ContactHost::cap_commit(Solver& s, GraphCtx& g, const double* x) {
  cudaStream_t st = g.cur();
  int64_t& lc = launch_counter();
  const int lagSort = (int)std::min<size_t>(lagCap, kBlockSortMax);
  CView v = cview(*this, s);
  // the sorted prefix becomes entries 0..lagCount-1 with their values in place
  k_cap_copy_vals<<<cnb(lagSort), kCT, 0, st>>>(lval, lsorted, lagSort, acnt + AC_LAG);
  k_iota<<<cnb(lagSort), kCT, 0, st>>>(lp0, lagSort, acnt + AC_LAG);
  k_contact_commit<<<cnb((long)actCap), kCT, 0, st>>>(v, x, -1, lk0, lp0, lval, 0, 0);
  k_cap_lag_total<<<1, 1, 0, st>>>(acnt);
  lc += 4;
  // one-block sort (192-bit keys, an even number of passes: the result stays in
  // (lk0, lp0)); a table past its capacity is reported, not sorted
  radix_sort_dev<6>(lk0, lp0, lk1, lp1, acnt + AC_NTOT, lagSort, 192, lhist, st, &lc);
  k_gather_vals<<<cnb(lagSort), kCT, 0, st>>>(lval, lp0, lagSort, lsorted, acnt + AC_NTOT);
  k_cap_lag_advance<<<1, 1, 0, st>>>(acnt, lagSort);
  lc += 2;
}

void ContactHost::cap_kill_approach_velocity(Solver& s, GraphCtx& g) {
  cap_update_active_set(s, g, s.d.x);
  cudaStream_t st = g.cur();
  CView v = cview(*this, s);
  const long cap = (long)actCap;
  k_kill_pred<<<cnb(4 * cap), kCT, 0, st>>>(v, rk0, rp0, cOff, (int)(4 * cap), (int)cap, kpred);
  k_kill_vtee_rounds<<<1, kKillThreads, 48 * 1024, st>>>(v, s.d.v, (int)cap, kpred);
  k_kill_vtee<<<1, 1, 0, st>>>(v, s.d.v, (int)cap);
  k_kill_floor<<<cnb(cap), kCT, 0, st>>>(v, s.d.v, 0, (int)cap);
  launch_counter() += 4;
}

void ContactHost::cap_collect(const int* ha, const int* hc, double rejectionsDev) {
  nCand = ha[AC_NCAND];
  nFloor = ha[AC_NFLOOR];
  nVT = ha[AC_NVT];
  lagCount = ha[AC_LAG];
  commitNo = ha[AC_COMMIT];
  nSup = ha[AC_NSUP];
  nSupS = ha[AC_NSUPS];
  candidatePairs = 15.0 * (uint32_t)ha[AC_QSELF] + 12.0 * (uint32_t)(ms > 0 ? ha[AC_QSTATIC] : 0);
  (void)hc;
  activePairs = nCand + nFloor;
  vtPairs = nVT;
  eePairs = nCand - nVT;
  floorPairs = nFloor;
  rejections = rejectionsDev;
  supValid = false;  // the next host-driven query rebuilds the superset
}

void ContactHost::cap_grow(Solver& s, const int* ha, const int* hc) {
  (void)ha;
  (void)hc;
  // Counts past a capacity were clamped on the device, so grow by doubling;
  // the host-driven repeat of the step grows further as it needs.
  ensure_cands(2 * (size_t)cand.cap);
  ensure_active(s, 2 * actCap);
  ensure_lag(2 * lagCap);
  ensure_pairs(2 * pairCap, 2 * spairCap);
  ensure_flags(2 * flagCap);
  supCap = 2 * supCap;
  dalloc(supPairs, supCap);
  if (ms > 0) {
    supSCap = 2 * supSCap;
    dalloc(supSPairs, supSCap);
  }
  supValid = false;
  CK(cudaMemsetAsync(supMemo, 0, sizeof(int), s.stream));
}

void set_contact(Solver& s, const cs_contact_params* p, int floor_on, double floor_y, const float* sp, int ns,
                 const uint32_t* si, int ms) {
  if (!p) {
    s.contact.reset();
    s.d.hasContact = 0;
    s.initEpoch++;
    return;
  }
  if (!(p->dhat > 0) || !(p->dmin >= 0) || !(p->kappa >= 0) || !(p->eps > 0) || !(p->mu >= 0))
    throw std::invalid_argument("bad contact parameters");
  if ((ns > 0) != (ms > 0) || (ms > 0 && (!sp || !si))) throw std::invalid_argument("bad static mesh");
  auto c = std::make_unique<ContactHost>();
  c->init(s, p, floor_on, floor_y, sp, ns, si, ms);
  s.contact = std::move(c);
  s.initEpoch++;
}

}  // namespace cs
