// Mixed-precision PCG (pcg.ts:11-95 + the newton.ts:152-179 epilogue) run by
// ONE thread-block cluster: up to 16 CTAs on one GPC, synchronized with the
// hardware cluster barrier and reducing through distributed shared memory.
// For sheets that fit a cluster this replaces a grid-wide barrier (a round
// trip through L2 and every SM) with an on-GPC one, and fuses each iteration
// into two phases:
//
//   A  per vertex (T lanes splitting its incident triangles): p_k = z + beta
//      p_{k-1} formed on the fly for the vertex and its element neighbours,
//      the membrane HVP of every incident triangle (corner share only) from the
//      stored FP32 (F, S), the frozen-contact HVP, Ap = M/h^2 p + H p; partial
//      p.Ap                                            -- cluster barrier --
//   B  per Schwarz domain (one warp, lane = local dof, up to three domains
//      per warp in flight together) or per dof (Jacobi):
//      alpha, x += alpha p, r -= alpha Ap, z = M^-1 r; partial r.r and r.z
//                                                      -- cluster barrier --
//
// Every dot product accumulates in FP64; each CTA's partial is read by every
// CTA in rank order, so all CTAs take the same branch and the result does not
// depend on timing. Compiled with FMA contraction on.
//
// Resident phase A (ClPlan.resident, when the CTA's lists fit in shared
// memory): each CTA copies its triangles' records, hinges' Gauss-Newton
// factors and owned vertices' incidence lists into shared memory once per
// launch. An iteration then stages p on the CTA's halo (one global load per
// halo vertex), computes every listed triangle's HVP (g1, g2) and hinge's
// g . p from shared memory, and sums them per owned vertex in incidence order.
// Without it phase A gathers vertex-major records from global memory, a chain
// of dependent loads per incidence.
#include <cooperative_groups.h>

#include <mutex>

#include "cluster_plan.hpp"
#include "contact.cuh"
#include "hvp32.cuh"
#include "mixed.cuh"

namespace cg = cooperative_groups;

namespace cs {

constexpr int kClT = 512;
static_assert(kClT == 32 * kClWarps, "the per-CTA lists assume kClWarps warps per CTA");

struct ClArgs {
  Dev d;
  MixBufs mb;
  float* pA;      // search direction, double-buffered (3n each)
  float* pB;
  double* coef;   // per active contact: barrier curvature at the frozen distance (0 outside dHat)
  int maxIters;
  double tol;
  ClPlan plan;
};

// Partial sums of one reduction, one row per source CTA: every CTA pushes its
// row into every peer's copy before the cluster barrier, so after it each CTA
// reads only its own shared memory.
typedef double RedBank[16][4];

// Cluster-wide totals of K partials from the local bank: in every warp, lane r
// reads CTA r's row and a fixed shuffle tree adds the rows, so every warp of
// every CTA holds identical bits without a block barrier. The bank is
// rewritten only after the next cluster barrier, which no thread passes
// before its own read.
template <int K>
__device__ __forceinline__ void cl_totals(const RedBank& bank, int nrank, double* out) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < K; k++) {
    double s = lane < nrank ? bank[lane][k] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    out[k] = __shfl_sync(0xffffffffu, s, 0);
  }
}

// This CTA's sums of K per-thread values, pushed as row `rank` of every peer's
// bank (lane q of warp 0 stores into CTA q): warp shuffle trees, one block
// barrier, warp 0 adds the warp partials in a fixed order. wsm holds K x 32
// doubles; it is rewritten only after the next cluster barrier, by which time
// warp 0 has read it. A bank is rewritten only after the cluster barrier that
// follows every CTA's read of it (banks alternate between reductions).
template <int K>
__device__ __forceinline__ void block_partials(cg::cluster_group& cl, const double* v, RedBank& bank, int rank,
                                               int nrank, double* wsm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; k++) {
    double w = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
    if (lane == 0) wsm[k * 32 + warp] = w;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    double t[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      double a = lane < nw ? wsm[k * 32 + lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
      t[k] = __shfl_sync(0xffffffffu, a, 0);
    }
    if (lane < nrank) {
      double* dst = cl.map_shared_rank(&bank[rank][0], lane);
#pragma unroll
      for (int k = 0; k < K; k++) dst[k] = t[k];
    }
  }
}

__device__ __forceinline__ float3 ld_p(const float* z, const float* pc, float beta, bool first, int v) {
  const float z0 = z[v * 3], z1 = z[v * 3 + 1], z2 = z[v * 3 + 2];
  if (first) return make_float3(z0, z1, z2);
  return make_float3(__fmaf_rn(beta, pc[v * 3], z0), __fmaf_rn(beta, pc[v * 3 + 1], z1),
                     __fmaf_rn(beta, pc[v * 3 + 2], z2));
}

// Jacobian of the frozen distance along the current direction (distJvp,
// contact-assembly.ts:394-414), with p formed on the fly. FP64.
__device__ __forceinline__ double cl_jvp(const Frozen& f, const float* z, const float* pc, float beta, bool first) {
  if (f.kind == 2) return (double)ld_p(z, pc, beta, first, f.p).y;
  const int vs[4] = {f.kind == 0 ? f.p : f.a, f.kind == 0 ? f.a : f.b, f.kind == 0 ? f.b : f.c,
                     f.kind == 0 ? f.c : f.d};
  double nv[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    nv[q] = 0;
    if (vs[q] >= 0) {
      const float3 pv = ld_p(z, pc, beta, first, vs[q]);
      nv[q] = f.nx * (double)pv.x + f.ny * (double)pv.y + f.nz * (double)pv.z;
    }
  }
  if (f.kind == 0) return nv[0] - f.w0 * nv[1] - f.w1 * nv[2] - f.w2 * nv[3];
  return f.w0 * nv[0] + f.w1 * nv[1] + f.w2 * nv[2] + f.w3 * nv[3];
}

// Relative-slip Jacobian along the current direction (slip_jvp with p formed
// on the fly), for the exact-Newton friction term. FP64.
__device__ __forceinline__ void cl_slip_jvp(const Frozen& f, const float* z, const float* pc, float beta, bool first,
                                            double o[3]) {
  o[0] = o[1] = o[2] = 0;
  auto V = [&](int q, double s) {
    if (q < 0) return;
    const float3 pv = ld_p(z, pc, beta, first, q);
    o[0] += s * (double)pv.x; o[1] += s * (double)pv.y; o[2] += s * (double)pv.z;
  };
  if (f.kind == 2) { V(f.p, 1.0); return; }
  if (f.kind == 0) { V(f.p, 1.0); V(f.a, -f.w0); V(f.b, -f.w1); return; }
  V(f.a, f.w0); V(f.b, f.w1); V(f.c, f.w2); V(f.d, f.w3);
}

// Frozen-contact shares of the contact records [r0, r1) (vertex-major, one
// record per thread: a vertex may sit in many contacts), written to the record
// scratch and summed per vertex later in record order.
//
// Resident kernel: the first `cap` records' ids come from recS (copied at
// launch) and their shares go to shareS (shared memory, FP64, 3 per record);
// records beyond cap use the global record list and scratch.
__device__ __forceinline__ void cl_contact_records(const Dev& d, const MixBufs& mb, const double* coef,
                                                   const float* pc, float beta, bool first, uint32_t r0,
                                                   uint32_t r1, const uint32_t* recS = nullptr,
                                                   double* shareS = nullptr, uint32_t cap = 0) {
  const Contact& c = d.c;
  for (uint32_t q = r0 + threadIdx.x; q < r1; q += blockDim.x) {
    const bool onChip = q - r0 < cap;
    const uint32_t rec = onChip ? recS[q - r0] : c.cRec[q];
    const double g = coef[rec >> 2];
    double ch[3] = {0, 0, 0};
    if (g != 0) {
      const Frozen f = c.active[rec >> 2];
      dist_grad_slot(f, rec & 3, g * cl_jvp(f, mb.z, pc, beta, first), ch);
    }
    if (c.fric) {  // exact-Newton mode: friction potential Hessian
      const double* fh = c.fh + (size_t)(rec >> 2) * 8;
      if (fh[1] != 0) {
        const Frozen f = c.active[rec >> 2];
        double du[3], F[3];
        cl_slip_jvp(f, mb.z, pc, beta, first, du);
        fric_hess_apply(fh, du, F);
        slip_jt_slot(f, rec & 3, F, ch);
      }
    }
    double* o = onChip ? shareS + (size_t)(q - r0) * 3 : c.recScratch + (size_t)q * 3;
    o[0] = ch[0]; o[1] = ch[1]; o[2] = ch[2];
  }
}

// Loop-invariant facts of a warp's (up to 3) Schwarz domains dom0 + u * step,
// read once per launch: gi[u] = this lane's dof (-1: none); meta bit u = the
// dof is pinned, bits 8 + 4u .. = the domain's vertex count (0: no domain).
struct DomFacts {
  int gi[3];
  int meta;
};

__device__ __forceinline__ DomFacts cl_domain_facts(const Dev& d, int dom0, int step) {
  const int lane = threadIdx.x & 31;
  DomFacts f;
  f.meta = 0;
#pragma unroll
  for (int u = 0; u < 3; u++) {
    f.gi[u] = -1;
    const int dom = dom0 + u * step;
    if (dom < d.D) {
      const int start = d.domStart[dom], dv = d.domStart[dom + 1] - start;
      f.meta |= dv << (8 + 4 * u);
      if (lane < dv * 3) {
        const int gi = d.domVerts[start + lane / 3] * 3 + lane % 3;
        f.gi[u] = gi;
        if (d.pinned[gi / 3]) f.meta |= 1 << u;
      }
    }
  }
  return f;
}

// Resident kernel's contact records, in FP32 like the rest of the operator:
// everything a record reads from global memory (its frozen contact's ids,
// weights and normal, the barrier curvature and the friction terms) is issued
// at once, then the p of its stencil, from the halo when the vertex is owned by
// this CTA (always, for floor contacts) and from global memory otherwise. The
// terms are cl_contact_records' (dist_grad_slot, slip_jvp, fric_hess_apply,
// slip_jt_slot) on the same p values. On-chip shares are FP32 (shareS);
// records beyond cap go to the global scratch as FP64.
__device__ __forceinline__ void cl_contact_records_res(const Dev& d, const MixBufs& mb, const double* coef,
                                                       const float* pc, float beta, bool first, uint32_t r0,
                                                       uint32_t r1, const uint32_t* recS, float* shareS, uint32_t cap,
                                                       const float4* pH, const int* ownHS, int vb0, int nOwn) {
  const Contact& c = d.c;
  for (uint32_t q = r0 + threadIdx.x; q < r1; q += blockDim.x) {
    const bool onChip = q - r0 < cap;
    const uint32_t rec = onChip ? recS[q - r0] : c.cRec[q];
    const int ci = (int)(rec >> 2), slot = (int)(rec & 3);
    const Frozen* fr = c.active + ci;
    const int kind = fr->kind;
    // stencil: kind 0 (p, a, b, c), kind 1 (a, b, c, d), kind 2 (p)
    const int vs[4] = {kind == 1 ? fr->a : fr->p, kind == 1 ? fr->b : fr->a, kind == 1 ? fr->c : fr->b,
                       kind == 1 ? fr->d : fr->c};
    const float w[4] = {(float)fr->w0, (float)fr->w1, (float)fr->w2, (float)fr->w3};
    const float nx = (float)fr->nx, ny = (float)fr->ny, nz = (float)fr->nz;
    const float g = (float)coef[ci];
    float fs = 0.f, ft[3] = {0.f, 0.f, 0.f}, fn[3] = {0.f, 0.f, 0.f};
    if (c.fric) {
      const double* h = c.fh + (size_t)ci * 8;
      fs = (float)h[1];
      ft[0] = (float)h[2]; ft[1] = (float)h[3]; ft[2] = (float)h[4];
      fn[0] = (float)h[5]; fn[1] = (float)h[6]; fn[2] = (float)h[7];
    }
    float3 P[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      P[k] = make_float3(0.f, 0.f, 0.f);
      const int v = vs[k];
      if (v < 0 || (kind == 2 && k > 0)) continue;
      const int lv = v - vb0;
      if (lv >= 0 && lv < nOwn) {
        const float4 t = pH[ownHS[lv]];
        P[k] = make_float3(t.x, t.y, t.z);
      } else {
        P[k] = ld_p(mb.z, pc, beta, first, v);
      }
    }
    float ch[3] = {0.f, 0.f, 0.f};
    if (g != 0.f) {
      float jvp;
      if (kind == 2) {
        jvp = P[0].y;
      } else {
        float nv[4];
#pragma unroll
        for (int k = 0; k < 4; k++) nv[k] = nx * P[k].x + ny * P[k].y + nz * P[k].z;
        jvp = kind == 0 ? nv[0] - w[0] * nv[1] - w[1] * nv[2] - w[2] * nv[3]
                        : w[0] * nv[0] + w[1] * nv[1] + w[2] * nv[2] + w[3] * nv[3];
      }
      const float gj = g * jvp;
      if (kind == 2) {
        ch[1] += gj;
      } else {
        // dist_grad_slot: slot weight times the normal
        const float ws = kind == 0 ? (slot == 0 ? 1.f : -(slot == 1 ? w[0] : slot == 2 ? w[1] : w[2]))
                                   : (slot == 0 ? w[0] : slot == 1 ? w[1] : slot == 2 ? w[2] : w[3]);
        ch[0] += gj * ws * nx; ch[1] += gj * ws * ny; ch[2] += gj * ws * nz;
      }
    }
    if (fs != 0.f) {  // exact-Newton mode: friction potential Hessian (slip_jvp, fric_hess_apply)
      float du[3];
      if (kind == 2) {
        du[0] = P[0].x; du[1] = P[0].y; du[2] = P[0].z;
      } else if (kind == 0) {
        du[0] = P[0].x - w[0] * P[1].x - w[1] * P[2].x;
        du[1] = P[0].y - w[0] * P[1].y - w[1] * P[2].y;
        du[2] = P[0].z - w[0] * P[1].z - w[1] * P[2].z;
      } else {
        du[0] = w[0] * P[0].x + w[1] * P[1].x + w[2] * P[2].x + w[3] * P[3].x;
        du[1] = w[0] * P[0].y + w[1] * P[1].y + w[2] * P[2].y + w[3] * P[3].y;
        du[2] = w[0] * P[0].z + w[1] * P[1].z + w[2] * P[2].z + w[3] * P[3].z;
      }
      const float nd = fn[0] * du[0] + fn[1] * du[1] + fn[2] * du[2];
      const float pu[3] = {du[0] - nd * fn[0], du[1] - nd * fn[1], du[2] - nd * fn[2]};
      const float td = ft[0] * pu[0] + ft[1] * pu[1] + ft[2] * pu[2];
      // slip_jt_slot weight of this slot
      const float wj = kind == 2 ? (slot == 0 ? 1.f : 0.f)
                       : kind == 0 ? (slot == 0 ? 1.f : slot == 1 ? -w[0] : slot == 2 ? -w[1] : 0.f)
                                   : (slot == 0 ? w[0] : slot == 1 ? w[1] : slot == 2 ? w[2] : w[3]);
#pragma unroll
      for (int k = 0; k < 3; k++) ch[k] += wj * (fs * (pu[k] - td * ft[k]));
    }
    if (onChip) {
      float* o = shareS + (size_t)(q - r0) * 3;
      o[0] = ch[0]; o[1] = ch[1]; o[2] = ch[2];
    } else {
      double* o = c.recScratch + (size_t)q * 3;
      o[0] = ch[0]; o[1] = ch[1]; o[2] = ch[2];
    }
  }
}

// Phase B on K Schwarz domains dom0, dom0 + step, ... at once (one warp, lane =
// local dof): the loads of all K are issued before any product, so their
// latencies overlap. Adds the (r.r, r.z) shares.
template <int K>
__device__ __forceinline__ void cl_domains(const Dev& d, const MixBufs& mb, const float* pn, float alpha, bool init,
                                           int dom0, int step, const DomFacts& f, double& rr, double& rz) {
  const int lane = threadIdx.x & 31;
  float rv[K];
#pragma unroll
  for (int u = 0; u < K; u++) {
    rv[u] = 0.f;
    const int gi = f.gi[u];
    if (gi >= 0) {
      float xi, ri;
      if (init) {
        xi = 0.f;
        ri = (float)(-d.g[gi]);
      } else {
        xi = mb.x[gi] + alpha * pn[gi];
        ri = mb.r[gi] - alpha * mb.Ap[gi];
      }
      if ((f.meta >> u) & 1) { xi = 0.f; ri = 0.f; }
      mb.x[gi] = xi;
      mb.r[gi] = ri;
      rv[u] = ri;
      rr += (double)ri * ri;
    }
  }
  // row `lane` of each 24x24 inverse: 96 bytes, in two halves of three 16-byte
  // loads (all K domains' halves in flight together)
  float zk[K];
#pragma unroll
  for (int u = 0; u < K; u++) zk[u] = 0.f;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    float4 L[K][3];
#pragma unroll
    for (int u = 0; u < K; u++) {
      const float4* Li = reinterpret_cast<const float4*>(mb.Linv + (size_t)(dom0 + u * step) * 576) + lane * 6 + h * 3;
#pragma unroll
      for (int j4 = 0; j4 < 3; j4++) L[u][j4] = f.gi[u] >= 0 ? __ldg(Li + j4) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < K; u++) {
#pragma unroll
      for (int j4 = 0; j4 < 3; j4++) {
        const int c = 4 * (h * 3 + j4);
        zk[u] = fmaf(L[u][j4].x, __shfl_sync(0xffffffffu, rv[u], c), zk[u]);
        zk[u] = fmaf(L[u][j4].y, __shfl_sync(0xffffffffu, rv[u], c + 1), zk[u]);
        zk[u] = fmaf(L[u][j4].z, __shfl_sync(0xffffffffu, rv[u], c + 2), zk[u]);
        zk[u] = fmaf(L[u][j4].w, __shfl_sync(0xffffffffu, rv[u], c + 3), zk[u]);
      }
    }
  }
#pragma unroll
  for (int u = 0; u < K; u++) {
    float z = zk[u];
    const int dv = (f.meta >> (8 + 4 * u)) & 15;
    if (mb.dcoarse && dv > 0) z += coarse_share(mb, dom0 + u * step, rv[u], dv);
    if (f.gi[u] >= 0) {
      if ((f.meta >> u) & 1) z = 0.f;
      mb.z[f.gi[u]] = z;
      rz += (double)rv[u] * z;
    }
  }
}

// Phase B over every domain, K = ceil(D / warps) per warp at once. Up to three
// domains per warp use the facts read at launch (f, for dom0 = gwarp); more
// re-read them per pass.
__device__ __forceinline__ void cl_all_domains(const Dev& d, const MixBufs& mb, const float* pn, float alpha,
                                               bool init, int gwarp, int nwarps, const DomFacts& f, double& rr,
                                               double& rz) {
  const int per = (d.D + nwarps - 1) / nwarps;
  if (per <= 1) {
    if (gwarp < d.D) cl_domains<1>(d, mb, pn, alpha, init, gwarp, nwarps, f, rr, rz);
  } else if (per == 2) {
    cl_domains<2>(d, mb, pn, alpha, init, gwarp, nwarps, f, rr, rz);
  } else if (per == 3) {
    cl_domains<3>(d, mb, pn, alpha, init, gwarp, nwarps, f, rr, rz);
  } else {
    for (int dom = gwarp; dom < d.D; dom += 3 * nwarps)
      cl_domains<3>(d, mb, pn, alpha, init, dom, nwarps, cl_domain_facts(d, dom, nwarps), rr, rz);
  }
}

// Resident phase B on the warp's (up to 3) domain slots u * W + wl: (Ap, p)
// pushed by the vertex owners and this lane's (x, r) are read from the slot's
// dof record, z = A_d^-1 r from the slot's packed symmetric inverse in shared
// memory (lane i reads row i). Only z goes to global memory (the next
// iteration's halos read it).
template <int K>
__device__ __forceinline__ void cl_res_domains_k(const Dev& d, const MixBufs& mb, float4* bufB, const float* Lp,
                                                 float alpha, bool init, int wl, int W, int gwarp, int nwarps,
                                                 const DomFacts& f, double& rr, double& rz) {
  const int lane = threadIdx.x & 31;
  float rv[K];
#pragma unroll
  for (int u = 0; u < K; u++) {
    rv[u] = 0.f;
    const int gi = f.gi[u];
    if (gi >= 0) {
      float4* rec = bufB + (u * W + wl) * 24 + lane;
      float xi, ri;
      if (init) {
        xi = 0.f;
        ri = (float)(-d.g[gi]);
      } else {
        const float4 b = *rec;  // (Ap, p, x, r)
        xi = b.z + alpha * b.y;
        ri = b.w - alpha * b.x;
      }
      if ((f.meta >> u) & 1) { xi = 0.f; ri = 0.f; }
      *(reinterpret_cast<float2*>(rec) + 1) = make_float2(xi, ri);
      rv[u] = ri;
      rr += (double)ri * ri;
    }
  }
  const int ii = min(lane, 23);
#pragma unroll
  for (int u = 0; u < K; u++) {
    const int dv = (f.meta >> (8 + 4 * u)) & 15;
    if (dv == 0) continue;  // warp-uniform: no domain in this slot
    const float* Ld = Lp + (u * W + wl) * 300;
    float z = 0.f;
#pragma unroll
    for (int j = 0; j < 24; j++) {
      const float rj = __shfl_sync(0xffffffffu, rv[u], j);
      const float a = j <= ii ? Ld[ii * (ii + 1) / 2 + j] : Ld[j * (j + 1) / 2 + ii];
      z = fmaf(a, rj, z);
    }
    if (mb.dcoarse) z += coarse_share(mb, gwarp + u * nwarps, rv[u], dv);
    if (f.gi[u] >= 0) {
      if ((f.meta >> u) & 1) z = 0.f;
      mb.z[f.gi[u]] = z;
      rz += (double)rv[u] * z;
    }
  }
}

__device__ __forceinline__ void cl_res_domains(const Dev& d, const MixBufs& mb, float4* bufB, const float* Lp,
                                               float alpha, bool init, int wl, int W, int gwarp, int nwarps,
                                               const DomFacts& f, double& rr, double& rz) {
  const int per = (d.D + nwarps - 1) / nwarps;
  if (per <= 1) cl_res_domains_k<1>(d, mb, bufB, Lp, alpha, init, wl, W, gwarp, nwarps, f, rr, rz);
  else if (per == 2) cl_res_domains_k<2>(d, mb, bufB, Lp, alpha, init, wl, W, gwarp, nwarps, f, rr, rz);
  else cl_res_domains_k<3>(d, mb, bufB, Lp, alpha, init, wl, W, gwarp, nwarps, f, rr, rz);
}

__device__ __forceinline__ void cl_dof(const Dev& d, const MixBufs& mb, const float* pn, float alpha, bool init, int i,
                                       double& rr, double& rz) {
  const bool pin = d.pinned[i / 3];
  float xi, ri;
  if (init) {
    xi = 0.f;
    ri = (float)(-d.g[i]);
  } else {
    xi = mb.x[i] + alpha * pn[i];
    ri = mb.r[i] - alpha * mb.Ap[i];
  }
  if (pin) { xi = 0.f; ri = 0.f; }
  mb.x[i] = xi;
  mb.r[i] = ri;
  rr += (double)ri * ri;
  float zi = d.diag[i] > 1e-12 ? (float)((double)ri / d.diag[i]) : ri;
  if (pin) zi = 0.f;
  mb.z[i] = zi;
  rz += (double)ri * zi;
}

template <bool RES>
__global__ void __launch_bounds__(kClT, 1) k_mx_pcg_cluster(ClArgs A) {
  cg::cluster_group cl = cg::this_cluster();
  __shared__ double sm[32];
  // Partials alternate between two banks: a bank is rewritten only after the
  // cluster barrier that follows every CTA's read of it.
  __shared__ RedBank red[2];
  __shared__ double bcs[2][4];   // broadcast banks of cl_totals, alternating per call
  __shared__ double wsm[3 * 32];
  int round = 0;
#define BC (bcs[round & 1])
  const Dev& d = A.d;
  const MixBufs& mb = A.mb;
  const int n3 = d.n * 3;
  const int rank = (int)cl.block_rank(), nrank = (int)cl.num_blocks();
  const int tid = rank * blockDim.x + threadIdx.x, nth = nrank * blockDim.x;
  const int gwarp = tid >> 5, nwarps = nth >> 5;
  const bool jacobi = d.precond == 0;
  const float invH2 = (float)d.invH2;
  const float C00 = mb.C00, C11 = mb.C11, C01 = mb.C01, G = mb.G;
  // lanes per vertex in phase A: 4, 2 or 1 as the cluster's threads allow
  const int T = nth >= 4 * d.n ? 4 : nth >= 2 * d.n ? 2 : 1;
  const int lane = threadIdx.x & (T - 1);
  const int vStride = nth / T, vRounds = (d.n + vStride - 1) / vStride;

  // ---- resident phase A: this CTA's lists into shared memory (once per launch) ----
  extern __shared__ __align__(16) unsigned char cl_dyn[];
  const ClPlan& P = A.plan;
  const bool useHin = mb.hrec != nullptr;
  constexpr int W = kClT / 32;  // warps per CTA
  // layout and counts live in shared memory (read where used) to keep them
  // out of the registers the PCG loop needs
  __shared__ ClSmem Ls;
  __shared__ int Lc[6];  // vb0, nOwn, nHalo, nTri, nHin, domain slots
  if constexpr (RES) {
    const int vb0 = P.vb[rank];
    const int nOwn = P.vb[rank + 1] - vb0;
    const int h0 = P.haloOff[rank], t0 = P.triOff[rank], g0 = P.hinOff[rank], i0 = P.incOff[vb0];
    const int nHalo = P.haloOff[rank + 1] - h0;
    const int nTri = P.triOff[rank + 1] - t0;
    const int nHin = useHin ? P.hinOff[rank + 1] - g0 : 0;
    const int nInc = P.incOff[vb0 + nOwn] - i0;
    // domain slots u * W + wl of this CTA's warps (dom = rank * W + wl + u * nwarps)
    int nSlots = 0;
    for (int u = 0; u < 3; u++) {
      const int first = rank * W + u * nwarps;
      if (first < d.D) nSlots = u * W + min(W, d.D - first);
    }
    const ClSmem L = cl_smem_layout(nHalo, nTri, nHin, nInc, nOwn, nSlots, useHin, P.cCap);
    if (threadIdx.x == 0) {
      Ls = L;
      Lc[0] = vb0; Lc[1] = nOwn; Lc[2] = nHalo; Lc[3] = nTri; Lc[4] = nHin; Lc[5] = nSlots;
    }
    // packed lower triangle of each slot's inverse (zero outside the domain's dofs)
    float* Lp = reinterpret_cast<float*>(cl_dyn + L.Lp);
    for (int t = threadIdx.x; t < nSlots * 576; t += blockDim.x) {
      const int slot = t / 576, i = (t / 24) % 24, j = t % 24;
      if (j > i) continue;
      const int dom = rank * W + slot % W + (slot / W) * nwarps;
      const int dw = (d.domStart[dom + 1] - d.domStart[dom]) * 3;
      Lp[slot * 300 + i * (i + 1) / 2 + j] = i < dw && j < dw ? mb.Linv[(size_t)dom * 576 + i * 24 + j] : 0.f;
    }
    int* ownDstS = reinterpret_cast<int*>(cl_dyn + L.ownDst);
    for (int lv = threadIdx.x; lv < nOwn; lv += blockDim.x) ownDstS[lv] = P.vDst[vb0 + lv];
    int* haloS = reinterpret_cast<int*>(cl_dyn + L.halo);
    for (int i = threadIdx.x; i < nHalo; i += blockDim.x) haloS[i] = P.halo[h0 + i];
    float4* triD = reinterpret_cast<float4*>(cl_dyn + L.triD);
    for (int sl = threadIdx.x; sl < nTri; sl += blockDim.x) {
      const float4* src = reinterpret_cast<const float4*>(mb.tris) + (size_t)P.triId[t0 + sl] * 4;
      const ushort4 lc = P.triLoc[t0 + sl];
      float4 t3 = src[3];
      t3.z = __uint_as_float((uint32_t)lc.x | ((uint32_t)lc.y << 16));
      t3.w = __uint_as_float((uint32_t)lc.z);
      triD[sl * 4] = src[0];
      triD[sl * 4 + 1] = src[1];
      triD[sl * 4 + 2] = src[2];
      triD[sl * 4 + 3] = t3;
    }
    if (useHin) {
      float4* hinG = reinterpret_cast<float4*>(cl_dyn + L.hinG);
      ushort4* hinL = reinterpret_cast<ushort4*>(cl_dyn + L.hinL);
      for (int sl = threadIdx.x; sl < nHin; sl += blockDim.x) {
        const float4* src = mb.hrec + (size_t)P.hinId[g0 + sl] * 4;
        hinG[sl * 3] = src[1];
        hinG[sl * 3 + 1] = src[2];
        hinG[sl * 3 + 2] = src[3];
        hinL[sl] = P.hinLoc[g0 + sl];
      }
    }
    uint32_t* incS = reinterpret_cast<uint32_t*>(cl_dyn + L.inc);
    for (int j = threadIdx.x; j < nInc; j += blockDim.x) incS[j] = P.inc[i0 + j];
    int* incOffS = reinterpret_cast<int*>(cl_dyn + L.incOff);
    int* incHinS = reinterpret_cast<int*>(cl_dyn + L.incHin);
    int* ownHS = reinterpret_cast<int*>(cl_dyn + L.ownH);
    float2* ownMP = reinterpret_cast<float2*>(cl_dyn + L.ownMP);
    uint32_t* cOffS = reinterpret_cast<uint32_t*>(cl_dyn + L.cOff);
    if (d.hasContact) {
      // this launch's contact records of the owned vertices: ids on chip up to the capacity
      const uint32_t r0 = d.c.cOff[vb0], nr = min(d.c.cOff[vb0 + nOwn] - r0, (uint32_t)L.cCap);
      uint32_t* recS = reinterpret_cast<uint32_t*>(cl_dyn + L.cRec);
      for (uint32_t q = threadIdx.x; q < nr; q += blockDim.x) recS[q] = d.c.cRec[r0 + q];
    }
    for (int lv = threadIdx.x; lv <= nOwn; lv += blockDim.x) {
      incOffS[lv] = P.incOff[vb0 + lv] - i0;
      if (d.hasContact) cOffS[lv] = d.c.cOff[vb0 + lv];
      if (lv < nOwn) {
        incHinS[lv] = P.incHin[vb0 + lv] - i0;
        ownHS[lv] = P.ownHalo[vb0 + lv];
        ownMP[lv] = make_float2(d.mass[vb0 + lv], d.pinned[vb0 + lv] ? 1.f : 0.f);
      }
    }
    __syncthreads();  // the init below reads the slots' inverses
  }

  DomFacts dfacts{{-1, -1, -1}, 0};
  if (!jacobi && d.D <= 3 * nwarps) dfacts = cl_domain_facts(d, gwarp, nwarps);

  // ---- init: r = -g (filtered), x = 0, z = M^-1 r; |b|^2, r.r, r.z -------------------
  double bb = 0, rr = 0, rz = 0;
  for (int i = tid; i < n3; i += nth) {
    const double bi = -d.g[i];
    bb += bi * bi;
  }
  if constexpr (RES) {
    cl_res_domains(d, mb, reinterpret_cast<float4*>(cl_dyn + Ls.bufB), reinterpret_cast<const float*>(cl_dyn + Ls.Lp),
                   0.f, true, threadIdx.x >> 5, W, gwarp, nwarps, dfacts, rr, rz);
  } else if (jacobi) {
    for (int i = tid; i < n3; i += nth) cl_dof(d, mb, nullptr, 0.f, true, i, rr, rz);
  } else {
    cl_all_domains(d, mb, nullptr, 0.f, true, gwarp, nwarps, dfacts, rr, rz);
  }
  if (d.hasContact) {
    const Contact& c = d.c;
    for (int i = tid, na = n_active(c); i < na; i += nth) {
      const double dist = js_max(frozen_dist(c, d.x, c.active[i]), 1e-12);
      A.coef[i] = dist < c.dHat ? barrier_curvature(dist, c.dHat, c.kappa) : 0.0;
    }
  }
  {
    const double v3[3] = {bb, rr, rz};
    block_partials<3>(cl, v3, red[round & 1], rank, nrank, wsm);
  }
  cl.sync();
  double tot[3];
  cl_totals<3>(red[round & 1], nrank, tot);
  round++;
  double rzCur = tot[2];
  const double bNorm = sqrt(tot[0]);
  const double absTol = fmax(A.tol * fmax(bNorm, 1e-12), 1e-12);
  double residual = sqrt(tot[1]);
  int iters = 0;
  bool done = residual < absTol;
  float beta = 0.f;
  bool first = true;
  float* pc = A.pA;  // p_{k-1}
  float* pn = A.pB;  // p_k
  int k = 0;
  for (; !done && k < A.maxIters; k++) {
    // ---- phase A: p_k, Ap_k, p.Ap ------------------------------------------------
    // T consecutive lanes share a vertex and split its incident records; each
    // lane issues the loads of up to three records before using any, so the
    // gathers overlap. The T shares are summed with a fixed xor tree.
    double pAp = 0;
    if constexpr (RES) {
      const ClSmem& L = Ls;
      const int vb0 = Lc[0], nOwn = Lc[1], nHalo = Lc[2], nTri = Lc[3], nHin = Lc[4];
      float4* pH = reinterpret_cast<float4*>(cl_dyn + L.pH);
      const float4* triD = reinterpret_cast<const float4*>(cl_dyn + L.triD);
      float* triO = reinterpret_cast<float*>(cl_dyn + L.triO);
      const float4* hinG = reinterpret_cast<const float4*>(cl_dyn + L.hinG);
      const ushort4* hinL = reinterpret_cast<const ushort4*>(cl_dyn + L.hinL);
      float* hinS = reinterpret_cast<float*>(cl_dyn + L.hinS);
      const uint32_t* incS = reinterpret_cast<const uint32_t*>(cl_dyn + L.inc);
      const int* incOffS = reinterpret_cast<const int*>(cl_dyn + L.incOff);
      const int* incHinS = reinterpret_cast<const int*>(cl_dyn + L.incHin);
      const int* ownHS = reinterpret_cast<const int*>(cl_dyn + L.ownH);
      const int* haloS = reinterpret_cast<const int*>(cl_dyn + L.halo);
      // A0: p_k on the halo
      for (int i = threadIdx.x; i < nHalo; i += blockDim.x) {
        const float3 pv = ld_p(mb.z, pc, beta, first, haloS[i]);
        pH[i] = make_float4(pv.x, pv.y, pv.z, 0.f);
      }
      __syncthreads();
      // contact records of the owned vertices (they read the halo)
      if (d.hasContact) {
        const uint32_t* cOffS = reinterpret_cast<const uint32_t*>(cl_dyn + L.cOff);
        cl_contact_records_res(d, mb, A.coef, pc, beta, first, cOffS[0], cOffS[nOwn],
                               reinterpret_cast<const uint32_t*>(cl_dyn + L.cRec),
                               reinterpret_cast<float*>(cl_dyn + L.cShare), (uint32_t)L.cCap, pH, ownHS, vb0, nOwn);
      }
      // A1: element HVPs from shared memory, triangles then hinges in one index space
      for (int e = threadIdx.x; e < nTri + nHin; e += blockDim.x) {
        if (e < nTri) {
          const float4 t3 = triD[e * 4 + 3];
          const uint32_t l01 = __float_as_uint(t3.z), l2 = __float_as_uint(t3.w);
          float g1[3], g2[3];
          tri_hvp_g12(triD[e * 4], triD[e * 4 + 1], triD[e * 4 + 2], t3, pH[l01 & 0xffffu], pH[l01 >> 16], pH[l2],
                      C00, C11, C01, G, g1, g2);
          float* o = triO + e * 9;  // corner shares: -(g1 + g2), g1, g2
#pragma unroll
          for (int q = 0; q < 3; q++) {
            o[q] = -(g1[q] + g2[q]);
            o[3 + q] = g1[q];
            o[6 + q] = g2[q];
          }
        } else {
          const int sl = e - nTri;
          const ushort4 l = hinL[sl];
          const float4 P0 = pH[l.x], P1 = pH[l.y], P2 = pH[l.z], P3 = pH[l.w];
          const float4 g0 = hinG[sl * 3], g1 = hinG[sl * 3 + 1], g2 = hinG[sl * 3 + 2];
          hinS[sl] = g0.x * P0.x + g0.y * P0.y + g0.z * P0.z + g0.w * P1.x + g1.x * P1.y + g1.y * P1.z +
                     g1.z * P2.x + g1.w * P2.y + g2.x * P2.z + g2.y * P3.x + g2.z * P3.y + g2.w * P3.z;
        }
      }
      __syncthreads();
      // A2: per owned vertex, T2 lanes split its incidences (each lane in CSR
      // order, four shared-memory gathers in flight), a fixed xor tree adds
      // the lanes, then contacts and the mass term
      const float2* ownMP = reinterpret_cast<const float2*>(cl_dyn + L.ownMP);
      const uint32_t* cOffS = reinterpret_cast<const uint32_t*>(cl_dyn + L.cOff);
      const int T2 = 2 * nOwn <= (int)blockDim.x ? 2 : 1;
      const int l2 = threadIdx.x & (T2 - 1);
      for (int base = 0; base < nOwn; base += blockDim.x / T2) {
        const int lv = base + threadIdx.x / T2;
        const bool valid = lv < nOwn;
        float sp[3] = {0.f, 0.f, 0.f};
        if (valid) {
          const int jh = incHinS[lv], je = incOffS[lv + 1];
          for (int j0 = incOffS[lv] + l2; j0 < jh; j0 += 4 * T2) {
            uint32_t rec[4];
#pragma unroll
            for (int u = 0; u < 4; u++) rec[u] = j0 + u * T2 < jh ? incS[j0 + u * T2] : 0xffffffffu;
#pragma unroll
            for (int u = 0; u < 4; u++) {
              if (rec[u] == 0xffffffffu) continue;
              const float* o = triO + (rec[u] >> 2) * 9 + (rec[u] & 3) * 3;
#pragma unroll
              for (int q = 0; q < 3; q++) sp[q] += o[q];
            }
          }
          if (useHin) {
            for (int j0 = jh + l2; j0 < je; j0 += 4 * T2) {
              uint32_t rec[4];
#pragma unroll
              for (int u = 0; u < 4; u++) rec[u] = j0 + u * T2 < je ? incS[j0 + u * T2] : 0xffffffffu;
#pragma unroll
              for (int u = 0; u < 4; u++) {
                if (rec[u] == 0xffffffffu) continue;
                const float gs = hinS[rec[u] >> 2];
                // this vertex's 3 values of g: floats 3c .. 3c + 2 of the hinge's 12
                const float* gc = reinterpret_cast<const float*>(hinG + (rec[u] >> 2) * 3) + (rec[u] & 3) * 3;
                sp[0] += gs * gc[0];
                sp[1] += gs * gc[1];
                sp[2] += gs * gc[2];
              }
            }
          }
        }
        if (T2 == 2) {
          sp[0] += __shfl_xor_sync(0xffffffffu, sp[0], 1);
          sp[1] += __shfl_xor_sync(0xffffffffu, sp[1], 1);
          sp[2] += __shfl_xor_sync(0xffffffffu, sp[2], 1);
        }
        if (!valid || l2 != 0) continue;
        const int v = vb0 + lv;
        const float4 pv = pH[ownHS[lv]];
        double ch[3] = {0, 0, 0};
        if (d.hasContact) {
          const Contact& c = d.c;
          const float* shareS = reinterpret_cast<const float*>(cl_dyn + L.cShare);
          const uint32_t r0 = cOffS[0], cap = (uint32_t)L.cCap;
          for (uint32_t q = cOffS[lv]; q < cOffS[lv + 1]; q++) {
            if (q - r0 < cap) {
              const float* o = shareS + (size_t)(q - r0) * 3;
              ch[0] += o[0]; ch[1] += o[1]; ch[2] += o[2];
            } else {
              const double* o = c.recScratch + (size_t)q * 3;
              ch[0] += o[0]; ch[1] += o[1]; ch[2] += o[2];
            }
          }
        }
        const float2 mp = ownMP[lv];
        const float pvv[3] = {pv.x, pv.y, pv.z};
        // (Ap, p) of the three dofs into the phase-B slot of the warp that owns
        // this vertex's Schwarz domain, in that CTA's shared memory
        const int dst = reinterpret_cast<const int*>(cl_dyn + L.ownDst)[lv];
        float4* rb = cl.map_shared_rank(reinterpret_cast<float4*>(cl_dyn + L.bufB), dst >> 24) + (dst & 0xffffff);
#pragma unroll
        for (int q = 0; q < 3; q++) {
          const int i = v * 3 + q;
          float ap = mp.x * pvv[q] * invH2 + sp[q] + (float)ch[q];
          if (mp.y != 0.f) ap = 0.f;
          pn[i] = pvv[q];
          *reinterpret_cast<float2*>(rb + q) = make_float2(ap, pvv[q]);
          pAp += (double)pvv[q] * ap;
        }
      }
    } else
    for (int it = 0; it < vRounds; it++) {
      const int v = tid / T + it * vStride;
      const bool valid = v < d.n;
      if (d.hasContact) {
        // Frozen-contact shares of this CTA's vertices [v0, v1) for this round,
        // one record per thread (a vertex may sit in many contacts), written to
        // the record scratch and summed per vertex below in record order. Later
        // rounds cover other vertices, hence other records; the next iteration
        // rewrites these only after two cluster barriers.
        const int v0 = min(d.n, rank * (kClT / T) + it * vStride), v1 = min(d.n, v0 + kClT / T);
        cl_contact_records(d, mb, A.coef, pc, beta, first, d.c.cOff[v0], d.c.cOff[v1]);
        __syncthreads();
      }
      float sp[3] = {0.f, 0.f, 0.f};
      if (valid) {
        const uint32_t q1 = d.memOff[v + 1];
        for (uint32_t qb = d.memOff[v] + lane; qb < q1; qb += 3 * T) {
          float4 ids[3];
#pragma unroll
          for (int u = 0; u < 3; u++) {
            const uint32_t q = qb + u * T;
            // record q = (triangle << 2 | corner): state + vertex ids, read contiguously
            ids[u] = q < q1 ? __ldg(mb.vrec + (size_t)q * 5 + 4) : make_float4(0.f, 0.f, 0.f, 0.f);
          }
          float3 P[3][3];
#pragma unroll
          for (int u = 0; u < 3; u++) {
            if (qb + u * T < q1) {
              P[u][0] = ld_p(mb.z, pc, beta, first, __float_as_int(ids[u].x));
              P[u][1] = ld_p(mb.z, pc, beta, first, __float_as_int(ids[u].y));
              P[u][2] = ld_p(mb.z, pc, beta, first, __float_as_int(ids[u].z));
            }
          }
#pragma unroll
          for (int u = 0; u < 3; u++) {
            const uint32_t q = qb + u * T;
            if (q < q1) {
              float o[3];
              tri_hvp_corner(reinterpret_cast<const float*>(mb.vrec + (size_t)q * 5), P[u][0], P[u][1], P[u][2],
                             __float_as_int(ids[u].w), C00, C11, C01, G, o);
              sp[0] += o[0]; sp[1] += o[1]; sp[2] += o[2];
            }
          }
        }
      }
      if (valid && mb.hrec) {
        // exact-Newton mode: Gauss-Newton bending g (g . p) of the incident
        // hinges (record = hinge << 2 | corner), split over the T lanes
        const uint32_t h1 = d.hinOff[v + 1];
        for (uint32_t q = d.hinOff[v] + lane; q < h1; q += T) {
          const uint32_t rec = d.hinRec[q];
          const float4* hr = mb.hrec + (size_t)(rec >> 2) * 4;
          const float4 hid = __ldg(hr), g0 = __ldg(hr + 1), g1 = __ldg(hr + 2), g2 = __ldg(hr + 3);
          const float3 P0 = ld_p(mb.z, pc, beta, first, __float_as_int(hid.x));
          const float3 P1 = ld_p(mb.z, pc, beta, first, __float_as_int(hid.y));
          const float3 P2 = ld_p(mb.z, pc, beta, first, __float_as_int(hid.z));
          const float3 P3 = ld_p(mb.z, pc, beta, first, __float_as_int(hid.w));
          const float gs = g0.x * P0.x + g0.y * P0.y + g0.z * P0.z + g0.w * P1.x + g1.x * P1.y + g1.y * P1.z +
                           g1.z * P2.x + g1.w * P2.y + g2.x * P2.z + g2.y * P3.x + g2.z * P3.y + g2.w * P3.z;
          const int c = (int)(rec & 3);  // this vertex's 3 values of g, selected without local memory
          const float ga = c == 0 ? g0.x : c == 1 ? g0.w : c == 2 ? g1.z : g2.y;
          const float gb = c == 0 ? g0.y : c == 1 ? g1.x : c == 2 ? g1.w : g2.z;
          const float gc = c == 0 ? g0.z : c == 1 ? g1.y : c == 2 ? g2.x : g2.w;
          sp[0] += gs * ga;
          sp[1] += gs * gb;
          sp[2] += gs * gc;
        }
      }
#pragma unroll
      for (int o = 1; o < T; o <<= 1) {
        sp[0] += __shfl_xor_sync(0xffffffffu, sp[0], o);
        sp[1] += __shfl_xor_sync(0xffffffffu, sp[1], o);
        sp[2] += __shfl_xor_sync(0xffffffffu, sp[2], o);
      }
      if (!valid || lane != 0) continue;
      const float3 pv = ld_p(mb.z, pc, beta, first, v);
      double ch[3] = {0, 0, 0};
      if (d.hasContact) {
        const Contact& c = d.c;
        for (uint32_t q = c.cOff[v]; q < c.cOff[v + 1]; q++) {
          const double* o = c.recScratch + (size_t)q * 3;
          ch[0] += o[0]; ch[1] += o[1]; ch[2] += o[2];
        }
      }
      const float M = d.mass[v];
      const bool pin = d.pinned[v];
      const float pvv[3] = {pv.x, pv.y, pv.z};
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const int i = v * 3 + q;
        float ap = M * pvv[q] * invH2 + sp[q] + (float)ch[q];
        if (pin) ap = 0.f;
        pn[i] = pvv[q];
        mb.Ap[i] = ap;
        pAp += (double)pvv[q] * ap;
      }
    }
    block_partials<1>(cl, &pAp, red[round & 1], rank, nrank, wsm);
    cl.sync();
    cl_totals<1>(red[round & 1], nrank, tot);
    round++;
    const double pApT = tot[0];
    if (!(pApT > 1e-30)) { iters = k; done = true; break; }
    const float alpha = (float)(rzCur / pApT);
    // ---- phase B: x, r, z; r.r, r.z ---------------------------------------------
    rr = 0;
    rz = 0;
    if constexpr (RES) {
      cl_res_domains(d, mb, reinterpret_cast<float4*>(cl_dyn + Ls.bufB),
                     reinterpret_cast<const float*>(cl_dyn + Ls.Lp), alpha, false, threadIdx.x >> 5, W, gwarp, nwarps,
                     dfacts, rr, rz);
    } else if (jacobi) {
      for (int i = tid; i < n3; i += nth) cl_dof(d, mb, pn, alpha, false, i, rr, rz);
    } else {
      cl_all_domains(d, mb, pn, alpha, false, gwarp, nwarps, dfacts, rr, rz);
    }
    {
      const double v2[2] = {rr, rz};
      block_partials<2>(cl, v2, red[round & 1], rank, nrank, wsm);
    }
    cl.sync();
    double t2[2];
    cl_totals<2>(red[round & 1], nrank, t2);
    round++;
    residual = sqrt(t2[0]);
    if (residual < absTol) { iters = k + 1; done = true; break; }
    beta = (float)(t2[1] / rzCur);
    rzCur = t2[1];
    first = false;
    float* tmp = pc;
    pc = pn;
    pn = tmp;
  }
  if (!done) iters = A.maxIters;
  if constexpr (RES) {
    // x lives in the phase-B slots during the solve
    const float4* bufB = reinterpret_cast<const float4*>(cl_dyn + Ls.bufB);
    const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
#pragma unroll
    for (int u = 0; u < 3; u++)
      if (dfacts.gi[u] >= 0) mb.x[dfacts.gi[u]] = bufB[(u * W + wl) * 24 + lane].z;
    cl.sync();
  }

  // ---- descent safeguard + trust region in FP64 (newton.ts:152-179) -------------------
  double gt = 0;
  for (int i = tid; i < n3; i += nth) {
    const double di = mb.x[i];
    d.dx[i] = di;
    gt += d.g[i] * di;
  }
  block_partials<1>(cl, &gt, red[round & 1], rank, nrank, wsm);
  cl.sync();
  double t1[1];
  cl_totals<1>(red[round & 1], nrank, t1);
  round++;
  double gtdx = t1[0];
  bool fallback = false;
  if (!isfinite(gtdx) || gtdx >= 0) {
    fallback = true;
    gt = 0;
    for (int i = tid; i < n3; i += nth) {
      const double di = -d.g[i] / d.diag[i];
      d.dx[i] = di;
      gt += d.g[i] * di;
    }
    block_partials<1>(cl, &gt, red[round & 1], rank, nrank, wsm);
    cl.sync();
    cl_totals<1>(red[round & 1], nrank, t1);
    round++;
    gtdx = t1[0];
  }
  double mxd = 0;
  for (int i = tid; i < n3; i += nth) mxd = fmax(mxd, fabs(d.dx[i]));
  {
    const double s = block_max(mxd, sm);
    if (threadIdx.x == 0) red[round & 1][0][0] = s;
    cl.sync();
    if (threadIdx.x == 0) {
      double r = 0;
      for (int q = 0; q < nrank; q++) r = fmax(r, *cl.map_shared_rank(&red[round & 1][0][0], q));
      BC[0] = r;
    }
    __syncthreads();
  }
  const double maxDx = BC[0];
  round++;
  if (maxDx > 0.002) {
    const double s = 0.002 / maxDx;
    for (int i = tid; i < n3; i += nth) d.dx[i] *= s;
    gtdx *= s;
  }
  if (rank == 0 && threadIdx.x == 0) {
    d.scal[S_PCG_ITERS] = iters;
    d.scal[S_PCG_RES] = residual;
    d.scal[S_GTDX] = gtdx;
    d.scal[S_FALLBACK] = fallback ? 1 : 0;
    d.scal[S_MAXDX] = maxDx;
  }
  cl.sync();  // no CTA leaves while a peer may still read its shared memory
#undef BC
}

// Largest cluster (16, then 8, 4, 2, 1 CTAs) the device can co-schedule for
// this kernel; 0 when none.
int mx_cluster_size() {
  static int cached = -1;
  if (cached >= 0) return cached;
  cudaFuncSetAttribute(k_mx_pcg_cluster<false>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaFuncSetAttribute(k_mx_pcg_cluster<true>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cached = 0;
  for (int cs = 16; cs >= 1; cs /= 2) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(kClT);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nc = 0;
    if (cudaOccupancyMaxActiveClusters(&nc, k_mx_pcg_cluster<false>, &cfg) == cudaSuccess && nc >= 1) {
      cached = cs;
      break;
    }
  }
  cudaGetLastError();
  return cached;
}

bool mx_cluster_resident_ok(int clusterSize, size_t smemBytes) {
  if (clusterSize < 1 || smemBytes > (size_t)kClMaxDynSmem) return false;
  // The kernel's limit is process-wide: it only grows, so a launch sized for
  // an earlier solver's mesh stays valid.
  static std::mutex mu;
  static size_t limit = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    if (smemBytes > limit) {
      if (cudaFuncSetAttribute(k_mx_pcg_cluster<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemBytes) !=
          cudaSuccess) {
        cudaGetLastError();
        return false;
      }
      limit = smemBytes;
    }
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(clusterSize);
  cfg.blockDim = dim3(kClT);
  cfg.dynamicSmemBytes = smemBytes;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = clusterSize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int nc = 0;
  const bool ok = cudaOccupancyMaxActiveClusters(&nc, k_mx_pcg_cluster<true>, &cfg) == cudaSuccess && nc >= 1;
  cudaGetLastError();
  return ok;
}

int mx_launch_pcg_cluster(const Dev& d, const MixBufs& mb, const ClPlan& plan, float* pA, float* pB, double* coef,
                          int maxIters, double tol, int clusterSize, cudaStream_t s) {
  ClArgs a{d, mb, pA, pB, coef, maxIters, tol, plan};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(clusterSize);
  cfg.blockDim = dim3(kClT);
  cfg.dynamicSmemBytes = plan.resident ? (size_t)plan.smemBytes : 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = clusterSize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return plan.resident ? (int)cudaLaunchKernelEx(&cfg, k_mx_pcg_cluster<true>, a)
                       : (int)cudaLaunchKernelEx(&cfg, k_mx_pcg_cluster<false>, a);
}

}  // namespace cs
