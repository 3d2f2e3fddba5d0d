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
#include <cooperative_groups.h>

#include "contact.cuh"
#include "hvp32.cuh"
#include "mixed.cuh"

namespace cg = cooperative_groups;

namespace cs {

constexpr int kClT = 512;

struct ClArgs {
  Dev d;
  MixBufs mb;
  float* pA;      // search direction, double-buffered (3n each)
  float* pB;
  double* coef;   // per active contact: barrier curvature at the frozen distance (0 outside dHat)
  int maxIters;
  double tol;
};

// Cluster-wide totals of `k` partials deposited in red[0..k) by every CTA.
// Lane r of warp 0 reads CTA r's partials, a fixed shuffle tree adds them, and
// the result is broadcast through shared memory: identical bits in every CTA.
template <int K>
__device__ __forceinline__ void cl_totals(cg::cluster_group& cl, double* red, double* out, double* bc) {
  if (threadIdx.x < 32) {
    const unsigned nr = cl.num_blocks();
    double v[K];
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = 0;
    if (threadIdx.x < nr) {
      const double* peer = cl.map_shared_rank(red, threadIdx.x);
#pragma unroll
      for (int k = 0; k < K; k++) v[k] = peer[k];
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
      double s = v[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      if (threadIdx.x == 0) bc[k] = s;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; k++) out[k] = bc[k];
  // no trailing barrier: consecutive calls alternate between two bc banks
}

// This CTA's sums of K per-thread values into out[0..K) (thread 0 writes):
// warp shuffle trees, one block barrier, warp 0 adds the warp partials in a
// fixed order. wsm holds K x 32 doubles; it is rewritten only after the next
// cluster barrier, by which time warp 0 has read it.
template <int K>
__device__ __forceinline__ void block_partials(const double* v, double* out, double* wsm) {
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
#pragma unroll
    for (int k = 0; k < K; k++) {
      double t = lane < nw ? wsm[k * 32 + lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      if (lane == 0) out[k] = t;
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

// Phase B on K Schwarz domains dom0, dom0 + step, ... at once (one warp, lane =
// local dof): the loads of all K are issued before any product, so their
// latencies overlap. Adds the (r.r, r.z) shares.
template <int K>
__device__ __forceinline__ void cl_domains(const Dev& d, const MixBufs& mb, const float* pn, float alpha, bool init,
                                           int dom0, int step, double& rr, double& rz) {
  const int lane = threadIdx.x & 31;
  float rv[K];
  int gi[K];
  bool pin[K], act[K];
#pragma unroll
  for (int u = 0; u < K; u++) {
    const int dom = dom0 + u * step;
    rv[u] = 0.f;
    gi[u] = -1;
    pin[u] = false;
    act[u] = false;
    if (dom < d.D) {
      const int start = d.domStart[dom], dw = (d.domStart[dom + 1] - start) * 3;
      act[u] = lane < dw;
      if (act[u]) {
        gi[u] = d.domVerts[start + lane / 3] * 3 + lane % 3;
        pin[u] = d.pinned[gi[u] / 3];
        float xi, ri;
        if (init) {
          xi = 0.f;
          ri = (float)(-d.g[gi[u]]);
        } else {
          xi = mb.x[gi[u]] + alpha * pn[gi[u]];
          ri = mb.r[gi[u]] - alpha * mb.Ap[gi[u]];
        }
        if (pin[u]) { xi = 0.f; ri = 0.f; }
        mb.x[gi[u]] = xi;
        mb.r[gi[u]] = ri;
        rv[u] = ri;
        rr += (double)ri * ri;
      }
    }
  }
  // row `lane` of each 24x24 inverse: 96 bytes, six 16-byte loads
  float4 L[K][6];
#pragma unroll
  for (int u = 0; u < K; u++) {
    const float4* Li = reinterpret_cast<const float4*>(mb.Linv + (size_t)(dom0 + u * step) * 576) + lane * 6;
#pragma unroll
    for (int j4 = 0; j4 < 6; j4++) L[u][j4] = act[u] ? __ldg(Li + j4) : make_float4(0.f, 0.f, 0.f, 0.f);
  }
#pragma unroll
  for (int u = 0; u < K; u++) {
    float z = 0.f;
#pragma unroll
    for (int j4 = 0; j4 < 6; j4++) {
      z = fmaf(L[u][j4].x, __shfl_sync(0xffffffffu, rv[u], 4 * j4), z);
      z = fmaf(L[u][j4].y, __shfl_sync(0xffffffffu, rv[u], 4 * j4 + 1), z);
      z = fmaf(L[u][j4].z, __shfl_sync(0xffffffffu, rv[u], 4 * j4 + 2), z);
      z = fmaf(L[u][j4].w, __shfl_sync(0xffffffffu, rv[u], 4 * j4 + 3), z);
    }
    if (mb.dcoarse) {
      const int dom = dom0 + u * step;
      if (dom < d.D) z += coarse_share(mb, dom, rv[u], d.domStart[dom + 1] - d.domStart[dom]);
    }
    if (act[u]) {
      if (pin[u]) z = 0.f;
      mb.z[gi[u]] = z;
      rz += (double)rv[u] * z;
    }
  }
}

// Phase B over every domain, K = ceil(D / warps) (at most 3) per warp at once.
__device__ __forceinline__ void cl_all_domains(const Dev& d, const MixBufs& mb, const float* pn, float alpha,
                                               bool init, int gwarp, int nwarps, double& rr, double& rz) {
  const int per = (d.D + nwarps - 1) / nwarps;
  if (per <= 1) {
    if (gwarp < d.D) cl_domains<1>(d, mb, pn, alpha, init, gwarp, nwarps, rr, rz);
  } else if (per == 2) {
    cl_domains<2>(d, mb, pn, alpha, init, gwarp, nwarps, rr, rz);
  } else {
    for (int dom = gwarp; dom < d.D; dom += 3 * nwarps) cl_domains<3>(d, mb, pn, alpha, init, dom, nwarps, rr, rz);
  }
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

__global__ void __launch_bounds__(kClT, 1) k_mx_pcg_cluster(ClArgs A) {
  cg::cluster_group cl = cg::this_cluster();
  __shared__ double sm[32];
  // Partials alternate between two banks: a bank is rewritten only after the
  // cluster barrier that follows every CTA's read of it.
  __shared__ double red[2][4];
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

  // ---- init: r = -g (filtered), x = 0, z = M^-1 r; |b|^2, r.r, r.z -------------------
  double bb = 0, rr = 0, rz = 0;
  for (int i = tid; i < n3; i += nth) {
    const double bi = -d.g[i];
    bb += bi * bi;
  }
  if (jacobi) {
    for (int i = tid; i < n3; i += nth) cl_dof(d, mb, nullptr, 0.f, true, i, rr, rz);
  } else {
    cl_all_domains(d, mb, nullptr, 0.f, true, gwarp, nwarps, rr, rz);
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
    block_partials<3>(v3, red[round & 1], wsm);
  }
  cl.sync();
  double tot[3];
  cl_totals<3>(cl, red[round & 1], tot, BC);
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
    for (int it = 0; it < vRounds; it++) {
      const int v = tid / T + it * vStride;
      const bool valid = v < d.n;
      if (d.hasContact) {
        // Frozen-contact shares of this CTA's vertices [v0, v1) for this round,
        // one record per thread (a vertex may sit in many contacts), written to
        // the record scratch and summed per vertex below in record order. Later
        // rounds cover other vertices, hence other records; the next iteration
        // rewrites these only after two cluster barriers.
        const Contact& c = d.c;
        const int v0 = min(d.n, rank * (kClT / T) + it * vStride), v1 = min(d.n, v0 + kClT / T);
        const uint32_t r0 = c.cOff[v0], r1 = c.cOff[v1];
        for (uint32_t q = r0 + threadIdx.x; q < r1; q += blockDim.x) {
          const uint32_t rec = c.cRec[q];
          const double g = A.coef[rec >> 2];
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
          double* o = c.recScratch + (size_t)q * 3;
          o[0] = ch[0]; o[1] = ch[1]; o[2] = ch[2];
        }
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
    block_partials<1>(&pAp, red[round & 1], wsm);
    cl.sync();
    cl_totals<1>(cl, red[round & 1], tot, BC);
    round++;
    const double pApT = tot[0];
    if (!(pApT > 1e-30)) { iters = k; done = true; break; }
    const float alpha = (float)(rzCur / pApT);
    // ---- phase B: x, r, z; r.r, r.z ---------------------------------------------
    rr = 0;
    rz = 0;
    if (jacobi) {
      for (int i = tid; i < n3; i += nth) cl_dof(d, mb, pn, alpha, false, i, rr, rz);
    } else {
      cl_all_domains(d, mb, pn, alpha, false, gwarp, nwarps, rr, rz);
    }
    {
      const double v2[2] = {rr, rz};
      block_partials<2>(v2, red[round & 1], wsm);
    }
    cl.sync();
    double t2[2];
    cl_totals<2>(cl, red[round & 1], t2, BC);
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

  // ---- descent safeguard + trust region in FP64 (newton.ts:152-179) -------------------
  double gt = 0;
  for (int i = tid; i < n3; i += nth) {
    const double di = mb.x[i];
    d.dx[i] = di;
    gt += d.g[i] * di;
  }
  block_partials<1>(&gt, red[round & 1], wsm);
  cl.sync();
  double t1[1];
  cl_totals<1>(cl, red[round & 1], t1, BC);
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
    block_partials<1>(&gt, red[round & 1], wsm);
    cl.sync();
    cl_totals<1>(cl, red[round & 1], t1, BC);
    round++;
    gtdx = t1[0];
  }
  double mxd = 0;
  for (int i = tid; i < n3; i += nth) mxd = fmax(mxd, fabs(d.dx[i]));
  {
    const double s = block_max(mxd, sm);
    if (threadIdx.x == 0) red[round & 1][0] = s;
    cl.sync();
    if (threadIdx.x == 0) {
      double r = 0;
      for (int q = 0; q < nrank; q++) r = fmax(r, *cl.map_shared_rank(&red[round & 1][0], q));
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
  cudaFuncSetAttribute(k_mx_pcg_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
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
    if (cudaOccupancyMaxActiveClusters(&nc, k_mx_pcg_cluster, &cfg) == cudaSuccess && nc >= 1) {
      cached = cs;
      break;
    }
  }
  cudaGetLastError();
  return cached;
}

int mx_launch_pcg_cluster(const Dev& d, const MixBufs& mb, float* pA, float* pB, double* coef, int maxIters,
                          double tol, int clusterSize, cudaStream_t s) {
  ClArgs a{d, mb, pA, pB, coef, maxIters, tol};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(clusterSize);
  cfg.blockDim = dim3(kClT);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = clusterSize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return (int)cudaLaunchKernelEx(&cfg, k_mx_pcg_cluster, a);
}

}  // namespace cs
