// LBVH broadphase kernels (FP64 path file: compiled with -fmad=false).
//
// The pipeline follows the reference's FP32 mirror (gpu-broadphase.ts:193-386):
// swept AABB + centroid per triangle, 30-bit centroid Morton key, (key, triId)
// order (a stable radix sort of the key over triangle order), Karras 2012
// hierarchy with the sorted-position tiebreak, refit, per-leaf traversal.
// The refit here is bottom-up with one atomic arrival counter per node (the
// second child to arrive merges and climbs; no thread ever waits).
//
// Exactness for the FP64 path: internal nodes carry outward-rounded f32 boxes
// of the exact f64 swept boxes, and every leaf hit is re-tested with the f64
// boxes, so the emitted pair set equals the reference CPU BVH's set (all
// non-adjacent triangle pairs whose padded swept boxes overlap, inclusive),
// independent of tree shape (src/collision/bvh.ts:79-124).
#include "broadphase.cuh"
#include "common.cuh"

namespace cs {

constexpr int kBT = 256;
static inline int nb(int n) { return (n + kBT - 1) / kBT; }

__device__ __forceinline__ float rd(double v) { return __double2float_rd(v); }
__device__ __forceinline__ float ru(double v) { return __double2float_ru(v); }

// ---- boxes (aabb.ts:9-31 in f64; gpu-broadphase.ts:54-93 in FP32) ----------------
__global__ void k_boxes(BvhBufs b, const double* x0, const double* x1, double pad) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b.m) return;
  const int ids[3] = {(int)b.idx[t * 3], (int)b.idx[t * 3 + 1], (int)b.idx[t * 3 + 2]};
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  float fmn[3] = {INFINITY, INFINITY, INFINITY}, fmx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int q = 0; q < 3; q++) {
    const int v = ids[q];
    for (int w = 0; w < 2; w++) {
      const double* x = w == 0 ? x0 : x1;
      for (int k = 0; k < 3; k++) {
        const double c = x[v * 3 + k];
        if (c < mn[k]) mn[k] = c;
        if (c > mx[k]) mx[k] = c;
        const float cf = (float)c;
        if (cf < fmn[k]) fmn[k] = cf;
        if (cf > fmx[k]) fmx[k] = cf;
      }
    }
  }
  const float pf = (float)pad;
  for (int k = 0; k < 3; k++) {
    const double lo = mn[k] - pad, hi = mx[k] + pad;
    b.box64[t * 6 + k] = lo;
    b.box64[t * 6 + 3 + k] = hi;
    b.boxc[t * 6 + k] = rd(lo);
    b.boxc[t * 6 + 3 + k] = ru(hi);
    b.boxr[t * 6 + k] = __fsub_rn(fmn[k], pf);
    b.boxr[t * 6 + 3 + k] = __fadd_rn(fmx[k], pf);
    float s = 0.f;
    for (int q = 0; q < 3; q++) {
      s = __fadd_rn(s, (float)x0[ids[q] * 3 + k]);
      s = __fadd_rn(s, (float)x1[ids[q] * 3 + k]);
    }
    b.cent[t * 3 + k] = __fdiv_rn(s, 6.f);
  }
}

// Centroid bounds (min/max are exact, so one block's fixed loop suffices).
__global__ void __launch_bounds__(1024) k_scene_bounds(BvhBufs b) {
  __shared__ float sm[6][1024];
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int t = threadIdx.x; t < b.m; t += blockDim.x)
    for (int k = 0; k < 3; k++) {
      const float c = b.cent[t * 3 + k];
      if (c < mn[k]) mn[k] = c;
      if (c > mx[k]) mx[k] = c;
    }
  for (int k = 0; k < 3; k++) { sm[k][threadIdx.x] = mn[k]; sm[3 + k][threadIdx.x] = mx[k]; }
  __syncthreads();
  for (int off = 512; off > 0; off >>= 1) {
    if ((int)threadIdx.x < off)
      for (int k = 0; k < 3; k++) {
        const float a = sm[k][threadIdx.x + off], c = sm[3 + k][threadIdx.x + off];
        if (a < sm[k][threadIdx.x]) sm[k][threadIdx.x] = a;
        if (c > sm[3 + k][threadIdx.x]) sm[3 + k][threadIdx.x] = c;
      }
    __syncthreads();
  }
  if (threadIdx.x < 6) b.scene[threadIdx.x] = sm[threadIdx.x][0];
}

__device__ __forceinline__ uint32_t expand10(uint32_t v) {
  uint32_t x = v & 1023u;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

// gpu-broadphase.ts:105-117 mortonKeyOf: span = max(f32 span, 1e-9 as a double),
// n = fround(fround(c - min) / span) clamped to [0,1], q = floor(n * 1023).
__global__ void k_morton(BvhBufs b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b.m) return;
  uint32_t q[3];
  for (int k = 0; k < 3; k++) {
    const float smin = b.scene[k], smax = b.scene[3 + k];
    double span = (double)__fsub_rn(smax, smin);
    if (!(span > 1e-9)) span = span != span ? span : 1e-9;
    const float dc = __fsub_rn(b.cent[t * 3 + k], smin);
    const float nf = __double2float_rn((double)dc / span);
    double nn = (double)nf;
    nn = js_min(1.0, js_max(0.0, nn));
    q[k] = (uint32_t)floor(nn * 1023.0);
  }
  b.k0[t].w[0] = (expand10(q[0]) << 2) | (expand10(q[1]) << 1) | expand10(q[2]);
  b.p0[t] = (uint32_t)t;
}

__device__ __forceinline__ int delta_pos(const Key<1>* keys, int p, int q, int n) {
  if (q < 0 || q >= n) return -1;
  const uint32_t kp = keys[p].w[0], kq = keys[q].w[0];
  if (kp != kq) return __clz(kp ^ kq);
  return 32 + __clz((uint32_t)(p ^ q));
}

// gpu-broadphase.ts:253-299: range + split per internal node (power-of-two strides).
// Also writes the children's codes into the node's traversal record.
__global__ void k_karras(BvhBufs b, const Key<1>* sk, const uint32_t* sp) {
  const int m = b.m;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m - 1) return;
  const int dNext = delta_pos(sk, i, i + 1, m);
  const int dPrev = delta_pos(sk, i, i - 1, m);
  int d = 1, dMin = dPrev;
  if (dPrev > dNext) { d = -1; dMin = dNext; }
  long lMax = 2;
  while (delta_pos(sk, i, (int)(i + d * lMax), m) > dMin) {
    lMax *= 2;
    if (lMax > m) break;
  }
  long l = 0, t = lMax / 2;
  while (t > 0) {
    if (delta_pos(sk, i, (int)(i + d * (l + t)), m) > dMin) l += t;
    t /= 2;
  }
  const int j = (int)(i + d * l);
  const int lo = min(i, j), hi = max(i, j);
  const int dNode = delta_pos(sk, lo, hi, m);
  int split = lo, stride = 1;
  while (stride * 2 <= hi - lo) stride *= 2;
  while (stride > 0) {
    const int mid = split + stride;
    if (mid < hi && delta_pos(sk, lo, mid, m) > dNode) split = mid;
    stride /= 2;
  }
  const bool leafL = split == lo, leafR = split + 1 == hi;
  const int L = leafL ? m - 1 + lo : split;
  const int R = leafR ? m - 1 + split + 1 : split + 1;
  b.left[i] = L;
  b.right[i] = R;
  b.parent[L] = i;
  b.parent[R] = i;
  const int codeL = leafL ? ~(int)sp[lo] : L;
  const int codeR = leafR ? ~(int)sp[split + 1] : R;
  b.rec[4 * i + 0].w = __int_as_float(codeL);
  b.rec[4 * i + 2].w = __int_as_float(codeR);
  if (lo == 0 && hi == m - 1) *b.root = i;
}

__global__ void k_topo_init(BvhBufs b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * b.m - 1) return;
  b.parent[i] = -1;
}

__global__ void k_refit_init(BvhBufs b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * b.m - 1) return;
  if (i < b.m - 1) {
    // A node the climb never reaches stays infinite, which keeps traversal conservative.
    for (int k = 0; k < 3; k++) { b.nbox[i * 6 + k] = -INFINITY; b.nbox[i * 6 + 3 + k] = INFINITY; }
    for (int q = 0; q < 4; q += 2) {
      float4 lo = b.rec[4 * i + q], hi = b.rec[4 * i + q + 1];
      lo.x = lo.y = lo.z = -INFINITY;
      hi.x = hi.y = hi.z = INFINITY;
      b.rec[4 * i + q] = lo;
      b.rec[4 * i + q + 1] = hi;
    }
  }
  b.visit[i] = 0;
  b.depth[i] = 1;
}

// Writes node `child`'s finished box into its parent's record.
__device__ __forceinline__ void put_child_box(BvhBufs& b, int parent, int child, const float* bx) {
  const int side = b.left[parent] == child ? 0 : 2;
  float* r = (float*)(b.rec + 4 * parent + side);
  r[0] = bx[0]; r[1] = bx[1]; r[2] = bx[2];
  r[4] = bx[3]; r[5] = bx[4]; r[6] = bx[5];
}

// Leaf boxes, then climb: the second child to arrive at a node merges both
// children and continues. Bounded by the node count.
__global__ void k_refit(BvhBufs b, const uint32_t* sp, bool mirror) {
  const int m = b.m;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= m) return;
  const int slot = m - 1 + s;
  const uint32_t tri = sp[s];
  const float* src = mirror ? b.boxr : b.boxc;
  float bx[6];
  for (int k = 0; k < 6; k++) {
    bx[k] = src[tri * 6 + k];
    b.nbox[slot * 6 + k] = bx[k];
  }
  b.depth[slot] = 1;
  int node = b.parent[slot];
  if (node >= 0) put_child_box(b, node, slot, bx);
  __threadfence();
  for (int guard = 0; node >= 0 && guard < 2 * m; guard++) {
    const uint32_t prev = atomicAdd(&b.visit[node], 1u);
    if (prev == 0) return;
    __threadfence();
    const int L = b.left[node], R = b.right[node];
    for (int k = 0; k < 3; k++) {
      const float a = ((volatile float*)b.nbox)[L * 6 + k], c = ((volatile float*)b.nbox)[R * 6 + k];
      bx[k] = fminf(a, c);
      const float a2 = ((volatile float*)b.nbox)[L * 6 + 3 + k], c2 = ((volatile float*)b.nbox)[R * 6 + 3 + k];
      bx[3 + k] = fmaxf(a2, c2);
    }
    for (int k = 0; k < 6; k++) b.nbox[node * 6 + k] = bx[k];
    const int dL = ((volatile int*)b.depth)[L], dR = ((volatile int*)b.depth)[R];
    b.depth[node] = max(dL, dR) + 1;
    const int up = b.parent[node];
    if (up >= 0) put_child_box(b, up, node, bx);
    __threadfence();
    node = up;
  }
}

__device__ __forceinline__ bool ov6(const float* a, const float* c) {
  return a[0] <= c[3] && a[3] >= c[0] && a[1] <= c[4] && a[4] >= c[1] && a[2] <= c[5] && a[5] >= c[2];
}
// query box a (min xyz, max xyz) against a record box (lo = min + code, hi = max)
__device__ __forceinline__ bool ov_rec(const float* a, const float4& lo, const float4& hi) {
  return a[0] <= hi.x && a[3] >= lo.x && a[1] <= hi.y && a[4] >= lo.y && a[2] <= hi.z && a[5] >= lo.z;
}
__device__ __forceinline__ bool ov6d(const double* a, const double* c) {
  return a[0] <= c[3] && a[3] >= c[0] && a[1] <= c[4] && a[4] >= c[1] && a[2] <= c[5] && a[5] >= c[2];
}
__device__ __forceinline__ bool share_vertex(const uint32_t* idx, int a, int c) {
  const uint32_t A0 = idx[a * 3], A1 = idx[a * 3 + 1], A2 = idx[a * 3 + 2];
  const uint32_t B0 = idx[c * 3], B1 = idx[c * 3 + 1], B2 = idx[c * 3 + 2];
  return A0 == B0 || A0 == B1 || A0 == B2 || A1 == B0 || A1 == B1 || A1 == B2 || A2 == B0 || A2 == B1 || A2 == B2;
}

constexpr int kStack = 64;
constexpr int kLocalPairs = 8;

// Appends a thread's buffered pairs to the output through one atomic.
__device__ __forceinline__ void flush_pairs(int2* out, uint32_t cap, uint32_t* counter, const int2* buf, int k) {
  if (k == 0) return;
  const uint32_t base = atomicAdd(counter, (uint32_t)k);
  for (int q = 0; q < k; q++)
    if (base + q < cap) out[base + q] = buf[q];
}

// Self traversal per sorted leaf s (gpu-broadphase.ts:321-357): children of
// each popped node are tested against the query leaf's box; leaves with a
// larger triangle id that share no vertex are pairs.
// MODE 0 counts per leaf, 1 writes at the scanned offsets (the reference's
// per-leaf stack order), 2 appends the exact set through b.cnt[0].
template <int MODE>
__global__ void __launch_bounds__(128) k_self(BvhBufs b, const uint32_t* sp, bool mirror) {
  const int m = b.m;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= m) return;
  const int q = (int)sp[s];
  const float* qb = (mirror ? b.boxr : b.boxc) + (size_t)q * 6;
  float qbox[6];
  for (int k = 0; k < 6; k++) qbox[k] = qb[k];
  const double* q64 = b.box64 + (size_t)q * 6;
  uint32_t count = 0;
  uint32_t out = MODE == 1 ? b.cnt[s] : 0;
  int2 buf[kLocalPairs];
  int nbuf = 0;
  int stack[kStack];
  int sp_ = 0;
  stack[sp_++] = *b.root;
  long guard = 0;
  while (sp_ > 0) {
    if (++guard > 4l * m + 8) { atomicOr(b.flags, 2); return; }
    const int node = stack[--sp_];
    const float4* r = b.rec + 4 * node;
    const float4 r0 = __ldg(r), r1 = __ldg(r + 1), r2 = __ldg(r + 2), r3 = __ldg(r + 3);
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const float4 lo = c == 0 ? r0 : r2, hi = c == 0 ? r1 : r3;
      if (!ov_rec(qbox, lo, hi)) continue;
      const int code = __float_as_int(lo.w);
      if (code < 0) {
        const int tL = ~code;
        if (tL > q && !share_vertex(b.idx, q, tL) && (mirror || ov6d(q64, b.box64 + (size_t)tL * 6))) {
          if (MODE == 1) b.pairs[out++] = make_int2(q, tL);
          if (MODE == 2) {
            buf[nbuf++] = make_int2(q, tL);
            if (nbuf == kLocalPairs) { flush_pairs(b.pairs, b.pairCap, b.cnt, buf, nbuf); nbuf = 0; }
          }
          count++;
        }
      } else {
        if (sp_ >= kStack) { atomicOr(b.flags, 1); return; }
        stack[sp_++] = code;
      }
    }
  }
  if (MODE == 0) b.cnt[s] = count;
  if (MODE == 2) flush_pairs(b.pairs, b.pairCap, b.cnt, buf, nbuf);
}

// Static triangles against the cloth hierarchy (contact-assembly.ts:96-140):
// box = f32 static vertices in f64 +- pad (static, not swept).
__device__ __forceinline__ void static_box(const BvhBufs& b, int st, double pad, double* o) {
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int q = 0; q < 3; q++) {
    const uint32_t v = b.sidx[st * 3 + q];
    for (int k = 0; k < 3; k++) {
      const double c = b.spos[v * 3 + k];
      mn[k] = js_min(mn[k], c);
      mx[k] = js_max(mx[k], c);
    }
  }
  for (int k = 0; k < 3; k++) { o[k] = mn[k] - pad; o[3 + k] = mx[k] + pad; }
}

__global__ void __launch_bounds__(128) k_static(BvhBufs b, const uint32_t* sp, double pad, int2* outp, uint32_t cap,
                                                uint32_t* counter) {
  const int st = blockIdx.x * blockDim.x + threadIdx.x;
  if (st >= b.ms) return;
  const int m = b.m;
  double s64[6];
  static_box(b, st, pad, s64);
  float sb[6];
  for (int k = 0; k < 3; k++) { sb[k] = __double2float_rd(s64[k]); sb[3 + k] = __double2float_ru(s64[3 + k]); }
  int2 buf[kLocalPairs];
  int nbuf = 0;
  int stack[kStack];
  int sp_ = 0;
  if (m == 1) {
    if (ov6d(b.box64, s64)) buf[nbuf++] = make_int2(0, st);
  } else {
    const int root = *b.root;
    // the root itself is tested too (queryBvhAll tests every popped node)
    if (ov6(sb, b.nbox + (size_t)root * 6)) stack[sp_++] = root;
  }
  long guard = 0;
  while (sp_ > 0) {
    if (++guard > 4l * m + 8) { atomicOr(b.flags, 2); return; }
    const int node = stack[--sp_];
    const float4* r = b.rec + 4 * node;
    const float4 r0 = __ldg(r), r1 = __ldg(r + 1), r2 = __ldg(r + 2), r3 = __ldg(r + 3);
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const float4 lo = c == 0 ? r0 : r2, hi = c == 0 ? r1 : r3;
      if (!ov_rec(sb, lo, hi)) continue;
      const int code = __float_as_int(lo.w);
      if (code < 0) {
        const int tL = ~code;
        if (ov6d(b.box64 + (size_t)tL * 6, s64)) {
          buf[nbuf++] = make_int2(tL, st);
          if (nbuf == kLocalPairs) { flush_pairs(outp, cap, counter, buf, nbuf); nbuf = 0; }
        }
      } else {
        if (sp_ >= kStack) { atomicOr(b.flags, 1); return; }
        stack[sp_++] = code;
      }
    }
  }
  flush_pairs(outp, cap, counter, buf, nbuf);
}

void scan_counts(uint32_t* cnt, int n, uint32_t* total, cudaStream_t s, int64_t* launches) {
  k_scan_exclusive<<<1, 1024, 0, s>>>(cnt, n, total);
  if (launches) *launches += 1;
}

static void boxes_and_refit(BvhBufs& b, const double* x0, const double* x1, double pad, bool mirror, cudaStream_t s,
                            int64_t* launches) {
  const int m = b.m;
  k_boxes<<<nb(m), kBT, 0, s>>>(b, x0, x1, pad);
  k_refit_init<<<nb(2 * m - 1), kBT, 0, s>>>(b);
  k_refit<<<nb(m), kBT, 0, s>>>(b, b.p0, mirror);
  *launches += 3;
}

void bvh_build(BvhBufs& b, const double* x0, const double* x1, double pad, bool mirror, cudaStream_t s,
               int64_t* launches) {
  const int m = b.m;
  k_boxes<<<nb(m), kBT, 0, s>>>(b, x0, x1, pad);
  k_scene_bounds<<<1, 1024, 0, s>>>(b);
  k_morton<<<nb(m), kBT, 0, s>>>(b);
  *launches += 3;
  const bool flip = radix_sort<1>(b.k0, b.p0, b.k1, b.p1, m, 30, b.hist, s, launches);
  if (flip) {  // keep the sorted result in (k0, p0)
    cudaMemcpyAsync(b.k0, b.k1, (size_t)m * sizeof(Key<1>), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(b.p0, b.p1, (size_t)m * 4, cudaMemcpyDeviceToDevice, s);
  }
  k_topo_init<<<nb(2 * m - 1), kBT, 0, s>>>(b);
  *launches += 1;
  cudaMemsetAsync(b.root, 0, sizeof(int), s);
  if (m > 1) {
    k_karras<<<nb(m - 1), kBT, 0, s>>>(b, b.k0, b.p0);
    *launches += 1;
  }
  k_refit_init<<<nb(2 * m - 1), kBT, 0, s>>>(b);
  k_refit<<<nb(m), kBT, 0, s>>>(b, b.p0, mirror);
  *launches += 2;
}

void bvh_refit(BvhBufs& b, const double* x0, const double* x1, double pad, bool mirror, cudaStream_t s,
               int64_t* launches) {
  boxes_and_refit(b, x0, x1, pad, mirror, s, launches);
}

static inline int nq(int n) { return (n + 127) / 128; }

void bvh_boxes(BvhBufs& b, const double* x0, const double* x1, double pad, cudaStream_t s, int64_t* launches) {
  k_boxes<<<nb(b.m), kBT, 0, s>>>(b, x0, x1, pad);
  *launches += 1;
}

// Warp-aggregated append of kept pairs.
__device__ __forceinline__ void append_pair(bool keep, int2 pr, int2* out, uint32_t cap, uint32_t* cnt) {
  const uint32_t mask = __ballot_sync(0xffffffffu, keep);
  if (!mask) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(cnt, (uint32_t)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (keep) {
    const uint32_t slot = base + __popc(mask & ((1u << lane) - 1u));
    if (slot < cap) out[slot] = pr;
  }
}

__global__ void __launch_bounds__(256) k_filter_self(BvhBufs b, const int2* sup, int nsup, int2* out, uint32_t cap,
                                                     uint32_t* cnt, const int* dn = nullptr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (dn) nsup = min(nsup, *dn);
  bool keep = false;
  int2 pr = make_int2(0, 0);
  if (i < nsup) {
    pr = sup[i];
    keep = ov6d(b.box64 + (size_t)pr.x * 6, b.box64 + (size_t)pr.y * 6);
  }
  append_pair(keep, pr, out, cap, cnt);
}

__global__ void __launch_bounds__(256) k_filter_static(BvhBufs b, const int2* sup, int nsup, double pad, int2* out,
                                                       uint32_t cap, uint32_t* cnt, const int* dn = nullptr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (dn) nsup = min(nsup, *dn);
  bool keep = false;
  int2 pr = make_int2(0, 0);
  if (i < nsup) {
    pr = sup[i];
    double s64[6];
    static_box(b, pr.y, pad, s64);
    keep = ov6d(b.box64 + (size_t)pr.x * 6, s64);
  }
  append_pair(keep, pr, out, cap, cnt);
}

void filter_pairs(const BvhBufs& b, const int2* sup, int nsup, int2* out, uint32_t cap, uint32_t* cnt,
                  const int2* ssup, int nssup, double pad, int2* sout, uint32_t scap, uint32_t* scnt, cudaStream_t s,
                  int64_t* launches) {
  if (nsup > 0) {
    k_filter_self<<<(nsup + 255) / 256, 256, 0, s>>>(b, sup, nsup, out, cap, cnt);
    *launches += 1;
  }
  if (nssup > 0) {
    k_filter_static<<<(nssup + 255) / 256, 256, 0, s>>>(b, ssup, nssup, pad, sout, scap, scnt);
    *launches += 1;
  }
}

// The same filter with the superset sizes read on the device (dn[0] self,
// dn[1] static pairs), launched for the capacities nsup / nssup.
void filter_pairs_dev(const BvhBufs& b, const int2* sup, int nsup, int2* out, uint32_t cap, uint32_t* cnt,
                      const int2* ssup, int nssup, double pad, int2* sout, uint32_t scap, uint32_t* scnt,
                      const int* dn, cudaStream_t s, int64_t* launches) {
  if (nsup > 0) {
    k_filter_self<<<(nsup + 255) / 256, 256, 0, s>>>(b, sup, nsup, out, cap, cnt, dn);
    *launches += 1;
  }
  if (nssup > 0) {
    k_filter_static<<<(nssup + 255) / 256, 256, 0, s>>>(b, ssup, nssup, pad, sout, scap, scnt, dn + 1);
    *launches += 1;
  }
}

void bvh_count_self(BvhBufs& b, bool mirror, cudaStream_t s, int64_t* launches) {
  if (b.m < 2) {
    cudaMemsetAsync(b.cnt, 0, (size_t)(b.m + 1) * 4, s);
    return;
  }
  k_self<0><<<nq(b.m), 128, 0, s>>>(b, b.p0, mirror);
  *launches += 1;
}
void bvh_emit_self(BvhBufs& b, bool mirror, cudaStream_t s, int64_t* launches) {
  if (b.m < 2) return;
  k_self<1><<<nq(b.m), 128, 0, s>>>(b, b.p0, mirror);
  *launches += 1;
}
void bvh_append_self(BvhBufs& b, cudaStream_t s, int64_t* launches) {
  if (b.m < 2) return;
  k_self<2><<<nq(b.m), 128, 0, s>>>(b, b.p0, false);
  *launches += 1;
}
void bvh_append_static(BvhBufs& b, double pad, int2* out, uint32_t cap, uint32_t* cnt, cudaStream_t s,
                       int64_t* launches) {
  if (b.ms <= 0) return;
  k_static<<<nq(b.ms), 128, 0, s>>>(b, b.p0, pad, out, cap, cnt);
  *launches += 1;
}

}  // namespace cs
