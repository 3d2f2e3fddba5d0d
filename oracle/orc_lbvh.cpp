// Oracle (test infrastructure only): the FP32 LBVH broadphase mirror of
// src/backend/webgpu/gpu-broadphase.ts:54-386 (swept AABB, centroid, 30-bit
// Morton key, (key, triId) sort, Karras 2012 hierarchy, span-ordered refit,
// per-leaf traversal with exclusion, sorted + deduplicated pairs).
// Math.fround(a op b) on f32 inputs equals the IEEE single-precision result,
// so float arithmetic here reproduces the mirror exactly.
#include <algorithm>
#include <numeric>
#include <stdexcept>

#include "orc.hpp"

namespace orc {

// gpu-broadphase.ts:95-102 expand10.
static uint32_t expand10(uint32_t v) {
  uint32_t x = v & 1023;
  x = (x | (x << 16)) & 0x030000ff;
  x = (x | (x << 8)) & 0x0300f00f;
  x = (x | (x << 4)) & 0x030c30c3;
  x = (x | (x << 2)) & 0x09249249;
  return x;
}

// gpu-broadphase.ts:105-117 mortonKeyOf. span = max(f32 span, 1e-9) where 1e-9 is
// a double; n = fround(fround(c - min) / span), quantized by floor(n * 1023) in f64.
uint32_t morton_key_of(const float c[3], const float sMin[3], const float sMax[3]) {
  uint32_t q[3];
  for (int k = 0; k < 3; k++) {
    const double span = js_max((double)(float)(sMax[k] - sMin[k]), 1e-9);
    const float dc = c[k] - sMin[k];
    const double nn = js_min(1, js_max(0, (double)(float)((double)dc / span)));
    q[k] = (uint32_t)std::floor(nn * 1023);
  }
  return (expand10(q[0]) << 2) | (expand10(q[1]) << 1) | expand10(q[2]);
}

static inline int clz32(uint32_t v) { return v == 0 ? 32 : __builtin_clz(v); }

// gpu-broadphase.ts:140-145 deltaPos (sorted-position tiebreak).
static int delta_pos(const std::vector<uint32_t>& keys, long p, long q, long n) {
  if (q < 0 || q >= n) return -1;
  const uint32_t kp = keys[p], kq = keys[q];
  if (kp != kq) return clz32(kp ^ kq);
  return 32 + clz32((uint32_t)(p ^ q));
}

void lbvh_mirror_build(const double* x0, const double* x1, const uint32_t* idx, int m, double pad,
                       const std::vector<int64_t>& excl, long capacity, LbvhMirror& o) {
  o = LbvhMirror();
  o.aabb.assign((size_t)m * 6, 0.f);
  o.centroid.assign((size_t)m * 3, 0.f);
  if (m == 0) return;
  float sMin[3] = {INFINITY, INFINITY, INFINITY}, sMax[3] = {-INFINITY, -INFINITY, -INFINITY};
  const float p = fr(pad);
  for (int t = 0; t < m; t++) {
    const int ids[3] = {(int)idx[t * 3], (int)idx[t * 3 + 1], (int)idx[t * 3 + 2]};
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int v : ids) {
      const double* xs[2] = {x0, x1};
      for (const double* x : xs)
        for (int k = 0; k < 3; k++) {
          const float c = fr(x[v * 3 + k]);
          if (c < mn[k]) mn[k] = c;
          if (c > mx[k]) mx[k] = c;
        }
    }
    for (int k = 0; k < 3; k++) {
      o.aabb[t * 6 + k] = mn[k] - p;
      o.aabb[t * 6 + 3 + k] = mx[k] + p;
    }
    for (int k = 0; k < 3; k++) {
      float s = 0.f;
      for (int v : ids) {
        s = s + fr(x0[v * 3 + k]);
        s = s + fr(x1[v * 3 + k]);
      }
      const float c = s / 6.f;
      o.centroid[t * 3 + k] = c;
      if (c < sMin[k]) sMin[k] = c;
      if (c > sMax[k]) sMax[k] = c;
    }
  }
  std::vector<uint32_t> keys(m), payload(m);
  for (int t = 0; t < m; t++) {
    keys[t] = morton_key_of(&o.centroid[t * 3], sMin, sMax);
    payload[t] = t;
  }
  std::vector<int> order(m);
  std::iota(order.begin(), order.end(), 0);
  std::sort(order.begin(), order.end(), [&](int a, int b) {
    return keys[a] != keys[b] ? keys[a] < keys[b] : payload[a] < payload[b];
  });
  o.morton.resize(m);
  o.payload.resize(m);
  for (int s = 0; s < m; s++) { o.morton[s] = keys[order[s]]; o.payload[s] = payload[order[s]]; }
  const long nodeCount = std::max(1, 2 * m - 1);
  o.nodeMin.assign(nodeCount * 3, 0.f);
  o.nodeMax.assign(nodeCount * 3, 0.f);
  o.nodeLeft.assign(nodeCount, -1);
  o.nodeRight.assign(nodeCount, -1);
  o.nodeLeafTri.assign(nodeCount, -1);
  o.root = 0;
  o.depth = 1;
  if (m == 1) {
    for (int k = 0; k < 3; k++) { o.nodeMin[k] = o.aabb[k]; o.nodeMax[k] = o.aabb[3 + k]; }
    o.nodeLeafTri[0] = o.payload[0];
  } else {
    for (int s = 0; s < m; s++) {
      const long slot = m - 1 + s;
      const uint32_t tri = o.payload[s];
      for (int k = 0; k < 3; k++) {
        o.nodeMin[slot * 3 + k] = o.aabb[tri * 6 + k];
        o.nodeMax[slot * 3 + k] = o.aabb[tri * 6 + 3 + k];
      }
      o.nodeLeafTri[slot] = (int32_t)tri;
    }
    std::vector<std::pair<long, long>> ranges(m - 1);
    const auto& sk = o.morton;
    for (long i = 0; i < m - 1; i++) {
      const int dNext = delta_pos(sk, i, i + 1, m);
      const int dPrev = delta_pos(sk, i, i - 1, m);
      long d = 1;
      int dMin = dPrev;
      if (dPrev > dNext) { d = -1; dMin = dNext; }
      long lMax = 2;
      while (delta_pos(sk, i, i + d * lMax, m) > dMin) {
        lMax *= 2;
        if (lMax > m) break;
      }
      long l = 0, t = lMax / 2;
      while (t > 0) {
        if (delta_pos(sk, i, i + d * (l + t), m) > dMin) l += t;
        t /= 2;
      }
      const long j = i + d * l;
      const long lo = std::min(i, j), hi = std::max(i, j);
      const int dNode = delta_pos(sk, lo, hi, m);
      long split = lo, stride = 1;
      while (stride * 2 <= hi - lo) stride *= 2;
      while (stride > 0) {
        const long mid = split + stride;
        if (mid < hi && delta_pos(sk, lo, mid, m) > dNode) split = mid;
        stride /= 2;
      }
      ranges[i] = {lo, hi};
      o.nodeLeft[i] = (int32_t)(split == lo ? m - 1 + lo : split);
      o.nodeRight[i] = (int32_t)(split + 1 == hi ? m - 1 + split + 1 : split + 1);
      if (lo == 0 && hi == m - 1) o.root = (int)i;
    }
    std::vector<long> internal(m - 1);
    std::iota(internal.begin(), internal.end(), 0);
    // JS Array.prototype.sort is stable: equal spans keep ascending id order.
    std::stable_sort(internal.begin(), internal.end(), [&](long a, long b) {
      return (ranges[a].second - ranges[a].first) < (ranges[b].second - ranges[b].first);
    });
    std::vector<int> depths(m - 1, 1);
    int maxDepth = 1;
    for (long i : internal) {
      const int L = o.nodeLeft[i], R = o.nodeRight[i];
      for (int k = 0; k < 3; k++) {
        o.nodeMin[i * 3 + k] = std::min(o.nodeMin[L * 3 + k], o.nodeMin[R * 3 + k]);
        o.nodeMax[i * 3 + k] = std::max(o.nodeMax[L * 3 + k], o.nodeMax[R * 3 + k]);
      }
      const int dL = o.nodeLeafTri[L] >= 0 ? 1 : depths[L];
      const int dR = o.nodeLeafTri[R] >= 0 ? 1 : depths[R];
      const int dd = std::max(dL, dR) + 1;
      depths[i] = dd;
      if (dd > maxDepth) maxDepth = dd;
    }
    o.depth = maxDepth;
    if (o.depth > 64) throw std::runtime_error("LBVH depth exceeds traverse stack (64)");
  }
  auto ov = [&](long q, long nn) {
    return o.nodeMin[q * 3] <= o.nodeMax[nn * 3] && o.nodeMax[q * 3] >= o.nodeMin[nn * 3] &&
           o.nodeMin[q * 3 + 1] <= o.nodeMax[nn * 3 + 1] && o.nodeMax[q * 3 + 1] >= o.nodeMin[nn * 3 + 1] &&
           o.nodeMin[q * 3 + 2] <= o.nodeMax[nn * 3 + 2] && o.nodeMax[q * 3 + 2] >= o.nodeMin[nn * 3 + 2];
  };
  std::vector<std::pair<int, int>> emitted;
  long scanned = 0;
  if (m > 1) {
    std::vector<int> stack;
    for (long s = 0; s < m; s++) {
      const int qTri = (int)o.payload[s];
      const long qSlot = m - 1 + s;
      stack.assign(1, o.root);
      while (!stack.empty()) {
        const int node = stack.back();
        stack.pop_back();
        const int ch[2] = {o.nodeLeft[node], o.nodeRight[node]};
        for (int child : ch) {
          if (!ov(qSlot, child)) continue;
          if (o.nodeLeafTri[child] >= 0) {
            const int tL = o.nodeLeafTri[child];
            const int64_t key = (int64_t)std::min(qTri, tL) * 1000003 + std::max(qTri, tL);
            if (tL > qTri && !std::binary_search(excl.begin(), excl.end(), key)) {
              scanned++;
              if ((long)emitted.size() < capacity) emitted.push_back({qTri, tL});
            }
          } else {
            stack.push_back(child);
          }
        }
      }
    }
  }
  o.scanned = scanned;
  o.overflow = scanned > capacity ? 1 : 0;
  std::sort(emitted.begin(), emitted.end());
  emitted.erase(std::unique(emitted.begin(), emitted.end()), emitted.end());
  o.pairs = std::move(emitted);
}

}  // namespace orc
