// Stand-alone broadphase handle behind the reference's BroadPhase interface
// (src/collision/broadphase.ts:61-64, GpuBroadPhase in
// src/backend/webgpu/gpu-broadphase.ts:147-386): build(x0, x1) over positions
// already resident on the device, returning the sorted candidate triangle
// pairs, the diagnostics block and the LBVH state the reference keeps as
// lastMirror (boxes, centroids, sorted Morton keys and payload, node boxes and
// topology, root, depth).
//
// Two pair sets are offered:
//   CS_BROADPHASE_MIRROR  the FP32 mirror's set: node and leaf tests on the
//                         FP32 boxes, as GpuBroadPhase (gpu-broadphase.ts:321-357);
//   CS_BROADPHASE_EXACT   the CPU BVH's set (src/collision/bvh.ts:79-124): tree
//                         tests on outward-rounded f32 boxes, every leaf hit
//                         re-tested on the f64 boxes (the set the FP64 contact
//                         path uses).
// Pairs are emitted per sorted leaf in the reference's stack order, cut at the
// capacity in that order, then sorted by (a, b) on the device, so even an
// overflowing build returns the reference's pairs.
#include <algorithm>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/closim_broadphase.h"
#include "broadphase.cuh"
#include "common.cuh"

namespace cs {
namespace {

struct BpError : std::runtime_error {
  int code;
  BpError(int c, const std::string& s) : std::runtime_error(s), code(c) {}
};

#define BPK(call)                                                                    \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) throw cs::BpError(CS_E_CUDA, cudaGetErrorString(e_));     \
  } while (0)

template <class T>
void bp_alloc(T*& p, size_t n) {
  if (p) cudaFree(p);
  p = nullptr;
  if (n) BPK(cudaMalloc(&p, n * sizeof(T)));
}
template <class T>
void bp_free(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

constexpr int kBpT = 256;

__global__ void k_pair_keys(const int2* pairs, int w, Key<2>* keys, uint32_t* pay) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w) return;
  keys[i].w[0] = (uint32_t)pairs[i].x;
  keys[i].w[1] = (uint32_t)pairs[i].y;
  pay[i] = (uint32_t)i;
}

}  // namespace

struct Broadphase {
  int n = 0, m = 0, mode = CS_BROADPHASE_MIRROR;
  double pad = 0;
  int64_t capacity = 0;
  cudaStream_t stream = nullptr;
  BvhBufs b;
  uint32_t* idx = nullptr;
  int* flags = nullptr;
  uint32_t* total = nullptr;
  Key<2>* pk0 = nullptr; Key<2>* pk1 = nullptr;
  uint32_t* pp0 = nullptr; uint32_t* pp1 = nullptr; uint32_t* phist = nullptr;
  size_t pairCap = 0;
  const Key<2>* sortedPairs = nullptr;
  int64_t scanned = 0, written = 0;
  int overflow = 0, depth = 0, root = 0;
  bool built = false;
  std::string err;

  ~Broadphase() {
    for (void** q : {(void**)&idx, (void**)&flags, (void**)&total, (void**)&pk0, (void**)&pk1, (void**)&pp0,
                     (void**)&pp1, (void**)&phist, (void**)&b.box64, (void**)&b.boxc, (void**)&b.boxr,
                     (void**)&b.cent, (void**)&b.scene, (void**)&b.k0, (void**)&b.k1, (void**)&b.p0,
                     (void**)&b.p1, (void**)&b.hist, (void**)&b.left, (void**)&b.right, (void**)&b.parent,
                     (void**)&b.depth, (void**)&b.nbox, (void**)&b.rec, (void**)&b.visit, (void**)&b.root, (void**)&b.cnt,
                     (void**)&b.pairs})
      if (*q) { cudaFree(*q); *q = nullptr; }
    if (stream) cudaStreamDestroy(stream);
  }

  void init(int nv, int mt, const uint32_t* hidx, double pd, int64_t cap, int md) {
    n = nv; m = mt; pad = pd; capacity = cap; mode = md;
    BPK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    const size_t nn = (size_t)std::max(1, 2 * m - 1);
    bp_alloc(idx, 3 * (size_t)m);
    BPK(cudaMemcpy(idx, hidx, 3 * (size_t)m * 4, cudaMemcpyHostToDevice));
    b.m = m; b.ns = 0; b.ms = 0; b.idx = idx;
    bp_alloc(b.box64, 6 * (size_t)m);
    bp_alloc(b.boxc, 6 * (size_t)m);
    bp_alloc(b.boxr, 6 * (size_t)m);
    bp_alloc(b.cent, 3 * (size_t)m);
    bp_alloc(b.scene, 6);
    bp_alloc(b.k0, (size_t)m);
    bp_alloc(b.k1, (size_t)m);
    bp_alloc(b.p0, (size_t)m);
    bp_alloc(b.p1, (size_t)m);
    bp_alloc(b.hist, 256 * (size_t)((m + kSortTile - 1) / kSortTile) + 1);
    bp_alloc(b.left, nn);
    bp_alloc(b.right, nn);
    bp_alloc(b.parent, nn);
    bp_alloc(b.depth, nn);
    bp_alloc(b.nbox, 6 * nn);
    bp_alloc(b.rec, 4 * (size_t)std::max(1, m - 1));
    bp_alloc(b.visit, nn);
    bp_alloc(b.root, 1);
    bp_alloc(b.cnt, (size_t)m + 1);
    bp_alloc(flags, 4);
    bp_alloc(total, 4);
    b.flags = flags;
  }

  void ensure_pairs(size_t np) {
    if (np <= pairCap) return;
    pairCap = np + np / 2 + 64;
    bp_alloc(b.pairs, pairCap);
    bp_alloc(pk0, pairCap);
    bp_alloc(pk1, pairCap);
    bp_alloc(pp0, pairCap);
    bp_alloc(pp1, pairCap);
    bp_alloc(phist, 256 * ((pairCap + kSortTile - 1) / kSortTile) + 1);
  }

  void build(const double* x0, const double* x1) {
    built = false;
    scanned = written = 0;
    overflow = 0;
    depth = m > 0 ? 1 : 0;
    root = 0;
    if (m == 0) { built = true; return; }
    int64_t lc = 0;
    const bool mirror = mode == CS_BROADPHASE_MIRROR;
    BPK(cudaMemsetAsync(flags, 0, 4 * sizeof(int), stream));
    BPK(cudaMemsetAsync(total, 0, 4 * sizeof(uint32_t), stream));
    bvh_build(b, x0, x1, pad, mirror, stream, &lc);
    bvh_count_self(b, mirror, stream, &lc);
    scan_counts(b.cnt, m, total, stream, &lc);
    int hflags[4];
    uint32_t htotal[4];
    BPK(cudaMemcpyAsync(hflags, flags, sizeof hflags, cudaMemcpyDeviceToHost, stream));
    BPK(cudaMemcpyAsync(htotal, total, sizeof htotal, cudaMemcpyDeviceToHost, stream));
    BPK(cudaMemcpyAsync(&root, b.root, sizeof(int), cudaMemcpyDeviceToHost, stream));
    BPK(cudaStreamSynchronize(stream));
    BPK(cudaMemcpy(&depth, b.depth + root, sizeof(int), cudaMemcpyDeviceToHost));
    if (hflags[0]) throw BpError(CS_E_CAPACITY, "LBVH traversal aborted (stack deeper than 64 or malformed tree)");
    scanned = htotal[0];
    written = std::min<int64_t>(scanned, capacity);
    overflow = scanned > capacity ? 1 : 0;
    ensure_pairs((size_t)std::max<int64_t>(scanned, 1));
    if (scanned > 0) bvh_emit_self(b, mirror, stream, &lc);
    sortedPairs = pk0;
    if (written > 0) {
      const int w = (int)written;
      k_pair_keys<<<(w + kBpT - 1) / kBpT, kBpT, 0, stream>>>(b.pairs, w, pk0, pp0);
      int bits = 32;
      while ((1ll << (bits - 32)) < m) bits++;
      const bool flip = radix_sort<2>(pk0, pp0, pk1, pp1, w, bits, phist, stream, &lc);
      sortedPairs = flip ? pk1 : pk0;
    }
    BPK(cudaGetLastError());
    BPK(cudaStreamSynchronize(stream));
    built = true;
  }
};

}  // namespace cs

namespace {

template <class F>
int bp_guarded(cs::Broadphase* h, F&& f) {
  if (!h) return CS_E_ARG;
  try {
    f();
    h->err.clear();
    return CS_OK;
  } catch (const cs::BpError& e) {
    h->err = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    h->err = "host allocation failed";
    return CS_E_CAPACITY;
  } catch (const std::exception& e) {
    h->err = e.what();
    return CS_E_CUDA;
  }
}

}  // namespace

extern "C" {

cs_broadphase* cs_broadphase_create(int32_t n, int32_t m, const uint32_t* indices, double pad, int64_t pair_capacity,
                                    int32_t mode) {
  if (n < 0 || m < 0 || (m > 0 && !indices) || pair_capacity < 0) return nullptr;
  if (mode != CS_BROADPHASE_MIRROR && mode != CS_BROADPHASE_EXACT) return nullptr;
  // The reference decodes exclusion keys as min*1000003+max (gpu-broadphase.ts:160-166).
  if (m >= 1000003) return nullptr;
  for (int64_t i = 0; i < 3ll * m; i++)
    if ((int64_t)indices[i] >= n) return nullptr;
  cs::Broadphase* h = nullptr;
  try {
    h = new cs::Broadphase();
    h->init(n, m, indices, pad, pair_capacity, mode);
  } catch (...) {
    delete h;
    return nullptr;
  }
  return reinterpret_cast<cs_broadphase*>(h);
}

void cs_broadphase_destroy(cs_broadphase* bp) { delete reinterpret_cast<cs::Broadphase*>(bp); }

const char* cs_broadphase_last_error(cs_broadphase* bp) {
  return bp ? reinterpret_cast<cs::Broadphase*>(bp)->err.c_str() : "null broadphase handle";
}

int cs_broadphase_build(cs_broadphase* bp, const double* x0, const double* x1) {
  cs::Broadphase* h = reinterpret_cast<cs::Broadphase*>(bp);
  if (h && h->m > 0 && (!x0 || !x1)) return CS_E_ARG;
  return bp_guarded(h, [&] { h->build(x0, x1); });
}

int cs_broadphase_diagnostics(cs_broadphase* bp, cs_broadphase_diag* out) {
  cs::Broadphase* h = reinterpret_cast<cs::Broadphase*>(bp);
  if (!h || !out) return CS_E_ARG;
  if (!h->built) return CS_E_UNINIT;
  out->scanned_count = h->scanned;
  out->written_count = h->written;
  out->capacity = h->capacity;
  out->candidate_overflow = h->overflow;
  out->tree_depth = h->depth;
  out->root = h->root;
  out->reserved = 0;
  return CS_OK;
}

int cs_broadphase_pairs(cs_broadphase* bp, int32_t* pairs) {
  cs::Broadphase* h = reinterpret_cast<cs::Broadphase*>(bp);
  if (!h || (!pairs && h->written > 0)) return CS_E_ARG;
  if (!h->built) return CS_E_UNINIT;
  return bp_guarded(h, [&] {
    if (h->written == 0) return;
    static_assert(sizeof(cs::Key<2>) == 8, "pair key is two u32 words");
    BPK(cudaMemcpy(pairs, h->sortedPairs, (size_t)h->written * 8, cudaMemcpyDeviceToHost));
  });
}

int cs_broadphase_state(cs_broadphase* bp, float* aabb, float* centroid, uint32_t* morton, uint32_t* payload,
                        float* node_min, float* node_max, int32_t* node_left, int32_t* node_right,
                        int32_t* node_leaf_tri) {
  cs::Broadphase* h = reinterpret_cast<cs::Broadphase*>(bp);
  if (!h) return CS_E_ARG;
  if (!h->built) return CS_E_UNINIT;
  return bp_guarded(h, [&] {
    const int m = h->m;
    if (m == 0) return;
    const size_t nn = (size_t)std::max(1, 2 * m - 1);
    auto d2h = [](void* dst, const void* src, size_t bytes) {
      if (dst && bytes) BPK(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
    };
    d2h(aabb, h->b.boxr, (size_t)m * 6 * 4);
    d2h(centroid, h->b.cent, (size_t)m * 3 * 4);
    static_assert(sizeof(cs::Key<1>) == 4, "Morton key is one u32 word");
    d2h(morton, h->b.k0, (size_t)m * 4);
    std::vector<uint32_t> pay(m);
    d2h(pay.data(), h->b.p0, (size_t)m * 4);
    if (payload) std::memcpy(payload, pay.data(), (size_t)m * 4);
    if (node_min || node_max) {
      std::vector<float> box(nn * 6);
      d2h(box.data(), h->b.nbox, box.size() * 4);
      for (size_t i = 0; i < nn; i++)
        for (int k = 0; k < 3; k++) {
          if (node_min) node_min[i * 3 + k] = box[i * 6 + k];
          if (node_max) node_max[i * 3 + k] = box[i * 6 + 3 + k];
        }
    }
    // Internal nodes 0..m-2 (Karras order), leaves m-1.. in sorted order; a
    // single triangle is one leaf at slot 0.
    std::vector<int32_t> l(nn, -1), r(nn, -1);
    if (m > 1) {
      d2h(l.data(), h->b.left, (size_t)(m - 1) * 4);
      d2h(r.data(), h->b.right, (size_t)(m - 1) * 4);
    }
    if (node_left) std::memcpy(node_left, l.data(), nn * 4);
    if (node_right) std::memcpy(node_right, r.data(), nn * 4);
    if (node_leaf_tri) {
      for (size_t i = 0; i < nn; i++) node_leaf_tri[i] = -1;
      for (int s = 0; s < m; s++) node_leaf_tri[(m > 1 ? m - 1 : 0) + s] = (int32_t)pay[s];
    }
  });
}

}  // extern "C"
