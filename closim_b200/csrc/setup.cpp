// Host-side set-up for the CUDA cloth solver: mesh preprocessing (the data
// the reference's ClothMeshData carries), element-ordered CSR incidence, and
// the static one-level Schwarz domain topology. Runs once per mesh.
#include "setup.hpp"

#include <algorithm>
#include <cmath>
#include <deque>
#include <set>
#include <stdexcept>
#include <unordered_map>

namespace cs {

static inline double jmax(double a, double b) { return (a != a || b != b) ? a + b : (a > b ? a : b); }
static inline double jmin(double a, double b) { return (a != a || b != b) ? a + b : (a < b ? a : b); }

// Math.hypot(a, b, c) as V8 evaluates it (max scaling + Kahan-compensated squares).
double hypot3_js(double a, double b, double c) {
  if (std::isinf(a) || std::isinf(b) || std::isinf(c)) return INFINITY;
  if (a != a || b != b || c != c) return NAN;
  const double v[3] = {std::fabs(a), std::fabs(b), std::fabs(c)};
  double mx = 0;
  for (double t : v) if (t > mx) mx = t;
  if (mx == 0) return 0;
  double sum = 0, comp = 0;
  for (double t : v) {
    const double q = t / mx;
    const double summand = q * q - comp;
    const double pre = sum + summand;
    comp = (pre - sum) - summand;
    sum = pre;
  }
  return std::sqrt(sum) * mx;
}

// src/mesh/mesh.ts:17-48: (nx+1)(ny+1) vertices in the XZ plane at y = 0.
void grid_mesh(int nx, int ny, double w, double h, std::vector<float>& pos, std::vector<float>& uv,
               std::vector<uint32_t>& idx) {
  const int n = (nx + 1) * (ny + 1);
  pos.assign((size_t)n * 3, 0.f);
  uv.assign((size_t)n * 2, 0.f);
  for (int j = 0; j <= ny; j++)
    for (int i = 0; i <= nx; i++) {
      const int id = j * (nx + 1) + i;
      const float x = (float)(((double)i / nx) * w), z = (float)(((double)j / ny) * h);
      pos[id * 3] = x; pos[id * 3 + 2] = z;
      uv[id * 2] = x; uv[id * 2 + 1] = z;
    }
  idx.clear();
  idx.reserve((size_t)nx * ny * 6);
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      const uint32_t a = j * (nx + 1) + i, b = a + 1, c = a + (nx + 1), d = c + 1;
      for (uint32_t q : {a, c, b, b, c, d}) idx.push_back(q);
    }
}

static double dihedral_f(const float* x, int v0, int v1, int v2, int v3) {
  auto X = [&](int v, int k) { return (double)x[v * 3 + k]; };
  const double e0x = X(v1, 0) - X(v0, 0), e0y = X(v1, 1) - X(v0, 1), e0z = X(v1, 2) - X(v0, 2);
  const double e1x = X(v2, 0) - X(v0, 0), e1y = X(v2, 1) - X(v0, 1), e1z = X(v2, 2) - X(v0, 2);
  const double e2x = X(v3, 0) - X(v0, 0), e2y = X(v3, 1) - X(v0, 1), e2z = X(v3, 2) - X(v0, 2);
  const double n1x = e0y * e1z - e0z * e1y, n1y = e0z * e1x - e0x * e1z, n1z = e0x * e1y - e0y * e1x;
  const double n2x = e0y * e2z - e0z * e2y, n2y = e0z * e2x - e0x * e2z, n2z = e0x * e2y - e0y * e2x;
  const double l1 = hypot3_js(n1x, n1y, n1z) + 1e-30, l2 = hypot3_js(n2x, n2y, n2z) + 1e-30;
  const double c = jmin(1, jmax(-1, (n1x * n2x + n1y * n2y + n1z * n2z) / (l1 * l2)));
  return std::acos(c);
}

// src/mesh/mesh.ts:50-126: Dm^-1, areas, lumped masses (Float32) and hinges.
void preprocess_mesh(const std::vector<float>& pos, const std::vector<float>& uv,
                     const std::vector<uint32_t>& idx, double density, HostMesh& out) {
  const int n = (int)pos.size() / 3, m = (int)idx.size() / 3;
  out.n = n; out.m = m;
  out.idx = idx;
  out.rest = pos;
  out.inv.assign((size_t)m * 4, 0.f);
  out.area.assign(m, 0.f);
  out.mass.assign(n, 0.f);
  for (int t = 0; t < m; t++) {
    const uint32_t i0 = idx[t * 3], i1 = idx[t * 3 + 1], i2 = idx[t * 3 + 2];
    const double du1 = (double)uv[i1 * 2] - uv[i0 * 2], dv1 = (double)uv[i1 * 2 + 1] - uv[i0 * 2 + 1];
    const double du2 = (double)uv[i2 * 2] - uv[i0 * 2], dv2 = (double)uv[i2 * 2 + 1] - uv[i0 * 2 + 1];
    const double det = du1 * dv2 - du2 * dv1;
    if (std::fabs(det) < 1e-12) throw std::runtime_error("degenerate triangle " + std::to_string(t));
    const double ar = 0.5 * std::fabs(det);
    out.area[t] = (float)ar;
    out.inv[t * 4] = (float)(dv2 / det);
    out.inv[t * 4 + 1] = (float)(-du2 / det);
    out.inv[t * 4 + 2] = (float)(-dv1 / det);
    out.inv[t * 4 + 3] = (float)(du1 / det);
    const double tm = density * ar / 3;
    for (uint32_t v : {i0, i1, i2}) out.mass[v] = (float)((double)out.mass[v] + tm);
  }
  // Edges in first-seen order; an interior edge (two triangles) is a hinge.
  struct Use { int tri, a, b, opp; };
  std::unordered_map<uint64_t, int> slot;
  std::vector<std::pair<Use, Use>> edges;
  std::vector<int> count;
  slot.reserve((size_t)m * 2);
  for (int t = 0; t < m; t++) {
    const int id3[3] = {(int)idx[t * 3], (int)idx[t * 3 + 1], (int)idx[t * 3 + 2]};
    for (int e = 0; e < 3; e++) {
      const int a = id3[e], b = id3[(e + 1) % 3], o = id3[(e + 2) % 3];
      const uint64_t key = ((uint64_t)(uint32_t)std::min(a, b) << 32) | (uint32_t)std::max(a, b);
      auto it = slot.find(key);
      if (it == slot.end()) {
        slot.emplace(key, (int)edges.size());
        edges.push_back({{t, a, b, o}, {}});
        count.push_back(1);
      } else {
        const int s = it->second;
        if (count[s] == 1) edges[s].second = {t, a, b, o};
        count[s]++;
      }
    }
  }
  out.hinge.clear();
  out.hmeta.clear();
  for (size_t s = 0; s < edges.size(); s++) {
    if (count[s] != 2) continue;
    const Use& e0 = edges[s].first;
    const Use& e1 = edges[s].second;
    out.hinge.insert(out.hinge.end(), {e0.a, e0.b, e0.opp, e1.opp});
    const double rest = dihedral_f(pos.data(), e0.a, e0.b, e0.opp, e1.opp);
    const double len = hypot3_js((double)pos[e0.a * 3] - pos[e0.b * 3], (double)pos[e0.a * 3 + 1] - pos[e0.b * 3 + 1],
                                 (double)pos[e0.a * 3 + 2] - pos[e0.b * 3 + 2]);
    out.hmeta.insert(out.hmeta.end(), {rest, len, (double)out.area[e0.tri] + (double)out.area[e1.tri]});
  }
  out.hg = (int)out.hinge.size() / 4;
}

// Element-ordered CSR: records appended in ascending element order, so a
// per-vertex gather sums exactly as the reference's element-order scatter.
static void csr(int n, const std::vector<std::array<uint32_t, 2>>& recs, std::vector<uint32_t>& off,
                std::vector<uint32_t>& out) {
  off.assign(n + 1, 0);
  for (auto& r : recs) off[r[0] + 1]++;
  for (int v = 0; v < n; v++) off[v + 1] += off[v];
  out.assign(recs.size(), 0);
  std::vector<uint32_t> cur(off.begin(), off.end() - 1);
  for (auto& r : recs) out[cur[r[0]]++] = r[1];
}

void build_topology(HostMesh& me) {
  std::vector<std::array<uint32_t, 2>> recs;
  recs.reserve((size_t)me.m * 3);
  for (int t = 0; t < me.m; t++)
    for (uint32_t c = 0; c < 3; c++) recs.push_back({me.idx[t * 3 + c], ((uint32_t)t << 2) | c});
  csr(me.n, recs, me.memOff, me.memRec);
  recs.clear();
  for (int h = 0; h < me.hg; h++)
    for (uint32_t c = 0; c < 4; c++) {
      bool dup = false;
      for (uint32_t q = 0; q < c; q++) dup |= me.hinge[h * 4 + q] == me.hinge[h * 4 + c];
      if (!dup) recs.push_back({(uint32_t)me.hinge[h * 4 + c], ((uint32_t)h << 2) | c});
    }
  csr(me.n, recs, me.hinOff, me.hinRec);
  recs.clear();
  for (int t = 0; t < me.m; t++)
    for (uint32_t c = 0; c < 3; c++) recs.push_back({me.idx[t * 3 + c], (uint32_t)t});
  csr(me.n, recs, me.v2tOff, me.v2t);
}

// src/solver/schwarz.ts:44-140: Morton-ordered seeds over the rest shape, BFS
// growth to `target` vertices along mesh edges (ascending neighbours), merge of
// sub-minimum domains into the smallest adjacent one, members sorted.
void build_schwarz(HostMesh& me, int target, int minSize) {
  const int n = me.n;
  std::vector<std::vector<int>> adj(n);
  {
    std::vector<std::set<int>> s(n);
    for (int t = 0; t < me.m; t++) {
      const int a = me.idx[t * 3], b = me.idx[t * 3 + 1], c = me.idx[t * 3 + 2];
      s[a].insert(b); s[a].insert(c); s[b].insert(a); s[b].insert(c); s[c].insert(a); s[c].insert(b);
    }
    for (int v = 0; v < n; v++) adj[v].assign(s[v].begin(), s[v].end());
  }
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int v = 0; v < n; v++)
    for (int k = 0; k < 3; k++) {
      lo[k] = jmin(lo[k], me.rest[v * 3 + k]);
      hi[k] = jmax(hi[k], me.rest[v * 3 + k]);
    }
  double span[3];
  for (int k = 0; k < 3; k++) span[k] = jmax(hi[k] - lo[k], 1e-12);
  std::vector<uint32_t> code(n);
  for (int v = 0; v < n; v++) {
    int q[3];
    for (int k = 0; k < 3; k++) {
      const double f = std::floor((((double)me.rest[v * 3 + k] - lo[k]) / span[k]) * 1024);
      q[k] = (int)jmax(0, jmin(1023, f));
    }
    uint32_t c = 0;
    for (int b = 9; b >= 0; b--)
      c = (c << 3) | (((q[0] >> b) & 1) << 2) | (((q[1] >> b) & 1) << 1) | ((q[2] >> b) & 1);
    code[v] = c;
  }
  std::vector<int> order(n);
  for (int v = 0; v < n; v++) order[v] = v;
  std::sort(order.begin(), order.end(), [&](int a, int b) { return code[a] != code[b] ? code[a] < code[b] : a < b; });
  std::vector<int> dom(n, -1);
  std::vector<std::vector<int>> mem;
  for (int seed : order) {
    if (dom[seed] >= 0) continue;
    const int id = (int)mem.size();
    mem.push_back({seed});
    dom[seed] = id;
    std::deque<int> qu{seed};
    while ((int)mem[id].size() < target && !qu.empty()) {
      const int cur = qu.front();
      qu.pop_front();
      for (int w : adj[cur]) {
        if ((int)mem[id].size() >= target) break;
        if (dom[w] >= 0) continue;
        dom[w] = id;
        mem[id].push_back(w);
        qu.push_back(w);
      }
    }
  }
  for (;;) {
    int small = -1;
    for (int d = 0; d < (int)mem.size(); d++) {
      const int len = (int)mem[d].size();
      if (len > 0 && len < minSize && n >= minSize && (small < 0 || len < (int)mem[small].size())) small = d;
    }
    if (small < 0) break;
    std::set<int> nb;
    for (int t = 0; t < me.m; t++) {
      const int ds[3] = {dom[me.idx[t * 3]], dom[me.idx[t * 3 + 1]], dom[me.idx[t * 3 + 2]]};
      if (ds[0] != small && ds[1] != small && ds[2] != small) continue;
      for (int x : ds) if (x != small) nb.insert(x);
    }
    int best = -1;
    for (int c : nb)
      if (!mem[c].empty() && (best < 0 || mem[c].size() < mem[best].size())) best = c;
    if (best < 0) break;
    for (int v : mem[small]) { dom[v] = best; mem[best].push_back(v); }
    mem[small].clear();
  }
  me.domStart.assign(1, 0);
  me.domVerts.clear();
  for (auto& m : mem) {
    if (m.empty()) continue;
    std::vector<int> s = m;
    std::sort(s.begin(), s.end());
    me.domVerts.insert(me.domVerts.end(), s.begin(), s.end());
    me.domStart.push_back((int)me.domVerts.size());
  }
  me.D = (int)me.domStart.size() - 1;
  me.maxDomain = 0;
  for (int d = 0; d < me.D; d++) me.maxDomain = std::max(me.maxDomain, me.domStart[d + 1] - me.domStart[d]);
}

}  // namespace cs
