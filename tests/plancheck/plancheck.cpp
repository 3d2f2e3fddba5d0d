// Test helper: host build of the one-cluster PCG's per-CTA list builder
// (closim_b200/csrc/cluster_plan.cpp) with a checker of its invariants, for
// CPU tests. Returns 0 when every invariant holds, else a code naming the
// first one broken.
#include <cstdint>
#include <vector>

#include "../../closim_b200/csrc/cluster_plan.hpp"
#include "../../closim_b200/csrc/setup.hpp"

extern "C" int pc_check(int n, int m, int hg, const uint32_t* idx, const int* hinge, const float* rest, int nrank,
                        int64_t* info) {
  // info: smem without / with hinges, ok, halo, triangle and hinge list sizes, domains
  cs::HostMesh me;
  me.n = n; me.m = m; me.hg = hg;
  me.idx.assign(idx, idx + 3 * (size_t)m);
  me.hinge.assign(hinge, hinge + 4 * (size_t)hg);
  cs::build_topology(me);
  me.rest.assign(rest, rest + 3 * (size_t)n);
  cs::build_schwarz(me, 8, 1);
  cs::ClusterPlanHost p;
  cs::build_cluster_plan(me, nrank, 16, p);
  info[0] = (int64_t)p.smemNoHinge;
  info[1] = (int64_t)p.smemHinge;
  info[2] = p.ok ? 1 : 0;
  info[3] = (int64_t)p.halo.size();
  info[4] = (int64_t)p.triId.size();
  info[5] = (int64_t)p.hinId.size();
  if (!p.ok) return 1;
  if ((int)p.vb.size() != nrank + 1 || p.vb[0] != 0 || p.vb[nrank] != n) return 2;
  for (int r = 0; r < nrank; r++) {
    if (p.vb[r] > p.vb[r + 1]) return 3;
    const int h0 = p.haloOff[r], nh = p.haloOff[r + 1] - h0;
    const int t0 = p.triOff[r], nt = p.triOff[r + 1] - t0;
    const int g0 = p.hinOff[r], ng = p.hinOff[r + 1] - g0;
    for (int i = 1; i < nh; i++)
      if (p.halo[h0 + i] <= p.halo[h0 + i - 1]) return 4;  // sorted, unique
    for (int s = 0; s < nt; s++) {
      const int t = p.triId[t0 + s];
      for (int c = 0; c < 3; c++) {
        const int l = p.triLoc[4 * (size_t)(t0 + s) + c];
        if (l >= nh || p.halo[h0 + l] != (int)me.idx[3 * (size_t)t + c]) return 5;
      }
    }
    for (int s = 0; s < ng; s++) {
      const int h = p.hinId[g0 + s];
      for (int c = 0; c < 4; c++) {
        const int l = p.hinLoc[4 * (size_t)(g0 + s) + c];
        if (l >= nh || p.halo[h0 + l] != me.hinge[4 * (size_t)h + c]) return 6;
      }
    }
    for (int v = p.vb[r]; v < p.vb[r + 1]; v++) {
      if (p.ownHalo[v] >= nh || p.halo[h0 + p.ownHalo[v]] != v) return 7;
      // triangle incidences: the CSR's records, in its order, by local slot
      int j = p.incOff[v];
      for (uint32_t q = me.memOff[v]; q < me.memOff[v + 1]; q++, j++) {
        if (j >= p.incHin[v]) return 8;
        const uint32_t rec = p.inc[j], slot = rec >> 2, c = rec & 3;
        if ((int)slot >= nt || p.triId[t0 + slot] != (int)(me.memRec[q] >> 2) || c != (me.memRec[q] & 3)) return 9;
        if (p.triLoc[4 * (size_t)(t0 + slot) + c] != p.ownHalo[v]) return 10;
      }
      if (j != p.incHin[v]) return 11;
      for (uint32_t q = me.hinOff[v]; q < me.hinOff[v + 1]; q++, j++) {
        if (j >= p.incOff[v + 1]) return 12;
        const uint32_t rec = p.inc[j], slot = rec >> 2, c = rec & 3;
        if ((int)slot >= ng || p.hinId[g0 + slot] != (int)(me.hinRec[q] >> 2) || c != (me.hinRec[q] & 3)) return 13;
        if (p.hinLoc[4 * (size_t)(g0 + slot) + c] != p.ownHalo[v]) return 14;
      }
      if (j != p.incOff[v + 1]) return 15;
    }
    // every listed element touches an owned vertex
    for (int s = 0; s < nt; s++) {
      const int t = p.triId[t0 + s];
      bool own = false;
      for (int c = 0; c < 3; c++) own |= (int)me.idx[3 * (size_t)t + c] >= p.vb[r] && (int)me.idx[3 * (size_t)t + c] < p.vb[r + 1];
      if (!own) return 16;
    }
    const int nInc = p.incOff[p.vb[r + 1]] - p.incOff[p.vb[r]], nOwn = p.vb[r + 1] - p.vb[r];
    const cs::ClSmem L = cs::cl_smem_layout(nh, nt, ng, nInc, nOwn, p.nSlots[r], true);
    if ((size_t)L.total > p.smemHinge) return 17;
    if (L.bufB != 0) return 21;  // written by peers: the same offset in every CTA
    for (int off : {L.pH, L.triD, L.triO, L.hinG, L.hinL, L.hinS, L.inc, L.incOff, L.incHin, L.ownH, L.ownMP, L.cOff,
                    L.ownDst, L.bufB, L.Lp, L.halo})
      if (off % 16) return 18;
  }
  // phase B: each vertex's dofs sit in the slot of the warp that owns its domain
  for (int dom = 0; dom < me.D; dom++) {
    const int gw = dom % p.nwarps, u = dom / p.nwarps;
    const int r = gw / 16, slot = u * 16 + gw % 16;
    if (u > 2 || slot >= p.nSlots[r]) return 19;
    for (int l = 0; l < me.domStart[dom + 1] - me.domStart[dom]; l++) {
      const int v = me.domVerts[me.domStart[dom] + l];
      if (p.vDst[v] != ((r << 24) | (slot * 24 + l * 3))) return 20;
    }
  }
  info[6] = me.D;
  return 0;
}
