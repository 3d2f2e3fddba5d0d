// Builds the per-CTA element lists of the one-cluster PCG (cluster_plan.hpp)
// from the membrane and hinge incidence CSRs.
#include "cluster_plan.hpp"

#include <algorithm>

#include "setup.hpp"

namespace cs {

void build_cluster_plan(const HostMesh& me, int nrank, int warpsPerCta, ClusterPlanHost& p) {
  p = ClusterPlanHost{};
  p.nrank = nrank;
  p.warpsPerCta = warpsPerCta;
  p.nwarps = nrank * warpsPerCta;
  p.ok = nrank > 0 && warpsPerCta > 0 && me.D <= 3 * p.nwarps;
  if (!p.ok) return;
  const int n = me.n;
  // phase B: domain slots per CTA and where each vertex's dofs live
  p.vDst.assign(n, -1);
  p.nSlots.assign(nrank, 0);
  for (int dom = 0; dom < me.D; dom++) {
    const int gw = dom % p.nwarps, u = dom / p.nwarps, r = gw / warpsPerCta, slot = u * warpsPerCta + gw % warpsPerCta;
    p.nSlots[r] = std::max(p.nSlots[r], slot + 1);
    for (int l = 0; l < me.domStart[dom + 1] - me.domStart[dom]; l++) {
      const int v = me.domVerts[me.domStart[dom] + l];
      if (l >= 8 || v < 0 || v >= n || p.vDst[v] != -1) { p.ok = false; return; }
      p.vDst[v] = (r << 24) | (slot * 24 + l * 3);
    }
  }
  for (int v = 0; v < n; v++)
    if (p.vDst[v] < 0) { p.ok = false; return; }
  p.vb.resize(nrank + 1);
  for (int r = 0; r <= nrank; r++) p.vb[r] = (int)((int64_t)r * n / nrank);
  p.haloOff.assign(1, 0);
  p.triOff.assign(1, 0);
  p.hinOff.assign(1, 0);
  p.incOff.assign(n + 1, 0);
  p.incHin.assign(n, 0);
  p.ownHalo.assign(n, 0);
  std::vector<int> loc(n, -1), tslot(me.m, -1), hslot(me.hg, -1);
  std::vector<int> tris, hins, halo;
  for (int r = 0; r < nrank; r++) {
    const int v0 = p.vb[r], v1 = p.vb[r + 1];
    tris.clear();
    hins.clear();
    halo.clear();
    for (int v = v0; v < v1; v++) {
      halo.push_back(v);
      for (uint32_t q = me.memOff[v]; q < me.memOff[v + 1]; q++) tris.push_back((int)(me.memRec[q] >> 2));
      for (uint32_t q = me.hinOff[v]; q < me.hinOff[v + 1]; q++) hins.push_back((int)(me.hinRec[q] >> 2));
    }
    std::sort(tris.begin(), tris.end());
    tris.erase(std::unique(tris.begin(), tris.end()), tris.end());
    std::sort(hins.begin(), hins.end());
    hins.erase(std::unique(hins.begin(), hins.end()), hins.end());
    for (int t : tris)
      for (int c = 0; c < 3; c++) halo.push_back((int)me.idx[3 * (size_t)t + c]);
    for (int h : hins)
      for (int c = 0; c < 4; c++) halo.push_back(me.hinge[4 * (size_t)h + c]);
    std::sort(halo.begin(), halo.end());
    halo.erase(std::unique(halo.begin(), halo.end()), halo.end());
    if (halo.size() > 65535) p.ok = false;
    for (size_t i = 0; i < halo.size(); i++) loc[halo[i]] = (int)i;
    for (size_t s = 0; s < tris.size(); s++) {
      const int t = tris[s];
      tslot[t] = (int)s;
      for (int c = 0; c < 3; c++) p.triLoc.push_back((uint16_t)loc[me.idx[3 * (size_t)t + c]]);
      p.triLoc.push_back(0);
    }
    for (size_t s = 0; s < hins.size(); s++) {
      const int h = hins[s];
      hslot[h] = (int)s;
      for (int c = 0; c < 4; c++) p.hinLoc.push_back((uint16_t)loc[me.hinge[4 * (size_t)h + c]]);
    }
    const size_t inc0 = p.inc.size();
    for (int v = v0; v < v1; v++) {
      p.incOff[v] = (int)p.inc.size();
      for (uint32_t q = me.memOff[v]; q < me.memOff[v + 1]; q++) {
        const uint32_t rec = me.memRec[q];
        p.inc.push_back(((uint32_t)tslot[rec >> 2] << 2) | (rec & 3));
      }
      p.incHin[v] = (int)p.inc.size();
      for (uint32_t q = me.hinOff[v]; q < me.hinOff[v + 1]; q++) {
        const uint32_t rec = me.hinRec[q];
        p.inc.push_back(((uint32_t)hslot[rec >> 2] << 2) | (rec & 3));
      }
      p.ownHalo[v] = loc[v];
    }
    const int nInc = (int)(p.inc.size() - inc0), nOwn = v1 - v0;
    p.triId.insert(p.triId.end(), tris.begin(), tris.end());
    p.hinId.insert(p.hinId.end(), hins.begin(), hins.end());
    p.halo.insert(p.halo.end(), halo.begin(), halo.end());
    p.triOff.push_back((int)p.triId.size());
    p.hinOff.push_back((int)p.hinId.size());
    p.haloOff.push_back((int)p.halo.size());
    const int nh = (int)halo.size(), nt = (int)tris.size(), ng = (int)hins.size();
    const int ns = p.nSlots[r];
    p.smemNoHinge = std::max(p.smemNoHinge, (size_t)cl_smem_layout(nh, nt, ng, nInc, nOwn, ns, false).total);
    p.smemHinge = std::max(p.smemHinge, (size_t)cl_smem_layout(nh, nt, ng, nInc, nOwn, ns, true).total);
  }
  p.incOff[n] = (int)p.inc.size();
}

}  // namespace cs
