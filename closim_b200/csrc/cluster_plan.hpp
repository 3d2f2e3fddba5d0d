// Per-CTA element lists of the one-cluster PCG's resident phase A.
//
// CTA r of the cluster owns the vertices [vb[r], vb[r+1]). Its lists hold
// every triangle and hinge incident to an owned vertex (boundary elements
// appear in two CTAs' lists) and its halo: the owned vertices plus every
// vertex of those elements, sorted. Element vertex ids are halo-local
// (16 bit), so once p is staged on the halo in shared memory an element's
// HVP reads nothing from global memory. Per owned vertex, `inc` lists its
// triangle incidences (local slot << 2 | corner, in the membrane CSR's order)
// and then its hinge incidences (in the hinge CSR's order).
//
// Phase B (one warp per Schwarz domain, lane = local dof) is resident too:
// domain dom = w + u * nwarps belongs to warp w of CTA w / warpsPerCta, in
// that CTA's domain slot u * warpsPerCta + (w % warpsPerCta). The slot holds
// the domain's packed symmetric FP32 inverse (300 floats) and its 24 dof
// records (Ap, p, x, r). vDst[v] = CTA << 24 | (slot * 24 + member * 3) tells
// vertex v's owner where to push Ap and p over distributed shared memory.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#ifdef __CUDACC__
#define CL_HD __host__ __device__
#else
#define CL_HD
#endif

namespace cs {

struct HostMesh;

// Byte offsets of one CTA's shared-memory regions (16-byte aligned).
struct ClSmem {
  int pH, triD, triO, hinG, hinL, hinS, inc, incOff, incHin, ownH, ownMP, cOff, ownDst, bufB, Lp, halo, cShare, cRec,
      cCap, total;
};

// Bytes of shared memory per on-chip contact record (id + 3 FP32 shares).
constexpr int kClRecBytes = 16;
// Dynamic shared memory a CTA of the one-cluster PCG may take: the 227 KB
// opt-in limit less the kernel's static shared memory (about 2.2 KB) and a margin.
constexpr int kClMaxDynSmem = 227 * 1024 - 4096;

CL_HD inline int cl_up16(int b) { return (b + 15) & ~15; }

// cap: contact records kept on chip (the rest of the CTA's records use global
// scratch); sized on the host to fill the launch's shared memory.
CL_HD inline ClSmem cl_smem_layout(int nHalo, int nTri, int nHin, int nInc, int nOwned, int nSlots, bool hinges,
                                   int cap = 0) {
  ClSmem s;
  int o = 0;
  // first: peers write into it through distributed shared memory at the same
  // offset in every CTA
  s.bufB = o; o += cl_up16(nSlots * 24 * 16);  // per domain dof: Ap, p, x, r
  s.pH = o;   o += cl_up16(nHalo * 16);        // p on the halo, float4
  s.triD = o; o += cl_up16(nTri * 64);         // triangle record: 14 floats + packed local ids
  s.triO = o; o += cl_up16(nTri * 36);         // triangle output: the three corner shares
  const int nh = hinges ? nHin : 0;
  s.hinG = o; o += cl_up16(nh * 48);           // Gauss-Newton factor g (12 floats)
  s.hinL = o; o += cl_up16(nh * 8);            // 4 local ids
  s.hinS = o; o += cl_up16(nh * 4);            // g . p
  s.inc = o;  o += cl_up16(nInc * 4);
  s.incOff = o; o += cl_up16((nOwned + 1) * 4);
  s.incHin = o; o += cl_up16(nOwned * 4);
  s.ownH = o; o += cl_up16(nOwned * 4);
  s.ownMP = o; o += cl_up16(nOwned * 8);       // mass, pinned flag of the owned vertices
  s.cOff = o; o += cl_up16((nOwned + 1) * 4);  // contact-record CSR offsets of the owned vertices
  s.ownDst = o; o += cl_up16(nOwned * 4);      // vDst of the owned vertices
  s.Lp = o;   o += cl_up16(nSlots * 300 * 4);  // packed lower triangle of each domain's inverse
  s.halo = o; o += cl_up16(nHalo * 4);         // global vertex ids of the halo
  s.cCap = cap;
  s.cShare = o; o += cl_up16(cap * 12);        // contact shares (FP32) of the on-chip records
  s.cRec = o; o += cl_up16(cap * 4);           // their record ids
  s.total = o;
  return s;
}

struct ClusterPlanHost {
  int nrank = 0;
  bool ok = false;  // every halo fits 16-bit local ids
  std::vector<int> vb, haloOff, halo, triOff, triId, hinOff, hinId, incOff, incHin, ownHalo, vDst;
  int warpsPerCta = 0, nwarps = 0;
  std::vector<int> nSlots;  // domain slots of each CTA
  std::vector<uint16_t> triLoc, hinLoc;  // 4 per slot (triangles: x, y, z, 0)
  std::vector<uint32_t> inc;
  size_t smemNoHinge = 0, smemHinge = 0;  // largest CTA's dynamic shared memory
};

// ok stays false when a halo needs more than 16-bit ids, when the domains do
// not partition the vertices, or when some warp would own more than 3 domains.
void build_cluster_plan(const HostMesh& me, int nrank, int warpsPerCta, ClusterPlanHost& p);

}  // namespace cs
