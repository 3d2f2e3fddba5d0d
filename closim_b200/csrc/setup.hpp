// Host-side mesh set-up for the CUDA cloth solver.
#pragma once
#include <array>
#include <cstdint>
#include <vector>

namespace cs {

// ClothMeshData (reference src/mesh/mesh.ts:3-14) plus the derived topology.
struct HostMesh {
  int n = 0, m = 0, hg = 0;
  std::vector<uint32_t> idx;
  std::vector<float> rest, inv, area, mass;
  std::vector<int> hinge;       // 4 per hinge
  std::vector<double> hmeta;    // restAngle, edgeLen, areaSum per hinge
  std::vector<uint32_t> memOff, memRec, hinOff, hinRec, v2tOff, v2t;
  std::vector<int> domStart, domVerts;
  int D = 0, maxDomain = 0;
};

double hypot3_js(double a, double b, double c);
void grid_mesh(int nx, int ny, double w, double h, std::vector<float>& pos, std::vector<float>& uv,
               std::vector<uint32_t>& idx);
void preprocess_mesh(const std::vector<float>& pos, const std::vector<float>& uv,
                     const std::vector<uint32_t>& idx, double density, HostMesh& out);
void build_topology(HostMesh& me);
void build_schwarz(HostMesh& me, int target, int minSize);

}  // namespace cs
