// FP32 membrane HVP of one triangle from its stored state, shared by the
// mixed-precision PCG kernels.
#pragma once
#include <cuda_runtime.h>

namespace cs {

// Corner share of one triangle's membrane HVP (membrane-hvp.ts:18-75):
// dF = Ds(p) Dm^-1, dE, dS, dP = dF S + F dS, force = -area * dP Dm^-T.
__device__ __forceinline__ void tri_hvp_corner(const float* T, const float3 p0, const float3 p1, const float3 p2,
                                               int corner, float C00, float C11, float C01, float G, float o[3]) {
  const float4 t0 = __ldg((const float4*)T), t1 = __ldg((const float4*)(T + 4)), t2 = __ldg((const float4*)(T + 8)),
               t3 = __ldg((const float4*)(T + 12));
  const float F0[3] = {t0.x, t0.y, t0.z}, F1[3] = {t0.w, t1.x, t1.y};
  const float S00 = t1.z, S11 = t1.w, S01 = t2.x;
  const float a = t2.y, b = t2.z, c = t2.w, dd = t3.x, s = t3.y;
  const float w1[3] = {p1.x - p0.x, p1.y - p0.y, p1.z - p0.z};
  const float w2[3] = {p2.x - p0.x, p2.y - p0.y, p2.z - p0.z};
  float dF0[3], dF1[3];
#pragma unroll
  for (int q = 0; q < 3; q++) { dF0[q] = a * w1[q] + c * w2[q]; dF1[q] = b * w1[q] + dd * w2[q]; }
  const float dE00 = F0[0] * dF0[0] + F0[1] * dF0[1] + F0[2] * dF0[2];
  const float dE11 = F1[0] * dF1[0] + F1[1] * dF1[1] + F1[2] * dF1[2];
  const float dE01 = 0.5f * (dF0[0] * F1[0] + F0[0] * dF1[0] + dF0[1] * F1[1] + F0[1] * dF1[1] + dF0[2] * F1[2] +
                             F0[2] * dF1[2]);
  const float dS00 = C00 * dE00 + C01 * dE11;
  const float dS11 = C11 * dE11 + C01 * dE00;
  const float dS01 = 2.f * G * dE01;
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const float P0 = dF0[q] * S00 + F0[q] * dS00 + dF1[q] * S01 + F1[q] * dS01;
    const float P1 = dF0[q] * S01 + F0[q] * dS01 + dF1[q] * S11 + F1[q] * dS11;
    const float g1 = s * (P0 * a + P1 * b);
    const float g2 = s * (P0 * c + P1 * dd);
    o[q] = corner == 0 ? -(g1 + g2) : corner == 1 ? g1 : g2;
  }
}

// tri_hvp_corner's corner shares for the whole triangle from a record held in
// registers: corner 1 gets g1, corner 2 gets g2, corner 0 gets -(g1 + g2).
__device__ __forceinline__ void tri_hvp_g12(const float4 t0, const float4 t1, const float4 t2, const float4 t3,
                                            const float4 p0, const float4 p1, const float4 p2, float C00, float C11,
                                            float C01, float G, float g1o[3], float g2o[3]) {
  const float F0[3] = {t0.x, t0.y, t0.z}, F1[3] = {t0.w, t1.x, t1.y};
  const float S00 = t1.z, S11 = t1.w, S01 = t2.x;
  const float a = t2.y, b = t2.z, c = t2.w, dd = t3.x, s = t3.y;
  const float w1[3] = {p1.x - p0.x, p1.y - p0.y, p1.z - p0.z};
  const float w2[3] = {p2.x - p0.x, p2.y - p0.y, p2.z - p0.z};
  float dF0[3], dF1[3];
#pragma unroll
  for (int q = 0; q < 3; q++) { dF0[q] = a * w1[q] + c * w2[q]; dF1[q] = b * w1[q] + dd * w2[q]; }
  const float dE00 = F0[0] * dF0[0] + F0[1] * dF0[1] + F0[2] * dF0[2];
  const float dE11 = F1[0] * dF1[0] + F1[1] * dF1[1] + F1[2] * dF1[2];
  const float dE01 = 0.5f * (dF0[0] * F1[0] + F0[0] * dF1[0] + dF0[1] * F1[1] + F0[1] * dF1[1] + dF0[2] * F1[2] +
                             F0[2] * dF1[2]);
  const float dS00 = C00 * dE00 + C01 * dE11;
  const float dS11 = C11 * dE11 + C01 * dE00;
  const float dS01 = 2.f * G * dE01;
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const float P0 = dF0[q] * S00 + F0[q] * dS00 + dF1[q] * S01 + F1[q] * dS01;
    const float P1 = dF0[q] * S01 + F0[q] * dS01 + dF1[q] * S11 + F1[q] * dS11;
    g1o[q] = s * (P0 * a + P1 * b);
    g2o[q] = s * (P0 * c + P1 * dd);
  }
}

}  // namespace cs
