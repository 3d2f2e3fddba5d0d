// Contact data shared by the FP64 kernels: the frozen active set and the
// per-vertex gather structures of the barrier HVP.
#pragma once
#include "plain.cuh"

namespace cs {

// One frozen contact (contact-assembly.ts:22-30): kind 0 VT, 1 EE, 2 floor.
struct Frozen {
  int kind, p, a, b, c, d;
  double w0, w1, w2, w3, nx, ny, nz;
};

struct Contact {
  double dHat, kappa, dMin, mu, eps, floorY;
  int hasFloor;
  int nActive;           // active records
  Frozen* active;        // cap
  double* dd;            // per-contact HVP coefficient (coeff * J v)
  // vertex -> (contact << 2 | slot) records in contact order
  const uint32_t* cOff;  // n+1
  const uint32_t* cRec;
};

// Per-contact HVP coefficient (contact-assembly.ts:371-387).
__device__ __forceinline__ void contact_hvp_coeffs(const Dev& d, const double* v, int tid, int nth) {
  (void)d; (void)v; (void)tid; (void)nth;
}

// Per-vertex sum of the contact HVP contributions (contact-assembly.ts:388-391).
__device__ __forceinline__ void contact_hvp_gather(const Dev& d, int vtx, double out[3]) {
  (void)d; (void)vtx; out[0] = out[1] = out[2] = 0;
}

}  // namespace cs
