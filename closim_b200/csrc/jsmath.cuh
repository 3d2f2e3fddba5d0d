// Math.acos, Math.log and Math.cbrt as V8 evaluates them (host + device).
//
// V8 implements these in src/base/ieee754.cc as ports of the published
// fdlibm / FreeBSD msun routines (e_acos.c, e_log.c, s_cbrt.c). The FP64 path
// calls these instead of the CUDA library functions so that every hinge angle,
// barrier log term and CCD cubic root rounds exactly as the reference's
// JavaScript does; the CPU oracle carries its own copy of the same algorithms.
// Must be compiled without FMA contraction (-fmad=false / -ffp-contract=off).
#pragma once
#include <stdint.h>
#include <string.h>

namespace cs {

#define JSHD __host__ __device__ __forceinline__

JSHD int32_t js_hi(double x) {
#ifdef __CUDA_ARCH__
  return __double2hiint(x);
#else
  uint64_t u; memcpy(&u, &x, 8); return (int32_t)(u >> 32);
#endif
}
JSHD uint32_t js_lo(double x) {
#ifdef __CUDA_ARCH__
  return (uint32_t)__double2loint(x);
#else
  uint64_t u; memcpy(&u, &x, 8); return (uint32_t)u;
#endif
}
JSHD double js_make(int32_t hi, uint32_t lo) {
#ifdef __CUDA_ARCH__
  return __hiloint2double(hi, (int)lo);
#else
  const uint64_t u = ((uint64_t)(uint32_t)hi << 32) | lo;
  double x; memcpy(&x, &u, 8); return x;
#endif
}

// fdlibm e_acos.c (Sun Microsystems, 1993).
JSHD double js_acos(double x) {
  const double one = 1.0, pi = 3.14159265358979311600e+00, pio2_hi = 1.57079632679489655800e+00,
               pio2_lo = 6.12323399573676603587e-17, pS0 = 1.66666666666666657415e-01,
               pS1 = -3.25565818622400915405e-01, pS2 = 2.01212532134862925881e-01,
               pS3 = -4.00555345006794114027e-02, pS4 = 7.91534994289814532176e-04,
               pS5 = 3.47933107596021167570e-05, qS1 = -2.40339491173441421878e+00,
               qS2 = 2.02094576023350569471e+00, qS3 = -6.88283971605453293030e-01,
               qS4 = 7.70381505559019352791e-02;
  const int32_t hx = js_hi(x);
  const int32_t ix = hx & 0x7fffffff;
  if (ix >= 0x3ff00000) {
    if (((ix - 0x3ff00000) | (int32_t)js_lo(x)) == 0) {
      if (hx > 0) return 0.0;
      return pi + 2.0 * pio2_lo;
    }
    return (x - x) / (x - x);
  }
  if (ix < 0x3fe00000) {
    if (ix <= 0x3c600000) return pio2_hi + pio2_lo;
    const double z = x * x;
    const double p = z * (pS0 + z * (pS1 + z * (pS2 + z * (pS3 + z * (pS4 + z * pS5)))));
    const double q = one + z * (qS1 + z * (qS2 + z * (qS3 + z * qS4)));
    const double r = p / q;
    return pio2_hi - (x - (pio2_lo - x * r));
  } else if (hx < 0) {
    const double z = (one + x) * 0.5;
    const double p = z * (pS0 + z * (pS1 + z * (pS2 + z * (pS3 + z * (pS4 + z * pS5)))));
    const double q = one + z * (qS1 + z * (qS2 + z * (qS3 + z * qS4)));
    const double s = sqrt(z);
    const double r = p / q;
    const double w = r * s - pio2_lo;
    return pi - 2.0 * (s + w);
  } else {
    const double z = (one - x) * 0.5;
    const double s = sqrt(z);
    const double df = js_make(js_hi(s), 0);
    const double c = (z - df * df) / (s + df);
    const double p = z * (pS0 + z * (pS1 + z * (pS2 + z * (pS3 + z * (pS4 + z * pS5)))));
    const double q = one + z * (qS1 + z * (qS2 + z * (qS3 + z * qS4)));
    const double r = p / q;
    const double w = r * s + c;
    return 2.0 * (df + w);
  }
}

// fdlibm e_log.c.
JSHD double js_log(double x) {
  const double ln2_hi = 6.93147180369123816490e-01, ln2_lo = 1.90821492927058770002e-10,
               two54 = 1.80143985094819840000e+16, Lg1 = 6.666666666666735130e-01,
               Lg2 = 3.999999999940941908e-01, Lg3 = 2.857142874366239149e-01,
               Lg4 = 2.222219843214978396e-01, Lg5 = 1.818357216161805012e-01,
               Lg6 = 1.531383769920937332e-01, Lg7 = 1.479819860511658591e-01, zero = 0.0;
  int32_t hx = js_hi(x);
  const uint32_t lx = js_lo(x);
  int32_t k = 0;
  if (hx < 0x00100000) {
    if (((hx & 0x7fffffff) | (int32_t)lx) == 0) return -two54 / (x - x);  // -inf
    if (hx < 0) return (x - x) / (x - x);  // NaN
    k -= 54;
    x *= two54;
    hx = js_hi(x);
  }
  if (hx >= 0x7ff00000) return x + x;
  k += (hx >> 20) - 1023;
  hx &= 0x000fffff;
  int32_t i = (hx + 0x95f64) & 0x100000;
  x = js_make(hx | (i ^ 0x3ff00000), js_lo(x));
  k += (i >> 20);
  const double f = x - 1.0;
  if ((0x000fffff & (2 + hx)) < 3) {
    if (f == zero) {
      if (k == 0) return zero;
      const double dk = (double)k;
      return dk * ln2_hi + dk * ln2_lo;
    }
    const double R = f * f * (0.5 - 0.33333333333333333 * f);
    if (k == 0) return f - R;
    const double dk = (double)k;
    return dk * ln2_hi - ((R - dk * ln2_lo) - f);
  }
  const double s = f / (2.0 + f);
  const double dk = (double)k;
  const double z = s * s;
  i = hx - 0x6147a;
  const double w = z * z;
  const int32_t j = 0x6b851 - hx;
  const double t1 = w * (Lg2 + w * (Lg4 + w * Lg6));
  const double t2 = z * (Lg1 + w * (Lg3 + w * (Lg5 + w * Lg7)));
  i |= j;
  const double R = t2 + t1;
  if (i > 0) {
    const double hfsq = 0.5 * f * f;
    if (k == 0) return f - (hfsq - s * (hfsq + R));
    return dk * ln2_hi - ((hfsq - (s * (hfsq + R) + dk * ln2_lo)) - f);
  }
  if (k == 0) return f - s * (f - R);
  return dk * ln2_hi - ((s * (f - R) - dk * ln2_lo) - f);
}

// FreeBSD msun s_cbrt.c (Bruce D. Evans' revision, as ported by V8).
JSHD double js_cbrt(double x) {
  const uint32_t B1 = 715094163, B2 = 696219795;
  const double P0 = 1.87595182427177009643, P1 = -1.88497979543377169875, P2 = 1.621429720105354466140,
               P3 = -0.758397934778766047437, P4 = 0.145996192886612446982;
  int32_t hx = js_hi(x);
  const uint32_t low = js_lo(x);
  const uint32_t sign = (uint32_t)hx & 0x80000000u;
  hx ^= (int32_t)sign;
  if (hx >= 0x7ff00000) return x + x;
  double t;
  if (hx < 0x00100000) {
    if ((hx | (int32_t)low) == 0) return x;
    t = js_make(0x43500000, 0);
    t *= x;
    const uint32_t high = (uint32_t)js_hi(t);
    t = js_make((int32_t)(sign | ((high & 0x7fffffffu) / 3 + B2)), 0);
  } else {
    t = js_make((int32_t)(sign | ((uint32_t)hx / 3 + B1)), 0);
  }
  double r = (t * t) * (t / x);
  t = t * ((P0 + r * (P1 + r * P2)) + ((r * r) * r) * (P3 + r * P4));
  uint64_t bits = ((uint64_t)(uint32_t)js_hi(t) << 32) | js_lo(t);
  bits = (bits + 0x80000000ull) & 0xffffffffc0000000ull;
  t = js_make((int32_t)(bits >> 32), (uint32_t)bits);
  const double s = t * t;
  r = x / s;
  const double w = t + t;
  r = (r - t) / (w + r);
  t = t + t * r;
  return t;
}

}  // namespace cs
