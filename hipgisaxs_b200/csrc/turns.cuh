// FP32 phase helpers of the FP32C kernels that keep work off the SFU/conversion (XU) pipe:
// rounding to an integer by adding and subtracting a power-of-two constant (FP64 or FP32 add
// pipe), and sin/cos of pi x by polynomials on the FMA pipe.
#pragma once

#include <cuda_runtime.h>

namespace hgx {

// Round to the nearest integer (ties to even) on the FP64 add pipe, for |x| < 2^51: adding
// 1.5 * 2^52 leaves no fraction bits, subtracting it again returns the rounded value.
constexpr double RND52 = 6755399441055744.0;
__device__ __forceinline__ double round_fp64(double x) { return __dsub_rn(__dadd_rn(x, RND52), RND52); }
// The same in FP32 for |x| < 2^22 (1.5 * 2^23).
__device__ __forceinline__ float round_fp32(float x) { return __fsub_rn(__fadd_rn(x, 12582912.0f), 12582912.0f); }

// sin(pi x) and cos(pi x) for |x| <= 1 in FP32 on the FMA pipe: x = r + k/2 with k = rint(2x)
// (rounded by the 1.5 * 2^23 constant, whose low mantissa bits then hold k mod 4) and
// |r| <= 1/4 exact; Taylor polynomials of sin(pi r)/r (to r^8) and cos(pi r) (to r^10), whose
// truncation is below 2e-9 at |pi r| = pi/4; then the rotation by k quarter turns.  Absolute
// error about one FP32 ulp; sin keeps its relative accuracy near 0.
__device__ __forceinline__ void sincospi_f32(float x, float* s, float* c) {
  const float M = 12582912.0f;
  const float b = __fadd_rn(2.0f * x, M);
  const int q = __float_as_int(b) & 3;
  const float r = x - 0.5f * __fsub_rn(b, M);
  const float r2 = r * r;
  const float ps = fmaf(fmaf(fmaf(fmaf(0.08214588463306427f, r2, -0.5992645025253296f), r2,
                                  2.550163984298706f), r2, -5.167712688446045f), r2,
                        3.1415927410125732f);
  const float pc = fmaf(fmaf(fmaf(fmaf(fmaf(-0.025806890800595284f, r2, 0.23533062636852264f), r2,
                                       -1.3352627754211426f), r2, 4.058712005615234f), r2,
                             -4.934802055358887f), r2, 1.0f);
  const float sv = r * ps;
  float so = (q & 1) ? pc : sv, co = (q & 1) ? -sv : pc;
  if (q & 2) {
    so = -so;
    co = -co;
  }
  *s = so;
  *c = co;
}

}  // namespace hgx
