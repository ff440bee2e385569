// device_sincos.cuh -- FP64 sine and cosine for the pair kernels, table-driven.
//
// The pair kernels need sin and cos of the phase k R once per pair.  This is
// the classical table-driven method (P. T. P. Tang, "Table-driven
// implementation of the exponential function in IEEE floating-point
// arithmetic", ACM TOMS 15, 1989, applied to sin / cos): reduce x to the
// nearest multiple q pi/32 with a two-part pi/32 (the products q * part are
// exact inside the FMAs), so |r| <= pi/64 + tiny, then
//   sin x = S_m cos r + C_m sin r,   cos x = C_m cos r - S_m sin r,
// with (S_m, C_m) = (sin, cos)(m pi/32), m = q mod 64, from a 64-entry table,
// and sin r, cos r from their Taylor series through r^9 and r^8 (the first
// terms left out are below 1e-21 on |r| <= 0.0491).
// pi/32 = kScStepHi + kScStepLo: kScStepHi is the double nearest pi scaled by
// 2^-5 (exact), kScStepLo the scaled difference pi - fl(pi).  The table is
// built on the host in long double and copied to constant memory once per
// device; a kernel stages it in shared memory, since its lanes index it
// independently.  Error against long double sinl / cosl: below 1.6e-16
// absolute for |x| up to 1e5.
#pragma once

#include <cmath>
#include <mutex>

namespace lum {

constexpr int kScTab = 64;
constexpr double kScInvStep = 32.0 / 3.14159265358979323846;
constexpr double kScStepHi = 3.141592653589793 / 32.0;
constexpr double kScStepLo = 1.2246467991473532e-16 / 32.0;

// Each translation unit that includes this header has its own copy.
static __constant__ double2 c_sincos_tab[kScTab];

// Copies the table to this translation unit's constant memory on the
// current device, once per device.  Call it before launching (not while a
// stream is being captured).
static lum_status sincos_table_ready() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  LUM_TRY_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (dev >= 0 && dev < 64 && done[dev]) return LUM_OK;
  const long double pi = 3.14159265358979323846264338327950288L;
  double2 h[kScTab];
  for (int m = 0; m < kScTab; ++m) {
    h[m].x = (double)sinl(m * pi / 32);
    h[m].y = (double)cosl(m * pi / 32);
  }
  LUM_TRY_CUDA(cudaMemcpyToSymbol(c_sincos_tab, h, sizeof h));
  if (dev >= 0 && dev < 64) done[dev] = true;
  return LUM_OK;
}

// The first kScTab threads of a CTA copy the table into shared memory; the
// caller synchronises before the first use.
__device__ __forceinline__ void sincos_table_stage(double2* s_tab) {
  if (threadIdx.x < kScTab) s_tab[threadIdx.x] = c_sincos_tab[threadIdx.x];
}

__device__ __forceinline__ void sincos_tab(double x, const double2* __restrict__ s_tab,
                                           double* s, double* c) {
  const double q = rint(x * kScInvStep);
  double r = fma(-q, kScStepHi, x);
  r = fma(-q, kScStepLo, r);
  const int m = (int)((long long)q & (kScTab - 1));
  const double r2 = r * r;
  const double ps = fma(fma(fma(fma(r2, 1.0 / 362880.0, -1.0 / 5040.0), r2, 1.0 / 120.0), r2,
                            -1.0 / 6.0),
                        r2 * r, r);
  const double pc =
      fma(fma(fma(fma(r2, 1.0 / 40320.0, -1.0 / 720.0), r2, 1.0 / 24.0), r2, -0.5), r2, 1.0);
  const double2 t = s_tab[m];
  *s = fma(t.x, pc, t.y * ps);
  *c = fma(t.y, pc, -(t.x * ps));
}

}  // namespace lum
