// sommerfeld.cuh -- device functions of the Sommerfeld reflected Green's
// tensor (crates/lumina-core/src/solver/sommerfeld.rs): the module's Bessel
// functions, the principal complex root, the five k_par integrands and their
// Kronrod quadrature on the reference's segments.  Shared by the pair tables
// (sommerfeld.cu) and the FFT operator's reflected spectra (fft.cu).
#pragma once
#include "lumina_internal.cuh"
#include "device_physics.cuh"

namespace lum {

// Kronrod 15-point rule on [-1, 1] (sommerfeld.rs:43-76).
static __constant__ double c_somm_x[15] = {
    -0.991455371120813, -0.949107912342758, -0.864864423359769, -0.741531185599394,
    -0.586087235467691, -0.405845151377397, -0.207784955007898, 0.0,
    0.207784955007898,  0.405845151377397,  0.586087235467691,  0.741531185599394,
    0.864864423359769,  0.949107912342758,  0.991455371120813};
static __constant__ double c_somm_w[15] = {
    0.022935322010529, 0.063092092629979, 0.104790010322250, 0.140653259715525,
    0.169004726639267, 0.190350578064785, 0.204432940075298, 0.209482141084728,
    0.204432940075298, 0.190350578064785, 0.169004726639267, 0.140653259715525,
    0.104790010322250, 0.063092092629979, 0.022935322010529};


// J0 and J1 with the coefficients of sommerfeld.rs:103-146.  Their x >= 8
// branches (and four small-x J1 coefficients) are that module's own, not the
// Numerical Recipes values used for the lattice sums; the reflected tensor is
// defined by them, so they are kept as written.
__device__ __forceinline__ double somm_j0(double x) {
  const double ax = fabs(x);
  if (ax < 8.0) {
    const double y = x * x;
    const double p1 = 57568490574.0 + y * (-13362590354.0 + y * (651619640.7 +
                      y * (-11214424.18 + y * (77392.33017 + y * (-184.9052456)))));
    const double q1 = 57568490411.0 + y * (1029532985.0 + y * (9494680.718 +
                      y * (59272.64853 + y * (267.8532712 + y))));
    return p1 / q1;
  }
  const double z = 8.0 / ax, y = z * z, xx = ax - 0.7853981634;
  const double p1 = 1.0 + y * (-0.001098628627 + y * (0.000002734511 +
                    y * (-0.00000002073 + y * (-0.0000000002073))));
  const double q1 = -0.001562499995 + y * (0.000001430488 + y * (-0.000000006905 +
                    y * (0.0000000001077 + y * 0.00000000000272)));
  double s, c;
  sincos(xx, &s, &c);
  return sqrt(2.0 / (kPi * ax)) * (p1 * c - z * q1 * s);
}

__device__ __forceinline__ double somm_j1(double x) {
  const double ax = fabs(x);
  double val;
  if (ax < 8.0) {
    const double y = x * x;
    const double p1 = x * (72362614232.0 + y * (-7895059235.0 + y * (242396853.1 +
                      y * (-2972611.439 + y * (15704.4882 + y * (-30.1635081))))));
    const double q1 = 144725228442.0 + y * (2300535178.0 + y * (18583304.74 +
                      y * (99447.43526 + y * (376.9949199 + y))));
    val = p1 / q1;
  } else {
    const double z = 8.0 / ax, y = z * z, xx = ax - 2.356194491;
    const double p1 = 1.0 + y * (0.000183105 + y * (-0.0000035163965 +
                      y * (0.00000002457572 + y * 2.457520e-7)));
    const double q1 = 0.040957605 + y * (-0.000004976877 + y * (0.0000000798216 +
                      y * (-0.000000000944603 + y * 4.53491e-10)));
    double s, c;
    sincos(xx, &s, &c);
    val = sqrt(2.0 / (kPi * ax)) * (p1 * c - z * q1 * s);
  }
  return x < 0.0 ? -val : val;
}

// Principal square root with Im >= 0 (csqrt_pos_im, sommerfeld.rs:161-164).
// Algebraic form of the principal branch; agrees with the polar form to
// rounding.
__device__ __forceinline__ double2 somm_csqrt(double2 z) {
  double2 s;
  if (z.y == 0.0) {
    if (!signbit(z.x)) {
      s = make_double2(sqrt(z.x), z.y);
    } else {
      const double im = sqrt(-z.x);
      s = make_double2(0.0, signbit(z.y) ? -im : im);
    }
  } else {
    const double r = hypot(z.x, z.y);
    const double t = sqrt(0.5 * (r + fabs(z.x)));
    if (z.x >= 0.0)
      s = make_double2(t, z.y / (2.0 * t));
    else
      s = make_double2(fabs(z.y) / (2.0 * t), copysign(t, z.y));
  }
  if (s.y < 0.0) s = make_double2(-s.x, -s.y);
  return s;
}

__device__ __forceinline__ double2 cscale(double2 a, double s) {
  return make_double2(a.x * s, a.y * s);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}

struct SommInt {
  double2 s_j0, p_j0, zz, xz, j2;
};

// The five integrands at one k_par (sommerfeld.rs:376-413).  k_z in the
// environment is either real (propagating) or imaginary (evanescent), so
// k_z^2 = k^2 - k_par^2 is real and the phase is a pure rotation or a pure
// decay.
__device__ __forceinline__ void somm_integrand(const SommDev& S, double kpar, double rho,
                                               double dz, double w, SommInt& acc) {
  const double k = S.k_env, k2 = k * k;
  const double q = k2 - kpar * kpar;          // k_z^2 (real)
  double2 kz, factor, phase;                  // k_z, k_par / k_z, exp(i k_z dz)
  if (q >= 0.0) {
    const double r = sqrt(q);
    kz = make_double2(r, 0.0);
    factor = make_double2(kpar / r, 0.0);
    double s, c;
    sincos(r * dz, &s, &c);
    phase = make_double2(c, s);
  } else {
    const double r = sqrt(-q);
    kz = make_double2(0.0, r);
    factor = make_double2(0.0, -kpar / r);
    phase = make_double2(exp(-r * dz), 0.0);
  }
  const double a = k2 / S.eps_env;
  const double2 kzs = somm_csqrt(make_double2(S.eps_sub.x * a - kpar * kpar, S.eps_sub.y * a));
  const double2 r_s = cdiv(make_double2(kz.x - kzs.x, kz.y - kzs.y),
                           make_double2(kz.x + kzs.x, kz.y + kzs.y));
  const double2 ek = cmul(S.eps_sub, kz);
  const double2 r_p = cdiv(make_double2(ek.x - S.eps_env * kzs.x, ek.y - S.eps_env * kzs.y),
                           make_double2(ek.x + S.eps_env * kzs.x, ek.y + S.eps_env * kzs.y));
  const double arg = kpar * rho;
  const double j0v = somm_j0(arg), j1v = somm_j1(arg);
  const double j2v = fabs(arg) < 1e-15 ? 0.0 : (2.0 / arg) * j1v - j0v;
  const double2 F = cmul(phase, factor);
  const double2 rsF = cmul(r_s, F), rpF = cmul(r_p, F);
  const double qk = q / k2, pk = kpar * kpar / k2;
  acc.s_j0 = cadd(acc.s_j0, cscale(rsF, w * j0v));
  acc.p_j0 = cadd(acc.p_j0, cscale(rpF, w * qk * j0v));
  acc.zz = cadd(acc.zz, cscale(rpF, w * pk * j0v));
  acc.j2 = cadd(acc.j2, cscale(rpF, w * qk * j2v));
  const double2 kzp = cmul(kz, phase);
  acc.xz = cadd(acc.xz, cscale(cmul(r_p, kzp), w * (kpar / k) * (1.0 / k) * j1v));
}

__device__ __forceinline__ void somm_segment(const SommDev& S, double lo, double hi, double rho,
                                             double dz, SommInt& tot) {
  const double mid = 0.5 * (lo + hi), half = 0.5 * (hi - lo);
  SommInt acc;
  acc.s_j0 = acc.p_j0 = acc.zz = acc.xz = acc.j2 = make_double2(0.0, 0.0);
#pragma unroll 1
  for (int q = 0; q < 15; ++q)
    somm_integrand(S, mid + half * c_somm_x[q], rho, dz, c_somm_w[q] * half, acc);
  tot.s_j0 = cadd(tot.s_j0, acc.s_j0);
  tot.p_j0 = cadd(tot.p_j0, acc.p_j0);
  tot.zz = cadd(tot.zz, acc.zz);
  tot.xz = cadd(tot.xz, acc.xz);
  tot.j2 = cadd(tot.j2, acc.j2);
}

// integrate (sommerfeld.rs:316-352): [0, k_env], [k_env, Re k_sub] when
// Re k_sub > 1.001 k_env, then up to k_max = max(10 ln 10 / dz, 5 k_env).
__device__ __forceinline__ SommInt somm_integrals(const SommDev& S, double rho, double dz) {
  SommInt tot;
  tot.s_j0 = tot.p_j0 = tot.zz = tot.xz = tot.j2 = make_double2(0.0, 0.0);
  const double k_env = S.k_env;
  const double k_sub_real = fmax(S.k_sub.x, k_env);
  const bool seg2 = S.k_sub.x > k_env * 1.001;
  const double k_max = dz > 1e-6 ? fmax(10.0 * 2.302585092994045684 / dz, k_env * 5.0)
                                 : k_env * 20.0;
  somm_segment(S, 0.0, k_env, rho, dz, tot);
  if (seg2) somm_segment(S, k_env, k_sub_real, rho, dz, tot);
  const double lo = seg2 ? k_sub_real : k_env;
  if (k_max > lo * 1.001) somm_segment(S, lo, k_max, rho, dz, tot);
  return tot;
}

// Record values from the integrals: A = pre (I_s + I_p), B = pre I_J2,
// Z = pre I_zz, X = pre I_xz with pre = i / (8 pi) (sommerfeld.rs:281-289).
__device__ __forceinline__ void somm_record(const SommInt& I, double2 v[4]) {
  const double pw = 1.0 / (8.0 * kPi);   // (a + ib) i pw = (-b pw, a pw)
  const double2 sp = cadd(I.s_j0, I.p_j0);
  v[0] = make_double2(-sp.y * pw, sp.x * pw);
  v[1] = make_double2(-I.j2.y * pw, I.j2.x * pw);
  v[2] = make_double2(-I.zz.y * pw, I.zz.x * pw);
  v[3] = make_double2(-I.xz.y * pw, I.xz.x * pw);
}

}  // namespace lum
