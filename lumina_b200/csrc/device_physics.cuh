// device_physics.cuh -- FP64 device restatements of the reference's Green's
// tensors, shared by the on-the-fly and the assembly kernels.  Every
// function has internal linkage (static) so each translation unit carries
// its own copy and no device linking is needed.
#pragma once
#include "lumina_internal.cuh"

namespace lum {

// Reference point tensor (greens.rs:34-71 restated on the device, FP64).
static __device__ void greens_point_d(double rx, double ry, double rz, double k, double2 g[9]) {
  double r = sqrt(rx * rx + ry * ry + rz * rz);
  double kr = k * r;
  double kr2 = kr * kr;
  double sn, cs;
  sincos(kr, &sn, &cs);
  double pf = k * k / (4.0 * kPi * r);
  double pr = pf * cs, pi = pf * sn;
  double ar = 1.0 - 1.0 / kr2, ai = 1.0 / kr;
  double br = (3.0 - kr2) / kr2, bi = -3.0 / kr;
  double rh[3] = {rx / r, ry / r, rz / r};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double d = (a == b) ? 1.0 : 0.0;
      double vr = ar * d + br * rh[a] * rh[b];
      double vi = ai * d + bi * rh[a] * rh[b];
      g[3 * a + b] = make_double2(pr * vr - pi * vi, pr * vi + pi * vr);
    }
}

// ---------------------------------------------------------------------------
// Ewald periodic tensor (ewald.rs:91-338) in FP64, for the lattice path.
// The reference includes i == j (the R = 0 image is skipped) and ignores
// FCD when a lattice is set (assembly.rs:92-104).
// ---------------------------------------------------------------------------
static __device__ double erfc_as_d(double x) {  // ewald.rs:316-327 (A&S 7.1.26)
  double ax = x;
  if (x < 0.0) ax = -x;
  double t = 1.0 / (1.0 + 0.3275911 * ax);
  double poly = t * (0.254829592 +
                     t * (-0.284496736 + t * (1.421413741 + t * (-1.453152027 + t * 1.061405429))));
  double v = poly * exp(-ax * ax);
  if (x < 0.0) v = 2.0 - v;
  return v;
}

static __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
static __device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  double nn = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / nn, (a.y * b.x - a.x * b.y) / nn);
}
// sqrt(q2) of a real q2 with Im >= 0 (ewald.rs:334-338 on a real argument)
static __device__ __forceinline__ double2 csqrt_real_posim(double q2) {
  return q2 >= 0.0 ? make_double2(sqrt(q2), 0.0) : make_double2(0.0, sqrt(-q2));
}

// Bessel functions for the 1D chain spectral sum (ewald.rs:349-713).
static __device__ double bj0(double x) {
  double ax = fabs(x);
  if (ax < 8.0) {
    double y = x * x;
    return (57568490574.0 + y * (-13362590354.0 + y * (651619640.7 + y * (-11214424.18 + y * (77392.33017 + y * -184.9052456))))) /
           (57568490411.0 + y * (1029532985.0 + y * (9494680.718 + y * (59272.64853 + y * (267.8532712 + y * 1.0)))));
  }
  double z = 8.0 / ax, y = z * z, xx = ax - 0.785398164;
  double p = 1.0 + y * (-1.098628627e-3 + y * (2.734510407e-5 + y * (-2.073370639e-6 + y * 2.093887211e-7)));
  double q = -1.562499995e-2 + y * (1.430488765e-4 + y * (-6.911147651e-6 + y * (7.621095161e-7 + y * (-9.34945152e-8))));
  return sqrt(2.0 / (kPi * ax)) * (cos(xx) * p - z * sin(xx) * q);
}
static __device__ double bj1(double x) {
  double ax = fabs(x);
  double sign = (x < 0.0) ? -1.0 : 1.0;
  if (ax < 8.0) {
    double y = x * x;
    return x * (72362614232.0 + y * (-7895059235.0 + y * (242396853.1 + y * (-2972611.439 + y * (15704.48260 + y * -30.16036606))))) /
           (144725228442.0 + y * (2300535178.0 + y * (18583304.74 + y * (99447.43394 + y * (376.9991397 + y * 1.0)))));
  }
  double z = 8.0 / ax, y = z * z, xx = ax - 2.356194491;
  double p = 1.0 + y * (1.83105e-3 + y * (-3.516396496e-5 + y * (2.457520174e-6 + y * (-2.40337019e-7))));
  double q = 4.687499995e-2 + y * (-2.002690873e-4 + y * (8.449199096e-6 + y * (-8.8228987e-7 + y * 1.05787412e-7)));
  return sign * sqrt(2.0 / (kPi * ax)) * (cos(xx) * p - z * sin(xx) * q);
}
static __device__ double by0(double x) {
  if (x <= 3.0) {
    double h = x / 2.0, s = 0.0, term = -(h * h), hk = 1.0;
    for (int k = 1; k <= 30; ++k) {
      s += term * hk;
      double kp = (double)(k + 1);
      term *= -(h * h) / (kp * kp);
      hk += 1.0 / kp;
    }
    return (2.0 / kPi) * ((log(h) + 0.5772156649015329) * bj0(x) - s);
  }
  double z = 3.0 / x, y = z * z;
  double f0 = 0.79788456 + y * (-7.7e-7 + y * (-5.52740e-3 + y * (-9.512e-5 + y * (1.37237e-3 + y * (-7.2805e-4 + y * 1.4476e-4)))));
  double th = x - 0.785398164 + z * (-4.166397e-2 + z * (-3.954e-5 + z * (2.62573e-3 + z * (-5.4125e-4 + z * (-2.9333e-4 + z * 1.3558e-4)))));
  return f0 / sqrt(x) * sin(th);
}
static __device__ double by1(double x) {
  if (x <= 3.0) {
    double h = fmax(fmin(x * 1e-3, x / 4.0), 1e-15);
    return -((-by0(x + 2.0 * h) + 8.0 * by0(x + h) - 8.0 * by0(x - h) + by0(x - 2.0 * h)) / (12.0 * h));
  }
  double z = 3.0 / x, y = z * z;
  double f1 = 0.79788456 + y * (1.564e-4 + y * (1.659667e-2 + y * (1.7105e-4 + y * (-2.49511e-3 + y * (1.13653e-3 + y * (-2.0033e-4))))));
  double th = x - 2.35619449 + z * (1.2499612e-1 + z * (5.650e-5 + z * (-6.37879e-3 + z * (7.4348e-4 + z * (7.9824e-4 + z * (-2.9166e-4))))));
  return f1 / sqrt(x) * sin(th);
}
static __device__ double bi0(double x) {
  double ax = fabs(x);
  if (ax <= 3.75) {
    double y = (x / 3.75) * (x / 3.75);
    return 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 + y * (0.2659732 + y * (0.03600768 + y * 0.0045819)))));
  }
  double y = 3.75 / ax;
  return (0.39894228 + y * (0.01328592 + y * (0.00225319 + y * (-0.00157565 + y * (0.0091669 + y * (-0.02057064 + y * (0.02635537 + y * (-0.0164708 + y * 0.00392078)))))))) *
         exp(ax) / sqrt(ax);
}
static __device__ double bi1(double x) {
  double ax = fabs(x);
  double sign = (x < 0.0) ? -1.0 : 1.0;
  double v;
  if (ax <= 3.75) {
    double y = (x / 3.75) * (x / 3.75);
    v = ax * (0.5 + y * (0.87890594 + y * (0.51498869 + y * (0.15084934 + y * (0.02658733 + y * (0.00301532 + y * 0.00032411))))));
  } else {
    double y = 3.75 / ax;
    v = (0.39894228 + y * (-0.03988024 + y * (-0.00362018 + y * (0.0163801 + y * (-0.1031555 + y * (0.2282967 + y * (-0.2895312 + y * (0.1787654 + y * (-0.0420059))))))))) *
        exp(ax) / sqrt(ax);
  }
  return sign * v;
}
static __device__ double bk0(double x) {
  if (x <= 2.0) {
    double y = (x / 2.0) * (x / 2.0);
    return -bi0(x) * log(x / 2.0) + (-0.57721566 + y * (0.42278420 + y * (0.23069756 + y * (0.03488590 + y * (0.00262698 + y * (0.00010750 + y * 0.00000074))))));
  }
  double y = 2.0 / x;
  return (1.25331414 + y * (-0.07832358 + y * (0.02189568 + y * (-0.01062446 + y * (0.00587872 + y * (-0.00251540 + y * 0.00053208)))))) * exp(-x) / sqrt(x);
}
static __device__ double bk1(double x) {
  if (x <= 2.0) {
    double y = (x / 2.0) * (x / 2.0);
    return bi1(x) * log(x / 2.0) + (1.0 + y * (0.15443144 + y * (-0.67278579 + y * (-0.18156897 + y * (-0.01919402 + y * (-0.00110404 + y * (-0.00004686))))))) / x;
  }
  double y = 2.0 / x;
  return (1.25331414 + y * (0.23498619 + y * (-0.03655620 + y * (0.01504268 + y * (-0.00780353 + y * (0.00325614 + y * (-0.00068245))))))) * exp(-x) / sqrt(x);
}
// K0/K1 of a real or purely imaginary argument (ewald.rs:635-713).
static __device__ double2 bk0c(double2 z) {
  if (fabs(z.x) < 1e-12) {
    double a = z.y;
    if (a > 0.0) return make_double2(-(kPi / 2.0) * by0(a), (kPi / 2.0) * bj0(a));
    if (a < 0.0) return make_double2(-(kPi / 2.0) * by0(-a), -(kPi / 2.0) * bj0(-a));
    return make_double2(INFINITY, 0.0);
  }
  if (fabs(z.y) < 1e-12) {
    if (z.x > 0.0) return make_double2(bk0(z.x), 0.0);
    return make_double2(bk0(-z.x), -kPi * bi0(-z.x));
  }
  double r = hypot(z.x, z.y);
  return r > 1e-12 ? make_double2(bk0(r), 0.0) : make_double2(INFINITY, 0.0);
}
static __device__ double2 bk1c(double2 z) {
  if (fabs(z.x) < 1e-12) {
    double a = z.y;
    if (a > 0.0) return make_double2(-(kPi / 2.0) * bj1(a), -(kPi / 2.0) * by1(a));
    if (a < 0.0) return make_double2((kPi / 2.0) * bj1(-a), -(kPi / 2.0) * by1(-a));
    return make_double2(INFINITY, 0.0);
  }
  if (fabs(z.y) < 1e-12) {
    if (z.x > 0.0) return make_double2(bk1(z.x), 0.0);
    return make_double2(-bk1(-z.x), kPi * bi1(-z.x));
  }
  double r = hypot(z.x, z.y);
  return r > 1e-12 ? make_double2(bk1(r), 0.0) : make_double2(INFINITY, 0.0);
}

// Periodic tensor at displacement r; g accumulates real + reciprocal sums.
static __device__ void ewald_tensor(const LatticeDev& L, const double4* __restrict__ lreal,
                             const double4* __restrict__ lrecip, double rx, double ry,
                             double rz, const double* kb, double k, double2 g[9]) {
  for (int e = 0; e < 9; ++e) g[e] = make_double2(0.0, 0.0);
  const bool r_zero = (rx * rx + ry * ry + rz * rz) < 1e-24;
  // real space (ewald.rs:119-174)
  for (int p = 0; p < L.n_real; ++p) {
    const double4 lp = lreal[p];
    const bool lp_zero = fabs(lp.x) < 1e-12 && fabs(lp.y) < 1e-12 && fabs(lp.z) < 1e-12;
    if (r_zero && lp_zero) continue;
    double sx = rx - lp.x, sy = ry - lp.y, sz = rz - lp.z;
    double s2 = sx * sx + sy * sy + sz * sz;
    if (s2 < 1e-24) continue;
    double sn_ = sqrt(s2);
    double barg = kb[0] * lp.x + kb[1] * lp.y + kb[2] * lp.z;
    double bs, bc;
    sincos(barg, &bs, &bc);
    double damp = L.is_2d ? erfc_as_d(L.eta * sn_) : 1.0;
    double2 gs[9];
    greens_point_d(sx, sy, sz, k, gs);
    double2 ph = make_double2(bc * damp, bs * damp);
    for (int e = 0; e < 9; ++e) {
      double2 t = cmul(ph, gs[e]);
      g[e].x += t.x;
      g[e].y += t.y;
    }
  }
  if (L.is_2d) {
    // 2D spectral sum (ewald.rs:196-271)
    const double inv2a = 1.0 / (2.0 * L.area);
    const double abs_z = fabs(rz);
    const double sign_z = (rz >= 0.0) ? 1.0 : -1.0;
    const double k2 = k * k;
    for (int p = 0; p < L.n_recip; ++p) {
      const double4 gp = lrecip[p];
      double qx = kb[0] + gp.x, qy = kb[1] + gp.y;
      double2 q = csqrt_real_posim(qx * qx + qy * qy - k2);
      if (hypot(q.x, q.y) < 1e-10) continue;
      double parg = qx * rx + qy * ry;
      double ps, pc;
      sincos(parg, &ps, &pc);
      // exp(-q|z|)
      double ee = exp(-q.x * abs_z);
      double es, ec;
      sincos(-q.y * abs_z, &es, &ec);
      double2 eqz = make_double2(ee * ec, ee * es);
      double2 coeff = cmul(cmul(make_double2(0.0, inv2a), make_double2(pc, ps)), eqz);
      coeff = cdiv(coeff, q);
      double2 kt[3] = {make_double2(qx, 0.0), make_double2(qy, 0.0),
                       make_double2(-q.y * sign_z, q.x * sign_z)};
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          double2 kk = cmul(kt[a], kt[b]);
          double2 m = make_double2((a == b ? k2 : 0.0) - kk.x, -kk.y);
          double2 t = cmul(coeff, m);
          g[3 * a + b].x += t.x;
          g[3 * a + b].y += t.y;
        }
    }
  } else {
    // 1D spectral sum (ewald.rs:728-804)
    const double* e = L.e_hat;
    double x_par = rx * e[0] + ry * e[1] + rz * e[2];
    double rp[3] = {rx - x_par * e[0], ry - x_par * e[1], rz - x_par * e[2]};
    double rho = sqrt(rp[0] * rp[0] + rp[1] * rp[1] + rp[2] * rp[2]);
    if (rho < 1e-10) return;
    double rh[3] = {rp[0] / rho, rp[1] / rho, rp[2] / rho};
    double kbp = kb[0] * e[0] + kb[1] * e[1] + kb[2] * e[2];
    for (long m = -L.m_max; m <= L.m_max; ++m) {
      double g_m = kbp + 2.0 * kPi * (double)m / L.a1_len;
      double2 kappa = csqrt_real_posim(g_m * g_m - k * k);
      double2 arg = make_double2(kappa.x * rho, kappa.y * rho);
      double2 k0 = bk0c(arg), k1 = bk1c(arg);
      double2 k1r = cmul(kappa, k1);
      k1r.x /= rho;
      k1r.y /= rho;
      double ps, pc;
      sincos(g_m * x_par, &ps, &pc);
      double inv = 1.0 / (2.0 * kPi * L.a1_len);
      double2 pref = make_double2(pc * inv, ps * inv);
      double2 kk0 = make_double2(k * k * k0.x, k * k * k0.y);
      double2 c_delta = cmul(pref, make_double2(kk0.x - k1r.x, kk0.y - k1r.y));
      double2 gk0 = make_double2(g_m * g_m * k0.x, g_m * g_m * k0.y);
      double2 c_ee = cmul(pref, make_double2(k1r.x - gk0.x, k1r.y - gk0.y));
      double2 c_cross = cmul(cmul(pref, make_double2(0.0, -g_m)), k1r);
      double2 kap2k0 = cmul(cmul(kappa, kappa), k0);
      double2 c_rr = cmul(pref, make_double2(kap2k0.x + 2.0 * k1r.x, kap2k0.y + 2.0 * k1r.y));
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          double d = (a == b) ? 1.0 : 0.0;
          double see = e[a] * e[b], scr = e[a] * rh[b] + e[b] * rh[a], srr = rh[a] * rh[b];
          g[3 * a + b].x += c_delta.x * d + c_ee.x * see + c_cross.x * scr + c_rr.x * srr;
          g[3 * a + b].y += c_delta.y * d + c_ee.y * see + c_cross.y * scr + c_rr.y * srr;
        }
    }
  }
}


}  // namespace lum
