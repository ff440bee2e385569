// cda_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU FP64 restatement of the reference (JonesRobM/Lumina, Rust) coupled-dipole
// solve path, used as the correctness oracle for the CUDA library and as the
// timed host-CPU baseline.  Nothing in the product (lumina_b200/) links,
// loads or calls this file; only tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py do.
//
// Parity notes
//  * The reference's complex arithmetic is num-complex 0.4.6 (Cargo.lock).
//    Its published semantics are restated in the `C` helpers below:
//    (a+bi)(c+di) = (ac-bd) + (ad+bc)i, division by c+di through
//    (c*c+d*d), norm() = hypot(re, im), exp(x+iy) = e^x (cos y + i sin y),
//    sqrt on the principal branch.  Rust does not contract a*b+c into FMA,
//    so this file is built with -ffp-contract=off.
//  * Every function cites the reference file:line it restates.
//  * Loops keep the reference's order (rows parallel, j sequential), so the
//    per-row results do not depend on the thread count.

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include <algorithm>
#include <array>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double PI = 3.14159265358979323846;

struct C {
  double re, im;
};
inline C cc(double re, double im = 0.0) { return C{re, im}; }
inline C add(C a, C b) { return C{a.re + b.re, a.im + b.im}; }
inline C sub(C a, C b) { return C{a.re - b.re, a.im - b.im}; }
inline C mul(C a, C b) { return C{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline C div(C a, C b) {
  double n = b.re * b.re + b.im * b.im;
  double re = a.re * b.re + a.im * b.im;
  double im = a.im * b.re - a.re * b.im;
  return C{re / n, im / n};
}
inline C muls(C a, double s) { return C{a.re * s, a.im * s}; }   // Complex * f64
inline C divs(C a, double s) { return C{a.re / s, a.im / s}; }   // Complex / f64
inline C conj(C a) { return C{a.re, -a.im}; }
inline C neg(C a) { return C{-a.re, -a.im}; }
inline double norm(C a) { return std::hypot(a.re, a.im); }
inline double norm_sqr(C a) { return a.re * a.re + a.im * a.im; }
inline C cexp(C a) {
  double e = std::exp(a.re);
  return C{e * std::cos(a.im), e * std::sin(a.im)};
}
// num-complex principal-branch sqrt (Re >= 0), with its special cases for
// purely real and purely imaginary arguments.
inline C csqrt(C z) {
  if (z.im == 0.0) {
    if (!std::signbit(z.re)) return C{std::sqrt(z.re), z.im};
    double im = std::sqrt(-z.re);
    return std::signbit(z.im) ? C{0.0, -im} : C{0.0, im};
  }
  if (z.re == 0.0) {
    double x = std::sqrt(std::fabs(z.im) / 2.0);
    return std::signbit(z.im) ? C{x, -x} : C{x, x};
  }
  double r = std::hypot(z.re, z.im);
  double theta = std::atan2(z.im, z.re);
  double sr = std::sqrt(r);
  double h = theta / 2.0;
  return C{sr * std::cos(h), sr * std::sin(h)};
}

typedef C T3[3][3];

// ---------------------------------------------------------------------------
// Free-space dyadic Green's tensor.  greens.rs:34-71.
// Returns false for coincident points (the reference panics there).
// ---------------------------------------------------------------------------
bool greens(const double r1[3], const double r2[3], double k, T3 g) {
  double rx = r1[0] - r2[0];
  double ry = r1[1] - r2[1];
  double rz = r1[2] - r2[2];
  double r_sq = rx * rx + ry * ry + rz * rz;
  double r = std::sqrt(r_sq);
  if (!(r > 1e-15)) return false;
  double kr = k * r;
  double kr_sq = kr * kr;
  C ikr = cc(0.0, kr);
  C exp_ikr = cexp(ikr);
  C prefactor = divs(muls(exp_ikr, k * k), 4.0 * PI * r);
  C a = add(cc(1.0), div(sub(ikr, cc(1.0)), cc(kr_sq)));
  C b = div(sub(sub(cc(3.0), mul(cc(3.0), ikr)), cc(kr_sq)), cc(kr_sq));
  double rh[3] = {rx / r, ry / r, rz / r};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double delta = (i == j) ? 1.0 : 0.0;
      g[i][j] = mul(prefactor, add(muls(a, delta), muls(muls(b, rh[i]), rh[j])));
    }
  return true;
}

// Same tensor at a displacement s.  ewald.rs:283-307.
bool greens_at(const double s[3], double k, T3 g) {
  double r_sq = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
  double r = std::sqrt(r_sq);
  if (!(r > 1e-15)) return false;
  double kr = k * r;
  C ikr = cc(0.0, kr);
  C exp_ikr = cexp(ikr);
  C prefactor = divs(muls(exp_ikr, k * k), 4.0 * PI * r);
  C a = add(cc(1.0), div(sub(ikr, cc(1.0)), cc(kr * kr)));
  C b = div(sub(sub(cc(3.0), mul(cc(3.0), ikr)), cc(kr * kr)), cc(kr * kr));
  double rh[3] = {s[0] / r, s[1] / r, s[2] / r};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double delta = (i == j) ? 1.0 : 0.0;
      g[i][j] = mul(prefactor, add(muls(a, delta), muls(muls(b, rh[i]), rh[j])));
    }
  return true;
}

// FCD / integrated Green's tensor: 27-node Gauss-Legendre cell average for
// dist <= 2*cell_size.  greens.rs:94-167.
bool greens_filtered(const double ro[3], const double rs[3], double k, double cell, T3 out) {
  double dx = ro[0] - rs[0], dy = ro[1] - rs[1], dz = ro[2] - rs[2];
  double dist = std::sqrt(dx * dx + dy * dy + dz * dz);
  if (dist > 2.0 * cell) return greens(ro, rs, k, out);
  const double nodes[3] = {-std::sqrt(3.0 / 5.0), 0.0, std::sqrt(3.0 / 5.0)};
  const double weights[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  double half_d = cell / 2.0;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) out[a][b] = cc(0.0);
  double total_w = 0.0;
  for (int ix = 0; ix < 3; ++ix)
    for (int iy = 0; iy < 3; ++iy)
      for (int iz = 0; iz < 3; ++iz) {
        double rp[3] = {rs[0] + half_d * nodes[ix], rs[1] + half_d * nodes[iy],
                        rs[2] + half_d * nodes[iz]};
        double ddx = ro[0] - rp[0], ddy = ro[1] - rp[1], ddz = ro[2] - rp[2];
        double r_sq = ddx * ddx + ddy * ddy + ddz * ddz;
        if (r_sq < 1e-20) continue;
        double w = weights[ix] * weights[iy] * weights[iz];
        T3 g;
        greens(ro, rp, k, g);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) out[a][b] = add(out[a][b], mul(cc(w), g[a][b]));
        total_w += w;
      }
  if (total_w > 1e-30) {
    C inv_w = cc(1.0 / total_w);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) out[a][b] = mul(out[a][b], inv_w);
  }
  return true;
}

// 3x3 complex cofactor inverse.  assembly.rs:335-363.
bool invert3(const C m[9], C out[9]) {
  C a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], k = m[8];
  C det = add(sub(mul(a, sub(mul(e, k), mul(f, h))), mul(b, sub(mul(d, k), mul(f, g)))),
              mul(c, sub(mul(d, h), mul(e, g))));
  if (!(norm(det) > 1e-30)) return false;
  C inv_det = div(cc(1.0), det);
  out[0] = mul(inv_det, sub(mul(e, k), mul(f, h)));
  out[1] = mul(inv_det, sub(mul(c, h), mul(b, k)));
  out[2] = mul(inv_det, sub(mul(b, f), mul(c, e)));
  out[3] = mul(inv_det, sub(mul(f, g), mul(d, k)));
  out[4] = mul(inv_det, sub(mul(a, k), mul(c, g)));
  out[5] = mul(inv_det, sub(mul(c, d), mul(a, f)));
  out[6] = mul(inv_det, sub(mul(d, h), mul(e, g)));
  out[7] = mul(inv_det, sub(mul(b, g), mul(a, h)));
  out[8] = mul(inv_det, sub(mul(a, e), mul(b, d)));
  return true;
}

// ---------------------------------------------------------------------------
// Ewald periodic Green's tensor.  ewald.rs:67-338, 340-804; lattice.rs:29-233.
// ---------------------------------------------------------------------------
struct Lattice {
  double a1[3], a2[3];
  int is_2d;
  int has_eta;
  double eta;
  int trunc_real, trunc_recip;
};

double cell_measure(const Lattice& L) {  // lattice.rs:75-89
  if (L.is_2d) {
    double cx = L.a1[1] * L.a2[2] - L.a1[2] * L.a2[1];
    double cy = L.a1[2] * L.a2[0] - L.a1[0] * L.a2[2];
    double cz = L.a1[0] * L.a2[1] - L.a1[1] * L.a2[0];
    return std::sqrt(cx * cx + cy * cy + cz * cz);
  }
  return std::sqrt(L.a1[0] * L.a1[0] + L.a1[1] * L.a1[1] + L.a1[2] * L.a1[2]);
}

double lattice_eta(const Lattice& L) {  // lattice.rs:96-102
  if (L.has_eta) return L.eta;
  return std::sqrt(PI / cell_measure(L));
}

// lattice.rs:168-196 (m1 outer, m2 inner; origin included)
std::vector<std::array<double, 3>> real_points(const Lattice& L, int ns) {
  std::vector<std::array<double, 3>> pts;
  if (L.is_2d) {
    for (int m1 = -ns; m1 <= ns; ++m1)
      for (int m2 = -ns; m2 <= ns; ++m2)
        pts.push_back({(double)m1 * L.a1[0] + (double)m2 * L.a2[0],
                       (double)m1 * L.a1[1] + (double)m2 * L.a2[1],
                       (double)m1 * L.a1[2] + (double)m2 * L.a2[2]});
  } else {
    for (int m1 = -ns; m1 <= ns; ++m1)
      pts.push_back({(double)m1 * L.a1[0], (double)m1 * L.a1[1], (double)m1 * L.a1[2]});
  }
  return pts;
}

// lattice.rs:113-147 and 153-161, 203-233.
std::vector<std::array<double, 3>> recip_points(const Lattice& L, int ns) {
  std::vector<std::array<double, 3>> pts;
  const double two_pi = 2.0 * PI;
  if (L.is_2d) {
    const double* a1 = L.a1;
    const double* a2 = L.a2;
    double a2xz[3] = {a2[1], -a2[0], 0.0};
    double denom1 = a1[0] * a2xz[0] + a1[1] * a2xz[1];
    double b1[3] = {two_pi * a2xz[0] / denom1, two_pi * a2xz[1] / denom1, 0.0};
    double zxa1[3] = {-a1[1], a1[0], 0.0};
    double denom2 = a2[0] * zxa1[0] + a2[1] * zxa1[1];
    double b2[3] = {two_pi * zxa1[0] / denom2, two_pi * zxa1[1] / denom2, 0.0};
    for (int n1 = -ns; n1 <= ns; ++n1)
      for (int n2 = -ns; n2 <= ns; ++n2)
        pts.push_back({(double)n1 * b1[0] + (double)n2 * b2[0],
                       (double)n1 * b1[1] + (double)n2 * b2[1], 0.0});
  } else {
    double x = L.a1[0], y = L.a1[1], z = L.a1[2];
    double len_sq = x * x + y * y + z * z;
    double scale = 2.0 * PI / len_sq;
    double b1[3] = {x * scale, y * scale, z * scale};
    for (int n1 = -ns; n1 <= ns; ++n1)
      pts.push_back({(double)n1 * b1[0], (double)n1 * b1[1], (double)n1 * b1[2]});
  }
  return pts;
}

// A&S 7.1.26 rational erfc.  ewald.rs:316-327.
double erfc_as(double x) {
  if (x < 0.0) return 2.0 - erfc_as(-x);
  double t = 1.0 / (1.0 + 0.3275911 * x);
  double poly = t * (0.254829592 +
                     t * (-0.284496736 + t * (1.421413741 + t * (-1.453152027 + t * 1.061405429))));
  return poly * std::exp(-x * x);
}

// ewald.rs:334-338
C csqrt_pos_imag(C z) {
  C s = csqrt(z);
  return (s.im < 0.0) ? neg(s) : s;
}

// Bessel functions, ewald.rs:340-713 (Numerical Recipes 6.5 / A&S 9.4, 9.8).
const double GAMMA_EM = 0.5772156649015329;

double bessel_j0(double x) {
  double ax = std::fabs(x);
  if (ax < 8.0) {
    double y = x * x;
    return (57568490574.0 + y * (-13362590354.0 + y * (651619640.7 + y * (-11214424.18 + y * (77392.33017 + y * -184.9052456))))) /
           (57568490411.0 + y * (1029532985.0 + y * (9494680.718 + y * (59272.64853 + y * (267.8532712 + y * 1.0)))));
  }
  double z = 8.0 / ax, y = z * z, xx = ax - 0.785398164;
  double p = 1.0 + y * (-1.098628627e-3 + y * (2.734510407e-5 + y * (-2.073370639e-6 + y * 2.093887211e-7)));
  double q = -1.562499995e-2 + y * (1.430488765e-4 + y * (-6.911147651e-6 + y * (7.621095161e-7 + y * (-9.34945152e-8))));
  return std::sqrt(2.0 / (PI * ax)) * (std::cos(xx) * p - z * std::sin(xx) * q);
}

double bessel_j1(double x) {
  double ax = std::fabs(x);
  double sign = (x < 0.0) ? -1.0 : 1.0;
  if (ax < 8.0) {
    double y = x * x;
    return x * (72362614232.0 + y * (-7895059235.0 + y * (242396853.1 + y * (-2972611.439 + y * (15704.48260 + y * -30.16036606))))) /
           (144725228442.0 + y * (2300535178.0 + y * (18583304.74 + y * (99447.43394 + y * (376.9991397 + y * 1.0)))));
  }
  double z = 8.0 / ax, y = z * z, xx = ax - 2.356194491;
  double p = 1.0 + y * (1.83105e-3 + y * (-3.516396496e-5 + y * (2.457520174e-6 + y * (-2.40337019e-7))));
  double q = 4.687499995e-2 + y * (-2.002690873e-4 + y * (8.449199096e-6 + y * (-8.8228987e-7 + y * 1.05787412e-7)));
  return sign * std::sqrt(2.0 / (PI * ax)) * (std::cos(xx) * p - z * std::sin(xx) * q);
}

double bessel_y0(double x) {
  if (x <= 3.0) {
    double h = x / 2.0;
    double s = 0.0, term = -(h * h), hk = 1.0;
    for (int k = 1; k <= 30; ++k) {
      s += term * hk;
      double kp = (double)(k + 1);
      term *= -(h * h) / (kp * kp);
      hk += 1.0 / kp;
    }
    return (2.0 / PI) * ((std::log(h) + GAMMA_EM) * bessel_j0(x) - s);
  }
  double z = 3.0 / x, y = z * z;
  double f0 = 0.79788456 + y * (-7.7e-7 + y * (-5.52740e-3 + y * (-9.512e-5 + y * (1.37237e-3 + y * (-7.2805e-4 + y * 1.4476e-4)))));
  double th = x - 0.785398164 + z * (-4.166397e-2 + z * (-3.954e-5 + z * (2.62573e-3 + z * (-5.4125e-4 + z * (-2.9333e-4 + z * 1.3558e-4)))));
  return f0 / std::sqrt(x) * std::sin(th);
}

double bessel_y1(double x) {
  if (x <= 3.0) {
    double h = std::max(std::min(x * 1e-3, x / 4.0), 1e-15);
    double ypp = bessel_y0(x + 2.0 * h), yp = bessel_y0(x + h);
    double ym = bessel_y0(x - h), ymm = bessel_y0(x - 2.0 * h);
    return -((-ypp + 8.0 * yp - 8.0 * ym + ymm) / (12.0 * h));
  }
  double z = 3.0 / x, y = z * z;
  double f1 = 0.79788456 + y * (1.564e-4 + y * (1.659667e-2 + y * (1.7105e-4 + y * (-2.49511e-3 + y * (1.13653e-3 + y * (-2.0033e-4))))));
  double th = x - 2.35619449 + z * (1.2499612e-1 + z * (5.650e-5 + z * (-6.37879e-3 + z * (7.4348e-4 + z * (7.9824e-4 + z * (-2.9166e-4))))));
  return f1 / std::sqrt(x) * std::sin(th);
}

double bessel_i0(double x) {
  double ax = std::fabs(x);
  if (ax <= 3.75) {
    double y = (x / 3.75) * (x / 3.75);
    return 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 + y * (0.2659732 + y * (0.03600768 + y * 0.0045819)))));
  }
  double y = 3.75 / ax;
  double poly = 0.39894228 + y * (0.01328592 + y * (0.00225319 + y * (-0.00157565 + y * (0.0091669 + y * (-0.02057064 + y * (0.02635537 + y * (-0.0164708 + y * 0.00392078)))))));
  return poly * std::exp(ax) / std::sqrt(ax);
}

double bessel_i1(double x) {
  double ax = std::fabs(x);
  double sign = (x < 0.0) ? -1.0 : 1.0;
  double val;
  if (ax <= 3.75) {
    double y = (x / 3.75) * (x / 3.75);
    val = ax * (0.5 + y * (0.87890594 + y * (0.51498869 + y * (0.15084934 + y * (0.02658733 + y * (0.00301532 + y * 0.00032411))))));
  } else {
    double y = 3.75 / ax;
    double poly = 0.39894228 + y * (-0.03988024 + y * (-0.00362018 + y * (0.0163801 + y * (-0.1031555 + y * (0.2282967 + y * (-0.2895312 + y * (0.1787654 + y * (-0.0420059))))))));
    val = poly * std::exp(ax) / std::sqrt(ax);
  }
  return sign * val;
}

double bessel_k0(double x) {
  if (x <= 2.0) {
    double y = (x / 2.0) * (x / 2.0);
    double poly = -0.57721566 + y * (0.42278420 + y * (0.23069756 + y * (0.03488590 + y * (0.00262698 + y * (0.00010750 + y * 0.00000074)))));
    return -bessel_i0(x) * std::log(x / 2.0) + poly;
  }
  double y = 2.0 / x;
  double poly = 1.25331414 + y * (-0.07832358 + y * (0.02189568 + y * (-0.01062446 + y * (0.00587872 + y * (-0.00251540 + y * 0.00053208)))));
  return poly * std::exp(-x) / std::sqrt(x);
}

double bessel_k1(double x) {
  if (x <= 2.0) {
    double y = (x / 2.0) * (x / 2.0);
    double poly = 1.0 + y * (0.15443144 + y * (-0.67278579 + y * (-0.18156897 + y * (-0.01919402 + y * (-0.00110404 + y * (-0.00004686))))));
    return bessel_i1(x) * std::log(x / 2.0) + poly / x;
  }
  double y = 2.0 / x;
  double poly = 1.25331414 + y * (0.23498619 + y * (-0.03655620 + y * (0.01504268 + y * (-0.00780353 + y * (0.00325614 + y * (-0.00068245))))));
  return poly * std::exp(-x) / std::sqrt(x);
}

// ewald.rs:635-675.  The reference's "general complex" branch is a
// debug_assert!(false) followed by a real-argument fallback; the release
// behaviour (the fallback) is restated.
C bessel_k0c(C z) {
  if (std::fabs(z.re) < 1e-12) {
    double a = z.im;
    if (a > 0.0) return C{-(PI / 2.0) * bessel_y0(a), (PI / 2.0) * bessel_j0(a)};
    if (a < 0.0) return C{-(PI / 2.0) * bessel_y0(-a), -(PI / 2.0) * bessel_j0(-a)};
    return C{INFINITY, 0.0};
  }
  if (std::fabs(z.im) < 1e-12) {
    if (z.re > 0.0) return C{bessel_k0(z.re), 0.0};
    double xp = -z.re;
    return C{bessel_k0(xp), -PI * bessel_i0(xp)};
  }
  double r = norm(z);
  return (r > 1e-12) ? C{bessel_k0(r), 0.0} : C{INFINITY, 0.0};
}

// ewald.rs:682-713
C bessel_k1c(C z) {
  if (std::fabs(z.re) < 1e-12) {
    double a = z.im;
    if (a > 0.0) return C{-(PI / 2.0) * bessel_j1(a), -(PI / 2.0) * bessel_y1(a)};
    if (a < 0.0) return C{(PI / 2.0) * bessel_j1(-a), -(PI / 2.0) * bessel_y1(-a)};
    return C{INFINITY, 0.0};
  }
  if (std::fabs(z.im) < 1e-12) {
    if (z.re > 0.0) return C{bessel_k1(z.re), 0.0};
    double xp = -z.re;
    return C{-bessel_k1(xp), PI * bessel_i1(xp)};
  }
  double r = norm(z);
  return (r > 1e-12) ? C{bessel_k1(r), 0.0} : C{INFINITY, 0.0};
}

// Real-space sum.  ewald.rs:119-174.
void ewald_real(const Lattice& L, const double r[3], const double kb[3], double k, T3 g) {
  double r_norm_sq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  bool r_zero = r_norm_sq < 1e-24;
  double eta = lattice_eta(L);
  int ns = L.is_2d ? L.trunc_real : std::max(L.trunc_real, 20);
  auto pts = real_points(L, ns);
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) g[a][b] = cc(0.0);
  for (auto& lp : pts) {
    bool lp_zero = std::fabs(lp[0]) < 1e-12 && std::fabs(lp[1]) < 1e-12 && std::fabs(lp[2]) < 1e-12;
    if (r_zero && lp_zero) continue;
    double s[3] = {r[0] - lp[0], r[1] - lp[1], r[2] - lp[2]};
    double s_sq = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
    if (s_sq < 1e-24) continue;
    double s_norm = std::sqrt(s_sq);
    double barg = kb[0] * lp[0] + kb[1] * lp[1] + kb[2] * lp[2];
    C phase = C{std::cos(barg), std::sin(barg)};
    double damp = L.is_2d ? erfc_as(eta * s_norm) : 1.0;
    T3 gs{};  // greens_at fills it: s_sq >= 1e-24 above
    greens_at(s, k, gs);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) g[a][b] = add(g[a][b], mul(muls(phase, damp), gs[a][b]));
  }
}

// 1D spectral sum.  ewald.rs:728-804.
void ewald_recip_1d(const double r[3], const double kb[3], double k, const double a1[3], T3 t) {
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) t[a][b] = cc(0.0);
  double a1_len = std::sqrt(a1[0] * a1[0] + a1[1] * a1[1] + a1[2] * a1[2]);
  double e[3] = {a1[0] / a1_len, a1[1] / a1_len, a1[2] / a1_len};
  double x_par = r[0] * e[0] + r[1] * e[1] + r[2] * e[2];
  double rp[3] = {r[0] - x_par * e[0], r[1] - x_par * e[1], r[2] - x_par * e[2]};
  double rho = std::sqrt(rp[0] * rp[0] + rp[1] * rp[1] + rp[2] * rp[2]);
  if (rho < 1e-10) return;
  double rh[3] = {rp[0] / rho, rp[1] / rho, rp[2] / rho};
  double kbp = kb[0] * e[0] + kb[1] * e[1] + kb[2] * e[2];
  long m_max = std::min((long)std::ceil(k * a1_len / (2.0 * PI) + 10.0), 50L);
  for (long m = -m_max; m <= m_max; ++m) {
    double g_m = kbp + 2.0 * PI * (double)m / a1_len;
    C kappa = csqrt_pos_imag(C{g_m * g_m - k * k, 0.0});
    C arg = muls(kappa, rho);
    C k0 = bessel_k0c(arg);
    C k1 = bessel_k1c(arg);
    C k1_rho = divs(mul(kappa, k1), rho);
    C phase = cexp(C{0.0, g_m * x_par});
    C pref = divs(phase, 2.0 * PI * a1_len);
    C c_delta = mul(pref, sub(mul(cc(k * k), k0), k1_rho));
    C c_ee = mul(pref, sub(k1_rho, mul(cc(g_m * g_m), k0)));
    C c_cross = mul(mul(pref, C{0.0, -g_m}), k1_rho);
    C c_rr = mul(pref, add(mul(mul(kappa, kappa), k0), mul(cc(2.0), k1_rho)));
    for (int al = 0; al < 3; ++al)
      for (int be = 0; be < 3; ++be) {
        C delta = (al == be) ? cc(1.0) : cc(0.0);
        C term = add(add(add(mul(c_delta, delta), muls(c_ee, e[al] * e[be])),
                         muls(c_cross, e[al] * rh[be] + e[be] * rh[al])),
                     muls(c_rr, rh[al] * rh[be]));
        t[al][be] = add(t[al][be], term);
      }
  }
}

// Reciprocal-space sum.  ewald.rs:186-273.
void ewald_recip(const Lattice& L, const double r[3], const double kb[3], double k, T3 g) {
  if (!L.is_2d) {
    ewald_recip_1d(r, kb, k, L.a1, g);
    return;
  }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) g[a][b] = cc(0.0);
  double area = cell_measure(L);
  auto pts = recip_points(L, L.trunc_recip);
  C iu = C{0.0, 1.0};
  C scalar_pre = divs(iu, 2.0 * area);
  double rho_x = r[0], rho_y = r[1], z = r[2];
  double abs_z = std::fabs(z);
  double sign_z = (z >= 0.0) ? 1.0 : -1.0;
  C k2 = cc(k * k);
  for (auto& gp : pts) {
    double qx = kb[0] + gp[0];
    double qy = kb[1] + gp[1];
    double q2_real = qx * qx + qy * qy;
    C q = csqrt_pos_imag(sub(cc(q2_real), k2));
    if (norm(q) < 1e-10) continue;
    double parg = qx * rho_x + qy * rho_y;
    C bphase = C{std::cos(parg), std::sin(parg)};
    C exp_qz = cexp(muls(neg(q), abs_z));
    C coeff = div(mul(mul(scalar_pre, bphase), exp_qz), q);
    C kt[3] = {cc(qx), cc(qy), muls(mul(iu, q), sign_z)};
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        C delta = (a == b) ? k2 : cc(0.0);
        C m_ab = sub(delta, mul(kt[a], kt[b]));
        g[a][b] = add(g[a][b], mul(coeff, m_ab));
      }
  }
}

// ewald.rs:91-106
void ewald_eval(const Lattice& L, const double r[3], const double kb[3], double k, T3 g) {
  T3 gr, gg;
  ewald_real(L, r, kb, k, gr);
  ewald_recip(L, r, kb, k, gg);
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) g[a][b] = add(gr[a][b], gg[a][b]);
}

struct Substrate {
  double z_interface;
  double refl_re, refl_im;
};

// Per-pair contribution to A[i][j] as a 3x3 block, following the branch
// structure of assembly.rs:87-170 (assembly) and :238-305 (matvec).
// `direct` gets the -G term (skipped for i==j in free space), `sub_blk`
// gets the -m[col]*G_img substrate term.
struct PairCfg {
  double k;
  int use_fcd;
  double cell;
  const Lattice* lat;
  double kb[3];
  const Substrate* sub;
};

void pair_blocks(const PairCfg& P, const double* ri, const double* rj, bool same, T3 direct,
                 bool* has_direct, T3 subb, bool* has_sub) {
  *has_direct = false;
  *has_sub = false;
  bool skip_direct = same && P.lat == nullptr;
  if (!skip_direct) {
    if (P.lat) {
      double r[3] = {ri[0] - rj[0], ri[1] - rj[1], ri[2] - rj[2]};
      ewald_eval(*P.lat, r, P.kb, P.k, direct);
    } else if (P.use_fcd) {
      greens_filtered(ri, rj, P.k, P.cell, direct);
    } else {
      greens(ri, rj, P.k, direct);
    }
    *has_direct = true;
  }
  if (P.sub) {
    double img[3] = {rj[0], rj[1], 2.0 * P.sub->z_interface - rj[2]};
    double diff[3] = {ri[0] - img[0], ri[1] - img[1], ri[2] - img[2]};
    double dsq = diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2];
    if (dsq >= 1e-20) {
      if (P.lat)
        ewald_eval(*P.lat, diff, P.kb, P.k, subb);
      else
        greens(ri, img, P.k, subb);
      *has_sub = true;
    }
  }
}

void load_c(const double* p, C* out, int n) {
  for (int i = 0; i < n; ++i) out[i] = C{p[2 * i], p[2 * i + 1]};
}

int set_threads(int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) return nthreads;
  return omp_get_max_threads();
#else
  (void)nthreads;
  return 1;
#endif
}

// ---------------------------------------------------------------------------
// GMRES(min(30,n)), restated from iterative.rs:33-206.
// ---------------------------------------------------------------------------
typedef void (*MatvecCb)(void* ctx, const C* x, C* y);

double vnorm(const std::vector<C>& v) {  // iterative.rs:171-173
  double s = 0.0;
  for (auto& c : v) s += norm_sqr(c);
  return std::sqrt(s);
}
C vdot(const std::vector<C>& a, const std::vector<C>& b) {  // iterative.rs:163-168
  C s = cc(0.0);
  for (size_t i = 0; i < a.size(); ++i) s = add(s, mul(conj(a[i]), b[i]));
  return s;
}
void givens(C a, C b, double* c, C* s) {  // iterative.rs:180-191
  if (norm(b) < 1e-30) {
    *c = 1.0;
    *s = cc(0.0);
    return;
  }
  if (norm(a) < 1e-30) {
    *c = 0.0;
    *s = div(b, cc(norm(b)));
    return;
  }
  double r = std::sqrt(norm_sqr(a) + norm_sqr(b));
  *c = norm(a) / r;
  *s = div(mul(div(a, cc(norm(a))), conj(b)), cc(r));
}

struct GmresOut {
  int status;  // 0 converged, 4 not converged
  int iterations;
  int matvecs;
  int restarts;
  double rel_residual;
};

GmresOut gmres(MatvecCb mv, void* ctx, const std::vector<C>& rhs, double tol, int max_iter,
               int restart_max, std::vector<C>& x) {
  GmresOut out{0, 0, 0, 0, 0.0};
  size_t n = rhs.size();
  int m = (int)std::min<size_t>((size_t)restart_max, n);
  x.assign(n, cc(0.0));
  double rhs_norm = vnorm(rhs);
  if (rhs_norm < 1e-30) return out;
  double abs_tol = tol * rhs_norm;
  int total = 0;
  std::vector<C> tmp(n);
  for (;;) {
    // r = rhs - A x   (iterative.rs:55)
    mv(ctx, x.data(), tmp.data());
    out.matvecs++;
    std::vector<C> r(n);
    for (size_t i = 0; i < n; ++i) r[i] = sub(rhs[i], tmp[i]);
    double beta = vnorm(r);
    if (beta < abs_tol) {
      out.iterations = total;
      out.rel_residual = beta / rhs_norm;
      return out;
    }
    if (total >= max_iter) {
      out.status = 4;
      out.iterations = total;
      out.rel_residual = beta / rhs_norm;
      return out;
    }
    std::vector<std::vector<C>> V;
    V.reserve(m + 1);
    {
      std::vector<C> v0(n);
      for (size_t i = 0; i < n; ++i) v0[i] = div(r[i], cc(beta));
      V.push_back(std::move(v0));
    }
    std::vector<C> H((size_t)(m + 1) * m, cc(0.0));
    auto h = [&](int i, int j) -> C& { return H[(size_t)i * m + j]; };
    std::vector<double> cs;
    std::vector<C> sn;
    std::vector<C> g(m + 1, cc(0.0));
    g[0] = cc(beta);
    int j = 0;
    while (j < m && total < max_iter) {
      std::vector<C> w(n);
      mv(ctx, V[j].data(), w.data());
      out.matvecs++;
      for (int i = 0; i <= j; ++i) {  // modified Gram-Schmidt, :92-96
        C hij = vdot(V[i], w);
        h(i, j) = hij;
        for (size_t q = 0; q < n; ++q) w[q] = sub(w[q], mul(V[i][q], hij));
      }
      double hn = vnorm(w);
      h(j + 1, j) = cc(hn);
      if (hn > 1e-30) {
        std::vector<C> v(n);
        for (size_t q = 0; q < n; ++q) v[q] = div(w[q], cc(hn));
        V.push_back(std::move(v));
      } else {
        V.push_back(std::vector<C>(n, cc(0.0)));
      }
      for (int i = 0; i < j; ++i) {  // :109-113
        C temp = add(mul(cc(cs[i]), h(i, j)), mul(sn[i], h(i + 1, j)));
        h(i + 1, j) = add(mul(neg(conj(sn[i])), h(i, j)), mul(cc(cs[i]), h(i + 1, j)));
        h(i, j) = temp;
      }
      double c;
      C s;
      givens(h(j, j), h(j + 1, j), &c, &s);
      cs.push_back(c);
      sn.push_back(s);
      C temp = add(mul(cc(c), h(j, j)), mul(s, h(j + 1, j)));
      h(j + 1, j) = cc(0.0);
      h(j, j) = temp;
      C tg = add(mul(cc(c), g[j]), mul(s, g[j + 1]));
      g[j + 1] = add(mul(neg(conj(s)), g[j]), mul(cc(c), g[j + 1]));
      g[j] = tg;
      total++;
      j++;
      if (norm(g[j]) < abs_tol) break;
    }
    // back substitution, :194-206
    std::vector<C> y(j, cc(0.0));
    for (int i = j - 1; i >= 0; --i) {
      C sum = g[i];
      for (int q = i + 1; q < j; ++q) sum = sub(sum, mul(h(i, q), y[q]));
      if (norm(h(i, i)) > 1e-30) y[i] = div(sum, h(i, i));
    }
    for (int i = 0; i < j; ++i)
      for (size_t q = 0; q < n; ++q) x[q] = add(x[q], mul(V[i][q], y[i]));
    out.restarts++;
    mv(ctx, x.data(), tmp.data());
    out.matvecs++;
    double res = 0.0;
    for (size_t q = 0; q < n; ++q) res += norm_sqr(sub(rhs[q], tmp[q]));
    res = std::sqrt(res);
    if (res < abs_tol) {
      out.iterations = total;
      out.rel_residual = res / rhs_norm;
      return out;
    }
    if (total >= max_iter) {
      out.status = 4;
      out.iterations = total;
      out.rel_residual = res / rhs_norm;
      return out;
    }
  }
}

struct DenseCtx {
  int n;
  const C* A;
  int nthreads;
};
void dense_mv(void* vctx, const C* x, C* y) {
  DenseCtx* d = (DenseCtx*)vctx;
  int n = d->n;
#pragma omp parallel for schedule(static) num_threads(d->nthreads)
  for (int i = 0; i < n; ++i) {
    C s = cc(0.0);
    const C* row = d->A + (size_t)i * n;
    for (int j = 0; j < n; ++j) s = add(s, mul(row[j], x[j]));
    y[i] = s;
  }
}

struct OtfCtx {
  int n;
  const double* pos;
  const C* inv_alpha;  // 9 per dipole
  PairCfg P;
  int nthreads;
};

// On-the-fly matvec: assembly.rs:209-318.  inv_alpha is precomputed once
// (the reference inverts per row per call, with identical arithmetic).
void otf_mv(void* vctx, const C* x, C* y) {
  OtfCtx* o = (OtfCtx*)vctx;
  int n = o->n;
#pragma omp parallel for schedule(dynamic, 16) num_threads(o->nthreads)
  for (int i = 0; i < n; ++i) {
    C yi[3] = {cc(0.0), cc(0.0), cc(0.0)};
    const C* ia = o->inv_alpha + 9 * (size_t)i;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) yi[a] = add(yi[a], mul(ia[3 * a + b], x[3 * i + b]));
    const double* ri = o->pos + 3 * (size_t)i;
    for (int j = 0; j < n; ++j) {
      const double* rj = o->pos + 3 * (size_t)j;
      T3 dg, sg;
      bool hd, hs;
      pair_blocks(o->P, ri, rj, i == j, dg, &hd, sg, &hs);
      if (hd)
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) yi[a] = sub(yi[a], mul(dg[a][b], x[3 * j + b]));
      if (hs) {
        C rr = C{o->P.sub->refl_re, o->P.sub->refl_im};
        C m[3] = {neg(rr), neg(rr), rr};
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) yi[a] = sub(yi[a], mul(mul(m[b], sg[a][b]), x[3 * j + b]));
      }
    }
    y[3 * i] = yi[0];
    y[3 * i + 1] = yi[1];
    y[3 * i + 2] = yi[2];
  }
}

void matvec_cb_dense(void* ctx, const C* x, C* y) { dense_mv(ctx, x, y); }
void matvec_cb_otf(void* ctx, const C* x, C* y) { otf_mv(ctx, x, y); }

bool prepare_inv_alpha(int n, const double* alpha, std::vector<C>& inv) {
  inv.resize((size_t)9 * n);
  for (int i = 0; i < n; ++i) {
    C m[9];
    load_c(alpha + 18 * (size_t)i, m, 9);
    if (!invert3(m, &inv[9 * (size_t)i])) return false;
  }
  return true;
}

PairCfg make_cfg(double k, int use_fcd, double cell, const Lattice* lat, const double* kb,
                 const Substrate* sub) {
  PairCfg P;
  P.k = k;
  P.use_fcd = use_fcd;
  P.cell = cell;
  P.lat = lat;
  P.kb[0] = kb ? kb[0] : 0.0;
  P.kb[1] = kb ? kb[1] : 0.0;
  P.kb[2] = kb ? kb[2] : 0.0;
  P.sub = sub;
  return P;
}

}  // namespace

// ===========================================================================
// extern "C" surface for the Python test harness (tests/, bench.py baseline)
// Complex arrays are interleaved (re, im) doubles.
// ===========================================================================
extern "C" {

typedef struct {
  double a1[3];
  double a2[3];
  int is_2d;
  int has_eta;
  double eta;
  int truncation_real;
  int truncation_recip;
} orc_lattice;

typedef struct {
  double z_interface;
  double refl_re;
  double refl_im;
} orc_substrate;

static Lattice to_lat(const orc_lattice* l) {
  Lattice L;
  for (int i = 0; i < 3; ++i) {
    L.a1[i] = l->a1[i];
    L.a2[i] = l->a2[i];
  }
  L.is_2d = l->is_2d;
  L.has_eta = l->has_eta;
  L.eta = l->eta;
  L.trunc_real = l->truncation_real;
  L.trunc_recip = l->truncation_recip;
  return L;
}

static void store_t3(const T3 g, double* out) {
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      out[2 * (3 * a + b)] = g[a][b].re;
      out[2 * (3 * a + b) + 1] = g[a][b].im;
    }
}

int orc_greens(const double* r1, const double* r2, double k, double* out18) {
  T3 g;
  if (!greens(r1, r2, k, g)) return 1;
  store_t3(g, out18);
  return 0;
}

int orc_greens_filtered(const double* r1, const double* r2, double k, double cell, double* out18) {
  T3 g;
  if (!greens_filtered(r1, r2, k, cell, g)) return 1;
  store_t3(g, out18);
  return 0;
}

int orc_invert_3x3(const double* m18, double* out18) {
  C m[9], o[9];
  load_c(m18, m, 9);
  if (!invert3(m, o)) return 1;
  for (int i = 0; i < 9; ++i) {
    out18[2 * i] = o[i].re;
    out18[2 * i + 1] = o[i].im;
  }
  return 0;
}

// IncidentField::at_position, types.rs:60-73; assembly.rs:178-194
void orc_incident_field(int n, const double* pos, const double* dir, const double* pol,
                        double amplitude, double k, double* rhs) {
  for (int i = 0; i < n; ++i) {
    const double* p = pos + 3 * (size_t)i;
    double kdotr = k * (dir[0] * p[0] + dir[1] * p[1] + dir[2] * p[2]);
    C phase = cexp(C{0.0, kdotr});
    C e0 = cc(amplitude);
    for (int c = 0; c < 3; ++c) {
      C e = mul(muls(e0, pol[c]), phase);
      rhs[2 * (3 * (size_t)i + c)] = e.re;
      rhs[2 * (3 * (size_t)i + c) + 1] = e.im;
    }
  }
}

void orc_ewald_evaluate(const orc_lattice* lat, const double* r, const double* kb, double k,
                        int part /*0 full,1 real,2 recip*/, double* out18) {
  Lattice L = to_lat(lat);
  T3 g;
  if (part == 1)
    ewald_real(L, r, kb, k, g);
  else if (part == 2)
    ewald_recip(L, r, kb, k, g);
  else
    ewald_eval(L, r, kb, k, g);
  store_t3(g, out18);
}

double orc_lattice_eta(const orc_lattice* lat) { return lattice_eta(to_lat(lat)); }
double orc_erfc(double x) { return erfc_as(x); }
void orc_csqrt_pos_imag(double re, double im, double* out2) {
  C s = csqrt_pos_imag(C{re, im});
  out2[0] = s.re;
  out2[1] = s.im;
}
double orc_bessel(int which, double x) {
  switch (which) {
    case 0: return bessel_j0(x);
    case 1: return bessel_j1(x);
    case 2: return bessel_y0(x);
    case 3: return bessel_y1(x);
    case 4: return bessel_i0(x);
    case 5: return bessel_i1(x);
    case 6: return bessel_k0(x);
    case 7: return bessel_k1(x);
  }
  return NAN;
}
void orc_bessel_kc(int which, double re, double im, double* out2) {
  C r = which == 0 ? bessel_k0c(C{re, im}) : bessel_k1c(C{re, im});
  out2[0] = r.re;
  out2[1] = r.im;
}

// Dense interaction matrix.  assembly.rs:45-175.  A is (3N)x(3N) interleaved.
int orc_assemble(int n, const double* pos, const double* alpha, double k, int use_fcd,
                 double cell, const orc_lattice* lat, const double* kb, const orc_substrate* subs,
                 double* A, int nthreads) {
  std::vector<C> inv;
  if (!prepare_inv_alpha(n, alpha, inv)) return 6;
  Lattice L;
  if (lat) L = to_lat(lat);
  Substrate S;
  if (subs) S = Substrate{subs->z_interface, subs->refl_re, subs->refl_im};
  PairCfg P = make_cfg(k, use_fcd, cell, lat ? &L : nullptr, kb, subs ? &S : nullptr);
  size_t dim = 3 * (size_t)n;
  C* M = reinterpret_cast<C*>(A);
  for (size_t q = 0; q < dim * dim; ++q) M[q] = cc(0.0);
  for (int i = 0; i < n; ++i)
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) M[(3 * i + r) * dim + 3 * i + c] = inv[9 * (size_t)i + 3 * r + c];
  int nt = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
  for (int i = 0; i < n; ++i) {
    const double* ri = pos + 3 * (size_t)i;
    for (int j = 0; j < n; ++j) {
      const double* rj = pos + 3 * (size_t)j;
      T3 dg, sg;
      bool hd, hs;
      pair_blocks(P, ri, rj, i == j, dg, &hd, sg, &hs);
      if (hd)
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) {
            C& e = M[(3 * i + r) * dim + 3 * j + c];
            e = sub(e, dg[r][c]);
          }
      if (hs) {
        C rr = C{S.refl_re, S.refl_im};
        C m[3] = {neg(rr), neg(rr), rr};
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) {
            C& e = M[(3 * i + r) * dim + 3 * j + c];
            e = sub(e, mul(m[c], sg[r][c]));
          }
      }
    }
  }
  return 0;
}

// matvec_on_the_fly, assembly.rs:209-318
int orc_matvec_onthefly(int n, const double* pos, const double* alpha, const double* x,
                        double k, int use_fcd, double cell, const orc_lattice* lat,
                        const double* kb, const orc_substrate* subs, double* y, int nthreads) {
  std::vector<C> inv;
  if (!prepare_inv_alpha(n, alpha, inv)) return 6;
  Lattice L;
  if (lat) L = to_lat(lat);
  Substrate S;
  if (subs) S = Substrate{subs->z_interface, subs->refl_re, subs->refl_im};
  OtfCtx o{n, pos, inv.data(), make_cfg(k, use_fcd, cell, lat ? &L : nullptr, kb, subs ? &S : nullptr),
           set_threads(nthreads)};
  otf_mv(&o, reinterpret_cast<const C*>(x), reinterpret_cast<C*>(y));
  return 0;
}

// Matvec over a subset of rows [row0, row1): the bounded sample the CPU
// baseline times at full N.
int orc_matvec_onthefly_rows(int n, const double* pos, const double* alpha, const double* x,
                             double k, int use_fcd, double cell, int row0, int row1, double* y,
                             int nthreads) {
  std::vector<C> inv;
  if (!prepare_inv_alpha(n, alpha, inv)) return 6;
  PairCfg P = make_cfg(k, use_fcd, cell, nullptr, nullptr, nullptr);
  const C* xc = reinterpret_cast<const C*>(x);
  C* yc = reinterpret_cast<C*>(y);
  int nt = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
  for (int i = row0; i < row1; ++i) {
    C yi[3] = {cc(0.0), cc(0.0), cc(0.0)};
    const C* ia = &inv[9 * (size_t)i];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) yi[a] = add(yi[a], mul(ia[3 * a + b], xc[3 * i + b]));
    for (int j = 0; j < n; ++j) {
      T3 dg, sg;
      bool hd, hs;
      pair_blocks(P, pos + 3 * (size_t)i, pos + 3 * (size_t)j, i == j, dg, &hd, sg, &hs);
      if (hd)
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) yi[a] = sub(yi[a], mul(dg[a][b], xc[3 * j + b]));
    }
    for (int c = 0; c < 3; ++c) yc[3 * (i - row0) + c] = yi[c];
  }
  return 0;
}

// Rows [row0, row1) of matvec_on_the_fly with every optional term (Ewald
// lattice, Bloch vector, Fresnel image), the loop of otf_mv above restricted
// to a row range: bounded samples of the periodic operator at full size.
int orc_matvec_onthefly_rows_ex(int n, const double* pos, const double* alpha, const double* x,
                                double k, int use_fcd, double cell, const orc_lattice* lat,
                                const double* kb, const orc_substrate* subs, int row0, int row1,
                                double* y, int nthreads) {
  std::vector<C> inv;
  if (!prepare_inv_alpha(n, alpha, inv)) return 6;
  Lattice L;
  if (lat) L = to_lat(lat);
  Substrate S;
  if (subs) S = Substrate{subs->z_interface, subs->refl_re, subs->refl_im};
  OtfCtx o{n, pos, inv.data(), make_cfg(k, use_fcd, cell, lat ? &L : nullptr, kb, subs ? &S : nullptr),
           set_threads(nthreads)};
  const C* xc = reinterpret_cast<const C*>(x);
  C* yc = reinterpret_cast<C*>(y);
#pragma omp parallel for schedule(dynamic, 1) num_threads(o.nthreads)
  for (int i = row0; i < row1; ++i) {
    C yi[3] = {cc(0.0), cc(0.0), cc(0.0)};
    const C* ia = o.inv_alpha + 9 * (size_t)i;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) yi[a] = add(yi[a], mul(ia[3 * a + b], xc[3 * i + b]));
    const double* ri = pos + 3 * (size_t)i;
    for (int j = 0; j < n; ++j) {
      T3 dg, sg;
      bool hd, hs;
      pair_blocks(o.P, ri, pos + 3 * (size_t)j, i == j, dg, &hd, sg, &hs);
      if (hd)
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) yi[a] = sub(yi[a], mul(dg[a][b], xc[3 * j + b]));
      if (hs) {
        C rr = C{o.P.sub->refl_re, o.P.sub->refl_im};
        C m[3] = {neg(rr), neg(rr), rr};
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) yi[a] = sub(yi[a], mul(mul(m[b], sg[a][b]), xc[3 * j + b]));
      }
    }
    for (int c = 0; c < 3; ++c) yc[3 * (i - row0) + c] = yi[c];
  }
  return 0;
}

// solve_gmres over a dense matrix (iterative.rs:33-160 with the matrix matvec
// closure of iterative.rs:214-216 / cpu.rs:64-70).
int orc_gmres_dense(int dim, const double* A, const double* b, double tol, int max_iter,
                    int restart, double* x, int* iters, int* matvecs, double* rel_res,
                    int nthreads) {
  DenseCtx d{dim, reinterpret_cast<const C*>(A), set_threads(nthreads)};
  std::vector<C> rhs(dim), xs;
  load_c(b, rhs.data(), dim);
  GmresOut o = gmres(matvec_cb_dense, &d, rhs, tol, max_iter, restart, xs);
  for (int i = 0; i < dim; ++i) {
    x[2 * i] = xs[i].re;
    x[2 * i + 1] = xs[i].im;
  }
  if (iters) *iters = o.iterations;
  if (matvecs) *matvecs = o.matvecs;
  if (rel_res) *rel_res = o.rel_residual;
  return o.status;
}

// solve_gmres with the on-the-fly matvec closure (cda/mod.rs:378-390).
int orc_gmres_onthefly(int n, const double* pos, const double* alpha, const double* b,
                       double k, int use_fcd, double cell, const orc_lattice* lat,
                       const double* kb, const orc_substrate* subs, double tol, int max_iter,
                       double* x, int* iters, int* matvecs, double* rel_res, int nthreads) {
  std::vector<C> inv;
  if (!prepare_inv_alpha(n, alpha, inv)) return 6;
  Lattice L;
  if (lat) L = to_lat(lat);
  Substrate S;
  if (subs) S = Substrate{subs->z_interface, subs->refl_re, subs->refl_im};
  OtfCtx o{n, pos, inv.data(), make_cfg(k, use_fcd, cell, lat ? &L : nullptr, kb, subs ? &S : nullptr),
           set_threads(nthreads)};
  int dim = 3 * n;
  std::vector<C> rhs(dim), xs;
  load_c(b, rhs.data(), dim);
  GmresOut g = gmres(matvec_cb_otf, &o, rhs, tol, max_iter, 30, xs);
  for (int i = 0; i < dim; ++i) {
    x[2 * i] = xs[i].re;
    x[2 * i + 1] = xs[i].im;
  }
  if (iters) *iters = g.iterations;
  if (matvecs) *matvecs = g.matvecs;
  if (rel_res) *rel_res = g.rel_residual;
  return g.status;
}

// Partial-pivot LU solve (the role of faer's partial_piv_lu in direct.rs:23-60).
int orc_lu_solve(int dim, const double* A, const double* b, double* x) {
  std::vector<C> M((size_t)dim * dim), rhs(dim);
  load_c(A, M.data(), dim * dim);
  load_c(b, rhs.data(), dim);
  std::vector<int> piv(dim);
  for (int c = 0; c < dim; ++c) {
    int p = c;
    double best = norm(M[(size_t)c * dim + c]);
    for (int r = c + 1; r < dim; ++r) {
      double v = norm(M[(size_t)r * dim + c]);
      if (v > best) {
        best = v;
        p = r;
      }
    }
    if (best == 0.0) return 6;
    if (p != c) {
      for (int q = 0; q < dim; ++q) std::swap(M[(size_t)c * dim + q], M[(size_t)p * dim + q]);
      std::swap(rhs[c], rhs[p]);
    }
    C piv_inv = div(cc(1.0), M[(size_t)c * dim + c]);
    for (int r = c + 1; r < dim; ++r) {
      C f = mul(M[(size_t)r * dim + c], piv_inv);
      if (f.re == 0.0 && f.im == 0.0) continue;
      M[(size_t)r * dim + c] = f;
      C* rowr = &M[(size_t)r * dim];
      const C* rowc = &M[(size_t)c * dim];
      for (int q = c + 1; q < dim; ++q) rowr[q] = sub(rowr[q], mul(f, rowc[q]));
      rhs[r] = sub(rhs[r], mul(f, rhs[c]));
    }
  }
  for (int r = dim - 1; r >= 0; --r) {
    C s = rhs[r];
    for (int q = r + 1; q < dim; ++q) s = sub(s, mul(M[(size_t)r * dim + q], rhs[q]));
    rhs[r] = div(s, M[(size_t)r * dim + r]);
  }
  for (int i = 0; i < dim; ++i) {
    x[2 * i] = rhs[i].re;
    x[2 * i + 1] = rhs[i].im;
  }
  return 0;
}

// Cross sections, cda/mod.rs:175-236.  out = {C_ext, C_abs, C_sca(clamped)}.
int orc_cross_sections(int n, const double* pos, const double* alpha, const double* moments,
                       double k, const double* dir, const double* pol, double amplitude,
                       double* out3) {
  std::vector<C> inv;
  if (!prepare_inv_alpha(n, alpha, inv)) return 6;
  double e0_sq = amplitude * amplitude;
  double c_ext = 0.0;
  std::vector<double> einc(6 * (size_t)n);
  orc_incident_field(n, pos, dir, pol, amplitude, k, einc.data());
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      C e = C{einc[2 * (3 * i + c)], einc[2 * (3 * i + c) + 1]};
      C p = C{moments[2 * (3 * i + c)], moments[2 * (3 * i + c) + 1]};
      c_ext += mul(conj(e), p).im;
    }
  c_ext *= k / e0_sq;
  double c_abs = 0.0;
  double k3 = k * k * k;
  for (int i = 0; i < n; ++i) {
    C p[3];
    load_c(moments + 6 * (size_t)i, p, 3);
    C acc = cc(0.0);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) acc = add(acc, mul(mul(p[a], conj(inv[9 * (size_t)i + 3 * a + b])), conj(p[b])));
    double p_sq = norm_sqr(p[0]) + norm_sqr(p[1]) + norm_sqr(p[2]);
    c_abs += acc.im - (2.0 / 3.0) * k3 * p_sq;
  }
  c_abs *= k / e0_sq;
  out3[0] = c_ext;
  out3[1] = c_abs;
  out3[2] = std::max(c_ext - c_abs, 0.0);
  return 0;
}

// clausius_mossotti + radiative_correction, types.rs:243-259 (isotropic alpha)
void orc_rrcm(double volume, double eps_re, double eps_im, double eps_m, double k, int radiative,
              double* out2) {
  C eps = C{eps_re, eps_im};
  C em = cc(eps_m);
  C a_cm = div(muls(sub(eps, em), 3.0 * volume), add(eps, muls(em, 2.0)));
  C a = a_cm;
  if (radiative) {
    C corr = C{0.0, (k * k * k) / (6.0 * PI)};
    a = div(a_cm, sub(cc(1.0), mul(corr, a_cm)));
  }
  out2[0] = a.re;
  out2[1] = a.im;
}

// ellipsoid_polarisability_tensor, types.rs:286-317
void orc_ellipsoid_tensor(double volume, const double* depol, double eps_re, double eps_im,
                          double eps_m, double k, const double* rot, double* out18) {
  C eps = C{eps_re, eps_im};
  C em = cc(eps_m);
  C de = sub(eps, em);
  C al[3];
  for (int i = 0; i < 3; ++i) {
    C denom = add(em, mul(cc(depol[i]), de));
    C a_cm = div(muls(de, volume), denom);
    C corr = C{0.0, (k * k * k) / (6.0 * PI)};
    al[i] = div(a_cm, sub(cc(1.0), mul(corr, a_cm)));
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      C s = cc(0.0);
      for (int q = 0; q < 3; ++q) s = add(s, muls(muls(al[q], rot[i * 3 + q]), rot[j * 3 + q]));
      out18[2 * (3 * i + j)] = s.re;
      out18[2 * (3 * i + j) + 1] = s.im;
    }
}

// Fresnel reflection factors, substrate.rs:160-197
void orc_fresnel(double eps_re, double eps_im, double eps_env, int retarded, double* out2) {
  C es = C{eps_re, eps_im};
  C r;
  if (retarded) {
    C ns = csqrt(es);
    C ne = cc(std::sqrt(eps_env));
    r = div(sub(ns, ne), add(ns, ne));
  } else {
    C ee = cc(eps_env);
    r = div(sub(es, ee), add(es, ee));
  }
  out2[0] = r.re;
  out2[1] = r.im;
}

// Natural cubic spline, spline.rs:32-90.  y2 out has length nk.
void orc_spline_build(int nk, const double* xs, const double* ys, double* y2) {
  std::vector<double> u(nk - 1, 0.0);
  for (int i = 0; i < nk; ++i) y2[i] = 0.0;
  for (int i = 1; i < nk - 1; ++i) {
    double sig = (xs[i] - xs[i - 1]) / (xs[i + 1] - xs[i - 1]);
    double p = sig * y2[i - 1] + 2.0;
    y2[i] = (sig - 1.0) / p;
    u[i] = (ys[i + 1] - ys[i]) / (xs[i + 1] - xs[i]) - (ys[i] - ys[i - 1]) / (xs[i] - xs[i - 1]);
    u[i] = (6.0 * u[i] / (xs[i + 1] - xs[i - 1]) - sig * u[i - 1]) / p;
  }
  for (int k = nk - 3; k >= 0; --k) y2[k + 1] = y2[k + 1] * y2[k + 2] + u[k + 1];
}

double orc_spline_eval(int nk, const double* xs, const double* ys, const double* y2, double x) {
  int lo = 0, hi = nk - 1;
  while (hi - lo > 1) {
    int mid = (lo + hi) / 2;
    if (xs[mid] > x)
      hi = mid;
    else
      lo = mid;
  }
  double h = xs[hi] - xs[lo];
  double a = (xs[hi] - x) / h;
  double b = (x - xs[lo]) / h;
  return a * ys[lo] + b * ys[hi] + ((a * a * a - a) * y2[lo] + (b * b * b - b) * y2[hi]) * h * h / 6.0;
}

// compute_circular_dichroism, fields.rs:236-253
double orc_circular_dichroism(int n, const double* mom_x, const double* mom_y, double k) {
  double delta = 0.0;
  for (int i = 0; i < n; ++i) {
    double py_under_x = mom_x[2 * (3 * i + 1) + 1];
    double px_under_y = mom_y[2 * (3 * i + 0) + 1];
    delta += py_under_x - px_under_y;
  }
  return k * delta;
}

// ---------------------------------------------------------------------------
// Fields from solved moments, fields.rs.
// ---------------------------------------------------------------------------
// field_at_point, fields.rs:18-49: the incident field at the point, then, in
// dipole order, G(r_obs, r_i) . p_i for every dipole with r^2 >= 1e-20.
// moments are 3N complex; out is 3M complex.
void orc_field_at_points(int n, const double* pos, const double* moments, double k,
                         const double* dir, const double* pol, double amplitude, int m,
                         const double* obs, double* out) {
#pragma omp parallel for schedule(static)
  for (int q = 0; q < m; ++q) {
    const double* o = obs + 3 * (size_t)q;
    double einc[6];
    orc_incident_field(1, o, dir, pol, amplitude, k, einc);
    C e[3] = {C{einc[0], einc[1]}, C{einc[2], einc[3]}, C{einc[4], einc[5]}};
    for (int i = 0; i < n; ++i) {
      const double* r = pos + 3 * (size_t)i;
      double dx = o[0] - r[0], dy = o[1] - r[1], dz = o[2] - r[2];
      double r_sq = dx * dx + dy * dy + dz * dz;
      if (r_sq < 1e-20) continue;
      T3 g;
      if (!greens(o, r, k, g)) continue;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          const size_t at = 2 * (3 * (size_t)i + b);
          e[a] = add(e[a], mul(g[a][b], C{moments[at], moments[at + 1]}));
        }
    }
    for (int a = 0; a < 3; ++a) {
      out[2 * (3 * (size_t)q + a)] = e[a].re;
      out[2 * (3 * (size_t)q + a) + 1] = e[a].im;
    }
  }
}

// plane_basis + the grid of compute_near_field_map, fields.rs:52-139.
// positions: 3*nx*ny doubles (iy outer, ix inner); extent[4].
void orc_near_field_plane(const double* centre, const double* normal, double half_width,
                          double half_height, int nx, int ny, double* positions,
                          double* extent) {
  const double nl = std::sqrt(normal[0] * normal[0] + normal[1] * normal[1] +
                              normal[2] * normal[2]);
  const double n[3] = {normal[0] / nl, normal[1] / nl, normal[2] / nl};
  double seed[3] = {0.0, 1.0, 0.0};
  if (std::fabs(n[0]) < 0.9) {
    seed[0] = 1.0;
    seed[1] = 0.0;
  }
  const double dot = seed[0] * n[0] + seed[1] * n[1] + seed[2] * n[2];
  const double ur[3] = {seed[0] - dot * n[0], seed[1] - dot * n[1], seed[2] - dot * n[2]};
  const double ul = std::sqrt(ur[0] * ur[0] + ur[1] * ur[1] + ur[2] * ur[2]);
  const double u[3] = {ur[0] / ul, ur[1] / ul, ur[2] / ul};
  const double v[3] = {n[1] * u[2] - n[2] * u[1], n[2] * u[0] - n[0] * u[2],
                       n[0] * u[1] - n[1] * u[0]};
  const double x_min = -half_width, x_max = half_width;
  const double y_min = -half_height, y_max = half_height;
  const double dx = nx > 1 ? (x_max - x_min) / (double)(nx - 1) : 0.0;
  const double dy = ny > 1 ? (y_max - y_min) / (double)(ny - 1) : 0.0;
  size_t q = 0;
  for (int iy = 0; iy < ny; ++iy)
    for (int ix = 0; ix < nx; ++ix) {
      const double uu = x_min + (double)ix * dx;
      const double vv = y_min + (double)iy * dy;
      for (int c = 0; c < 3; ++c) positions[3 * q + c] = centre[c] + uu * u[c] + vv * v[c];
      ++q;
    }
  extent[0] = centre[0] + x_min * u[0] + y_min * v[0];
  extent[1] = centre[0] + x_max * u[0] + y_max * v[0];
  extent[2] = centre[1] + x_min * u[1] + y_min * v[1];
  extent[3] = centre[1] + x_max * u[1] + y_max * v[1];
}

// compute_far_field, fields.rs:147-221: intensity |(I - rr) . F|^2 with
// F = sum_i p_i exp(-i k r.r_i), theta = pi it/max(nt-1,1), phi = 2 pi ip/np.
void orc_far_field(int n, const double* pos, const double* moments, double k, int n_theta,
                   int n_phi, double* theta, double* phi, double* intensity) {
#pragma omp parallel for schedule(static)
  for (int it = 0; it < n_theta; ++it) {
    const double th = PI * (double)it / (double)std::max(n_theta - 1, 1);
    const double sin_t = std::sin(th), cos_t = std::cos(th);
    for (int ip = 0; ip < n_phi; ++ip) {
      const double ph = 2.0 * PI * (double)ip / (double)n_phi;
      const double sin_p = std::sin(ph), cos_p = std::cos(ph);
      const double rh[3] = {sin_t * cos_p, sin_t * sin_p, cos_t};
      C f[3] = {cc(0.0), cc(0.0), cc(0.0)};
      for (int i = 0; i < n; ++i) {
        const double* r = pos + 3 * (size_t)i;
        const double kdotr = k * (rh[0] * r[0] + rh[1] * r[1] + rh[2] * r[2]);
        const C phase = cexp(C{0.0, -kdotr});
        for (int a = 0; a < 3; ++a) {
          const size_t at = 2 * (3 * (size_t)i + a);
          f[a] = add(f[a], mul(C{moments[at], moments[at + 1]}, phase));
        }
      }
      const C rdotf = add(add(muls(f[0], rh[0]), muls(f[1], rh[1])), muls(f[2], rh[2]));
      double inten = 0.0;
      for (int a = 0; a < 3; ++a) inten += norm_sqr(sub(f[a], muls(rdotf, rh[a])));
      const size_t q = (size_t)it * n_phi + ip;
      theta[q] = th;
      phi[q] = ph;
      intensity[q] = inten;
    }
  }
}

// compute_shg_sources / compute_thg_sources, nonlinear.rs:61-86, :233-258,
// with Chi2Tensor::contract / Chi3Tensor::contract (types.rs:355-365,
// :461-472): p[a] += chi[...] * e[b] * e[c] (* e[d]) in the loop order a, b,
// c (, d).  per_dipole = 0 uses one tensor for every dipole.
void orc_harmonic_sources(int order, int n, const double* e_loc, int per_dipole,
                          const double* chi, double* out) {
  const int nc = order == 2 ? 27 : 81;
  for (int i = 0; i < n; ++i) {
    const double* t = chi + 2 * (size_t)nc * (per_dipole ? i : 0);
    C e[3];
    for (int c = 0; c < 3; ++c) e[c] = C{e_loc[2 * (3 * (size_t)i + c)], e_loc[2 * (3 * (size_t)i + c) + 1]};
    for (int a = 0; a < 3; ++a) {
      C p = cc(0.0);
      for (int b = 0; b < 3; ++b)
        for (int c = 0; c < 3; ++c) {
          if (order == 2) {
            const int q = a * 9 + b * 3 + c;
            p = add(p, mul(mul(C{t[2 * q], t[2 * q + 1]}, e[b]), e[c]));
          } else {
            for (int d = 0; d < 3; ++d) {
              const int q = a * 27 + b * 9 + c * 3 + d;
              p = add(p, mul(mul(mul(C{t[2 * q], t[2 * q + 1]}, e[b]), e[c]), e[d]));
            }
          }
        }
      out[2 * (3 * (size_t)i + a)] = p.re;
      out[2 * (3 * (size_t)i + a) + 1] = p.im;
    }
  }
}

// The reference's WGSL shaders, restated in FP32 (the "reference GPU
// equivalent" of the cached path).  matrix_assemble.wgsl:21-103 and
// matvec.wgsl:19-39; the host diagonal patch is gpu.rs:585-603.
void orc_wgsl_assemble_f32(int n, const double* pos, const double* inv_alpha, double k,
                           float* A /* (3n)^2 complex, interleaved */) {
  int dim = 3 * n;
  float kf = (float)k;
  for (int row = 0; row < dim; ++row)
    for (int col = 0; col < dim; ++col) {
      int i = row / 3, j = col / 3, al = row % 3, be = col % 3;
      float* e = A + 2 * ((size_t)row * dim + col);
      if (i == j) {
        e[0] = (float)inv_alpha[2 * (9 * (size_t)i + 3 * al + be)];
        e[1] = (float)inv_alpha[2 * (9 * (size_t)i + 3 * al + be) + 1];
        continue;
      }
      float rx = (float)pos[3 * i] - (float)pos[3 * j];
      float ry = (float)pos[3 * i + 1] - (float)pos[3 * j + 1];
      float rz = (float)pos[3 * i + 2] - (float)pos[3 * j + 2];
      float r_sq = rx * rx + ry * ry + rz * rz;
      float gre = 0.f, gim = 0.f;
      if (!(r_sq < 1e-20f)) {
        float r = std::sqrt(r_sq);
        float kr = kf * r;
        float kr_sq = kr * kr;
        float er = std::cos(kr), ei = std::sin(kr);
        float scale = kf * kf / (4.0f * 3.14159265358979f * r);
        float pr = scale * er, pi = scale * ei;
        float a_re = 1.0f - 1.0f / kr_sq, a_im = 1.0f / kr;
        float b_re = (3.0f - kr_sq) / kr_sq, b_im = -3.0f / kr;
        float rh[3] = {rx / r, ry / r, rz / r};
        float delta = (al == be) ? 1.0f : 0.0f;
        float rr = rh[al] * rh[be];
        float vr = a_re * delta + b_re * rr, vi = a_im * delta + b_im * rr;
        gre = pr * vr - pi * vi;
        gim = pr * vi + pi * vr;
      }
      e[0] = -gre;
      e[1] = -gim;
    }
}

void orc_wgsl_matvec_f32(int dim, const float* A, const float* x, float* y) {
  for (int row = 0; row < dim; ++row) {
    float sr = 0.f, si = 0.f;
    const float* a = A + 2 * (size_t)row * dim;
    for (int col = 0; col < dim; ++col) {
      float ar = a[2 * col], ai = a[2 * col + 1], br = x[2 * col], bi = x[2 * col + 1];
      sr += ar * br - ai * bi;
      si += ar * bi + ai * br;
    }
    y[2 * row] = sr;
    y[2 * row + 1] = si;
  }
}

// ---------------------------------------------------------------------------
// Adjoint gradient of C_ext (no reference counterpart: its own restatement,
// pinned by central finite differences of orc_cross_sections in the tests).
// p = A^-1 E and mu = A^-1 conj(E) by dense LU; the tensor derivative is
// written in the r-hat form of greens.rs:34-71:
//   G_ab = g (P delta_ab + Q n_a n_b),  g = e^{ikR}/(4 pi R),
//   P = k^2 + ik/R - 1/R^2,  Q = -k^2 - 3ik/R + 3/R^2,  n = d/R,
//   dG_ab/dd_c = n_c [g'(P delta + Q n n) + g (P' delta + Q' n n)]_ab
//              + g Q [(delta_ac - n_a n_c) n_b + n_a (delta_bc - n_b n_c)] / R.
// ---------------------------------------------------------------------------
}  // extern "C"
namespace {
void dgreens(const double d[3], double k, C out[3][3][3]) {
  double R = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  double n[3] = {d[0] / R, d[1] / R, d[2] / R};
  C g = divs(cexp(cc(0.0, k * R)), 4.0 * PI * R);
  C gp = mul(g, cc(-1.0 / R, k));
  C P = cc(k * k - 1.0 / (R * R), k / R);
  C Pp = cc(2.0 / (R * R * R), -k / (R * R));
  C Q = cc(-k * k + 3.0 / (R * R), -3.0 * k / R);
  C Qp = cc(-6.0 / (R * R * R), 3.0 * k / (R * R));
  for (int c = 0; c < 3; ++c)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double dab = (a == b) ? 1.0 : 0.0, dac = (a == c) ? 1.0 : 0.0, dbc = (b == c) ? 1.0 : 0.0;
        C t1 = add(muls(P, dab), muls(Q, n[a] * n[b]));
        C t2 = add(muls(Pp, dab), muls(Qp, n[a] * n[b]));
        C v = muls(add(mul(gp, t1), mul(g, t2)), n[c]);
        double geo = ((dac - n[a] * n[c]) * n[b] + n[a] * (dbc - n[b] * n[c])) / R;
        out[c][a][b] = add(v, muls(mul(g, Q), geo));
      }
}

// d/dd of the tensor the forward operator uses for the pair (FCD average
// for near pairs, greens.rs:94-167 with the same node skip).
void dgreens_pair(const double ro[3], const double rs[3], double k, bool use_fcd, double cell,
                  C out[3][3][3]) {
  double dx = ro[0] - rs[0], dy = ro[1] - rs[1], dz = ro[2] - rs[2];
  double dist = std::sqrt(dx * dx + dy * dy + dz * dz);
  if (!use_fcd || dist > 2.0 * cell) {
    double d[3] = {dx, dy, dz};
    dgreens(d, k, out);
    return;
  }
  const double nodes[3] = {-std::sqrt(3.0 / 5.0), 0.0, std::sqrt(3.0 / 5.0)};
  const double weights[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  double half_d = cell / 2.0;
  for (int c = 0; c < 3; ++c)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) out[c][a][b] = cc(0.0);
  double total_w = 0.0;
  for (int ix = 0; ix < 3; ++ix)
    for (int iy = 0; iy < 3; ++iy)
      for (int iz = 0; iz < 3; ++iz) {
        double d[3] = {ro[0] - (rs[0] + half_d * nodes[ix]), ro[1] - (rs[1] + half_d * nodes[iy]),
                       ro[2] - (rs[2] + half_d * nodes[iz])};
        if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < 1e-20) continue;
        double w = weights[ix] * weights[iy] * weights[iz];
        C t[3][3][3];
        dgreens(d, k, t);
        for (int c = 0; c < 3; ++c)
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) out[c][a][b] = add(out[c][a][b], muls(t[c][a][b], w));
        total_w += w;
      }
  if (total_w > 1e-30)
    for (int c = 0; c < 3; ++c)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) out[c][a][b] = divs(out[c][a][b], total_w);
}
}  // namespace
extern "C" {

int orc_grad_cext(int n, const double* pos, const double* alpha, double k, int use_fcd,
                  double cell, const double* dir, const double* pol6, double amplitude,
                  const double* dinv18, double* c_ext, double* grad_r, double* grad_eps,
                  double* moments, int nthreads) {
  const size_t dim = 3 * (size_t)n;
  std::vector<double> A(2 * dim * dim);
  int st = orc_assemble(n, pos, alpha, k, use_fcd, cell, nullptr, nullptr, nullptr, A.data(),
                        nthreads);
  if (st) return st;
  std::vector<C> E(dim), Ec(dim);
  for (int i = 0; i < n; ++i) {
    const double* r = pos + 3 * (size_t)i;
    double kdotr = k * (dir[0] * r[0] + dir[1] * r[1] + dir[2] * r[2]);
    C ph = cexp(cc(0.0, kdotr));
    for (int a = 0; a < 3; ++a) {
      E[3 * i + a] = mul(cc(amplitude * pol6[2 * a], amplitude * pol6[2 * a + 1]), ph);
      Ec[3 * i + a] = conj(E[3 * i + a]);
    }
  }
  std::vector<C> p(dim), mu(dim);
  st = orc_lu_solve((int)dim, A.data(), reinterpret_cast<const double*>(E.data()),
                    reinterpret_cast<double*>(p.data()));
  if (st) return st;
  st = orc_lu_solve((int)dim, A.data(), reinterpret_cast<const double*>(Ec.data()),
                    reinterpret_cast<double*>(mu.data()));
  if (st) return st;
  const double scale = k / (amplitude * amplitude);
  C f = cc(0.0);
  for (size_t q = 0; q < dim; ++q) f = add(f, mul(conj(E[q]), p[q]));
  *c_ext = scale * f.im;
  if (moments)
    for (size_t q = 0; q < dim; ++q) {
      moments[2 * q] = p[q].re;
      moments[2 * q + 1] = p[q].im;
    }
  int nt = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
  for (int i = 0; i < n; ++i) {
    const double* ri = pos + 3 * (size_t)i;
    C df[3] = {cc(0.0), cc(0.0), cc(0.0)};
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      const double* rj = pos + 3 * (size_t)j;
      C dG[3][3][3];
      dgreens_pair(ri, rj, k, use_fcd != 0, cell, dG);
      for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) {
            df[c] = add(df[c], mul(mul(mu[3 * i + a], dG[c][a][b]), p[3 * j + b]));
            df[c] = add(df[c], mul(mul(mu[3 * j + a], dG[c][a][b]), p[3 * i + b]));
          }
    }
    C q = cc(0.0);
    for (int a = 0; a < 3; ++a) {
      q = add(q, mul(mu[3 * i + a], E[3 * i + a]));
      q = sub(q, mul(conj(E[3 * i + a]), p[3 * i + a]));
    }
    for (int c = 0; c < 3; ++c) {
      C inc = mul(cc(0.0, k * dir[c]), q);
      grad_r[3 * (size_t)i + c] = scale * add(df[c], inc).im;
    }
    if (grad_eps) {
      C fe = cc(0.0);
      if (dinv18)
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) {
            const double* D = dinv18 + 18 * (size_t)i + 2 * (3 * a + b);
            fe = add(fe, mul(mul(mu[3 * i + a], cc(D[0], D[1])), p[3 * i + b]));
          }
      grad_eps[2 * (size_t)i] = -scale * fe.im;
      grad_eps[2 * (size_t)i + 1] = -scale * fe.re;
    }
  }
  return 0;
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"

// ===========================================================================
// Sommerfeld reflected Green's tensor of a planar substrate
// (crates/lumina-core/src/solver/sommerfeld.rs) and the Sommerfeld substrate
// runtime (solver/substrate.rs:109-113, 126-130) in the assembly
// (assembly.rs:157-166) and the on-the-fly matvec (assembly.rs:296-303).
// ===========================================================================
namespace {

// Kronrod 15-point nodes and weights on [-1, 1], sommerfeld.rs:43-76.
const double SOMM_GK_X[15] = {
    -0.991455371120813, -0.949107912342758, -0.864864423359769, -0.741531185599394,
    -0.586087235467691, -0.405845151377397, -0.207784955007898, 0.0,
    0.207784955007898,  0.405845151377397,  0.586087235467691,  0.741531185599394,
    0.864864423359769,  0.949107912342758,  0.991455371120813};
const double SOMM_GK_W[15] = {
    0.022935322010529, 0.063092092629979, 0.104790010322250, 0.140653259715525,
    0.169004726639267, 0.190350578064785, 0.204432940075298, 0.209482141084728,
    0.204432940075298, 0.190350578064785, 0.169004726639267, 0.140653259715525,
    0.104790010322250, 0.063092092629979, 0.022935322010529};

// J0 of sommerfeld.rs:103-121.  The x >= 8 coefficients are the module's
// own (they are not the Numerical Recipes values of the Ewald module); they
// are restated as written because the reflected tensor is built from them.
double somm_j0(double x) {
  double ax = std::fabs(x);
  if (ax < 8.0) {
    double y = x * x;
    double p1 = 57568490574.0 + y * (-13362590354.0 + y * (651619640.7 + y * (-11214424.18 +
                y * (77392.33017 + y * (-184.9052456)))));
    double q1 = 57568490411.0 + y * (1029532985.0 + y * (9494680.718 + y * (59272.64853 +
                y * (267.8532712 + y))));
    return p1 / q1;
  }
  double z = 8.0 / ax, y = z * z, xx = ax - 0.7853981634;
  double p1 = 1.0 + y * (-0.001098628627 + y * (0.000002734511 + y * (-0.00000002073 +
              y * (-0.0000000002073))));
  double q1 = -0.001562499995 + y * (0.000001430488 + y * (-0.000000006905 +
              y * (0.0000000001077 + y * 0.00000000000272)));
  return std::sqrt(2.0 / (PI * ax)) * (p1 * std::cos(xx) - z * q1 * std::sin(xx));
}

// J1 of sommerfeld.rs:126-146 (module's own coefficients, as above).
double somm_j1(double x) {
  double ax = std::fabs(x), val;
  if (ax < 8.0) {
    double y = x * x;
    double p1 = x * (72362614232.0 + y * (-7895059235.0 + y * (242396853.1 + y * (-2972611.439 +
                y * (15704.4882 + y * (-30.1635081))))));
    double q1 = 144725228442.0 + y * (2300535178.0 + y * (18583304.74 + y * (99447.43526 +
                y * (376.9949199 + y))));
    val = p1 / q1;
  } else {
    double z = 8.0 / ax, y = z * z, xx = ax - 2.356194491;
    double p1 = 1.0 + y * (0.000183105 + y * (-0.0000035163965 + y * (0.00000002457572 +
                y * 2.457520e-7)));
    double q1 = 0.040957605 + y * (-0.000004976877 + y * (0.0000000798216 +
                y * (-0.000000000944603 + y * 4.53491e-10)));
    val = std::sqrt(2.0 / (PI * ax)) * (p1 * std::cos(xx) - z * q1 * std::sin(xx));
  }
  return x < 0.0 ? -val : val;
}

// sommerfeld.rs:150-153
double somm_j2(double x) {
  if (std::fabs(x) < 1e-15) return 0.0;
  return (2.0 / x) * somm_j1(x) - somm_j0(x);
}

struct Somm {
  double k_env;
  C k_sub;
  C eps_sub;
  double eps_env;
};

// SommerfeldGreens::new, sommerfeld.rs:236-241
Somm somm_new(double wavelength_nm, C eps_sub, double eps_env) {
  double k0 = 2.0 * PI / wavelength_nm;
  Somm S;
  S.k_env = k0 * std::sqrt(eps_env);
  S.k_sub = csqrt_pos_imag(mul(eps_sub, cc(k0 * k0, 0.0)));
  S.eps_sub = eps_sub;
  S.eps_env = eps_env;
  return S;
}

struct SommI {
  C s_j0, p_j0, zz, xz, j2;
};

// integrand, sommerfeld.rs:376-413
SommI somm_integrand(const Somm& S, double kpar, double rho, double dz) {
  double k = S.k_env, k2 = k * k;
  C kz_env = csqrt_pos_imag(cc(k2 - kpar * kpar, 0.0));
  C kz_sub = csqrt_pos_imag(sub(mul(S.eps_sub, cc(k2 / S.eps_env, 0.0)), cc(kpar * kpar, 0.0)));
  C r_s = div(sub(kz_env, kz_sub), add(kz_env, kz_sub));
  C ee = cc(S.eps_env, 0.0);
  C r_p = div(sub(mul(S.eps_sub, kz_env), mul(ee, kz_sub)),
              add(mul(S.eps_sub, kz_env), mul(ee, kz_sub)));
  C phase = cexp(muls(mul(cc(0.0, 1.0), kz_env), dz));
  double arg = kpar * rho;
  C j0v = cc(somm_j0(arg)), j1v = cc(somm_j1(arg)), j2v = cc(somm_j2(arg));
  C kpar_c = cc(kpar), k2_c = cc(k2);
  C kz_factor = div(kpar_c, kz_env);
  C kz2 = div(mul(kz_env, kz_env), k2_c);
  SommI o;
  o.s_j0 = mul(mul(mul(r_s, j0v), phase), kz_factor);
  o.p_j0 = mul(mul(mul(mul(r_p, kz2), j0v), phase), kz_factor);
  o.zz = mul(mul(mul(mul(r_p, div(mul(kpar_c, kpar_c), k2_c)), j0v), phase), kz_factor);
  o.xz = mul(mul(mul(mul(r_p, div(kpar_c, cc(k))), div(kz_env, cc(k))), j1v), phase);
  o.j2 = mul(mul(mul(mul(r_p, kz2), j2v), phase), kz_factor);
  return o;
}

// integrate_segment, sommerfeld.rs:355-373 (Kronrod weights x half-width)
void somm_segment(const Somm& S, double a, double b, double rho, double dz, SommI& tot) {
  double mid = 0.5 * (a + b), half = 0.5 * (b - a);
  SommI acc{cc(0), cc(0), cc(0), cc(0), cc(0)};
  for (int q = 0; q < 15; ++q) {
    double kpar = mid + half * SOMM_GK_X[q];
    double w = SOMM_GK_W[q] * half;
    SommI c = somm_integrand(S, kpar, rho, dz);
    acc.s_j0 = add(acc.s_j0, muls(c.s_j0, w));
    acc.p_j0 = add(acc.p_j0, muls(c.p_j0, w));
    acc.zz = add(acc.zz, muls(c.zz, w));
    acc.xz = add(acc.xz, muls(c.xz, w));
    acc.j2 = add(acc.j2, muls(c.j2, w));
  }
  tot.s_j0 = add(tot.s_j0, acc.s_j0);
  tot.p_j0 = add(tot.p_j0, acc.p_j0);
  tot.zz = add(tot.zz, acc.zz);
  tot.xz = add(tot.xz, acc.xz);
  tot.j2 = add(tot.j2, acc.j2);
}

// integrate, sommerfeld.rs:316-352: [0, k_env], [k_env, Re k_sub] when
// Re k_sub > 1.001 k_env, and [max(k_env, Re k_sub), k_max].
SommI somm_integrate(const Somm& S, double rho, double dz) {
  double k_env = S.k_env;
  double k_sub_real = std::max(S.k_sub.re, k_env);
  bool has_seg2 = S.k_sub.re > k_env * 1.001;
  double k_max = dz > 1e-6 ? std::max(10.0 * 2.302585092994045684 / dz, k_env * 5.0) : k_env * 20.0;
  SommI tot{cc(0), cc(0), cc(0), cc(0), cc(0)};
  somm_segment(S, 0.0, k_env, rho, dz, tot);
  if (has_seg2) somm_segment(S, k_env, k_sub_real, rho, dz, tot);
  double lo = has_seg2 ? k_sub_real : k_env;
  if (k_max > lo * 1.001) somm_segment(S, lo, k_max, rho, dz, tot);
  return tot;
}

// evaluate, sommerfeld.rs:254-300
void somm_tensor(const Somm& S, const double* ri, const double* rj, double z0, T3 g) {
  double dz = (ri[2] - z0) + (rj[2] - z0);
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) g[a][b] = cc(0.0);
  if (dz <= 0.0) return;
  double dx = ri[0] - rj[0], dy = ri[1] - rj[1];
  double rho = std::sqrt(dx * dx + dy * dy);
  double phi = std::atan2(dy, dx);
  double cp = std::cos(phi), sp = std::sin(phi);
  double c2 = 2.0 * cp * cp - 1.0, s2 = 2.0 * sp * cp;
  SommI I = somm_integrate(S, rho, dz);
  C pre = cc(0.0, 1.0 / (8.0 * PI));
  C sp_sum = add(I.s_j0, I.p_j0);
  g[0][0] = mul(pre, sub(sp_sum, muls(I.j2, c2)));
  g[1][1] = mul(pre, add(sp_sum, muls(I.j2, c2)));
  g[2][2] = mul(pre, neg(I.zz));
  g[0][1] = g[1][0] = mul(pre, muls(neg(I.j2), s2));
  g[0][2] = g[2][0] = mul(pre, muls(I.xz, cp));
  g[1][2] = g[2][1] = mul(pre, muls(I.xz, sp));
}

}  // namespace

extern "C" {

/* SommerfeldGreens parameters (SubstrateRuntime::from_spec, substrate.rs:126-130). */
typedef struct {
  double z_interface;
  double wavelength_nm;
  double eps_sub_re, eps_sub_im;
  double eps_env;
} orc_sommerfeld;

static Somm somm_of(const orc_sommerfeld* s) {
  return somm_new(s->wavelength_nm, cc(s->eps_sub_re, s->eps_sub_im), s->eps_env);
}

double orc_somm_bessel(int which, double x) {
  return which == 0 ? somm_j0(x) : which == 1 ? somm_j1(x) : somm_j2(x);
}

// G_refl for npairs (ri, rj) pairs, 9 interleaved complex values each.
void orc_sommerfeld_tensor(const orc_sommerfeld* s, int npairs, const double* ri,
                           const double* rj, double* out, int nthreads) {
  Somm S = somm_of(s);
  int nt = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16) num_threads(nt)
  for (int p = 0; p < npairs; ++p) {
    T3 g;
    somm_tensor(S, ri + 3 * (size_t)p, rj + 3 * (size_t)p, s->z_interface, g);
    store_t3(g, out + 18 * (size_t)p);
  }
}

// assemble_interaction_matrix with SubstrateRuntime::Sommerfeld
// (assembly.rs:157-166): the free-space / lattice matrix minus G_refl for
// every (i, j), i == j included.
int orc_assemble_sommerfeld(int n, const double* pos, const double* alpha, double k, int use_fcd,
                            double cell, const orc_lattice* lat, const double* kb,
                            const orc_sommerfeld* s, double* A, int nthreads) {
  int st = orc_assemble(n, pos, alpha, k, use_fcd, cell, lat, kb, nullptr, A, nthreads);
  if (st) return st;
  Somm S = somm_of(s);
  const size_t dim = 3 * (size_t)n;
  C* M = reinterpret_cast<C*>(A);
  int nt = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      T3 g;
      somm_tensor(S, pos + 3 * (size_t)i, pos + 3 * (size_t)j, s->z_interface, g);
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
          C& e = M[(3 * i + r) * dim + 3 * j + c];
          e = sub(e, g[r][c]);
        }
    }
  return 0;
}

// matvec_on_the_fly with SubstrateRuntime::Sommerfeld (assembly.rs:296-303).
int orc_matvec_sommerfeld(int n, const double* pos, const double* alpha, const double* x,
                          double k, int use_fcd, double cell, const orc_lattice* lat,
                          const double* kb, const orc_sommerfeld* s, double* y, int nthreads) {
  int st = orc_matvec_onthefly(n, pos, alpha, x, k, use_fcd, cell, lat, kb, nullptr, y, nthreads);
  if (st) return st;
  Somm S = somm_of(s);
  const C* xv = reinterpret_cast<const C*>(x);
  C* yv = reinterpret_cast<C*>(y);
  int nt = set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
  for (int i = 0; i < n; ++i) {
    C yi[3] = {yv[3 * i], yv[3 * i + 1], yv[3 * i + 2]};
    for (int j = 0; j < n; ++j) {
      T3 g;
      somm_tensor(S, pos + 3 * (size_t)i, pos + 3 * (size_t)j, s->z_interface, g);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) yi[a] = sub(yi[a], mul(g[a][b], xv[3 * j + b]));
    }
    for (int a = 0; a < 3; ++a) yv[3 * i + a] = yi[a];
  }
  return 0;
}

}  // extern "C"
