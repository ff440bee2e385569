// sommerfeld.cu -- the substrate's reflected Green's tensor by the Sommerfeld
// integral (crates/lumina-core/src/solver/sommerfeld.rs) on the device.
//
// G_refl(r_i, r_j) depends on the pair only through the lateral distance
// rho, the height sum dz = (z_i - z0) + (z_j - z0) and the azimuth phi.  The
// expensive part -- five k_par integrals by 15-node Kronrod quadrature on up
// to three segments (45 integrand evaluations, each with two complex square
// roots, two complex divisions, a complex exponential and J0/J1, FP64) -- is
// a function of (rho, dz) alone.  It is evaluated once per wavelength into a
// table of records of four pre-multiplied complex values
//
//   A = pre (I_s_J0 + I_p_J0),  B = pre I_J2,  Z = pre I_zz,  X = pre I_xz,
//   pre = i / (8 pi)                                    (sommerfeld.rs:281)
//
// keyed, on a cubic dipole lattice of pitch d with integer coordinates
// (a, b, c), by (s = da^2 + db^2, t = c_i + c_j): rho = d sqrt(s),
// dz = 2 (z_lo - z0) + d t.  That table has (max s + 1)(2 max c + 1) records
// -- a few MB for particles of tens of thousands of dipoles, so it stays in
// L2 -- and carries an FP32 copy for FP32 applications.  Off the lattice the
// table holds one record per unordered pair (n(n+1)/2 records in HBM).
// Every use rebuilds the 3x3 block from the ordered pair's own (dx, dy):
//
//   G_xx = A - B cos2phi   G_yy = A + B cos2phi   G_zz = -Z
//   G_xy = -B sin2phi      G_xz = X cos phi       G_yz = X sin phi
//
// (sommerfeld.rs:284-289; cos phi = dx / rho, sin phi = dy / rho, phi = 0 at
// rho = 0 as atan2(0, 0) gives).  The operator application y -= G_refl x
// (assembly.rs:296-303, every j including i) gathers the records, one warp
// per row; the dense assembly (assembly.rs:157-166) subtracts the same blocks
// from the stored matrix.  The stand-alone evaluator follows evaluate()
// (sommerfeld.rs:254-300) literally for parity checks.
#include "sommerfeld.cuh"

#include <cmath>

namespace lum {

constexpr int kSommBlock = 128;
constexpr int kSommRecordC = 4;   // complex values per table record

// The 3x3 block from a table record and the ordered pair's (dx, dy).
template <typename R, typename R2>
__device__ __forceinline__ void somm_block(const R2* __restrict__ rec, R dx, R dy, R2 g[9]) {
  const R r2 = dx * dx + dy * dy;
  R cp = R(1), sp = R(0);
  if (r2 > R(0)) {
    const R inv = rsqrt(r2);
    cp = dx * inv;
    sp = dy * inv;
  }
  const R c2 = R(2) * cp * cp - R(1), s2 = R(2) * sp * cp;
  const R2 A = rec[0], B = rec[1], Z = rec[2], X = rec[3];
  g[0].x = A.x - B.x * c2;  g[0].y = A.y - B.y * c2;
  g[4].x = A.x + B.x * c2;  g[4].y = A.y + B.y * c2;
  g[8].x = -Z.x;            g[8].y = -Z.y;
  g[1].x = -B.x * s2;       g[1].y = -B.y * s2;
  g[2].x = X.x * cp;        g[2].y = X.y * cp;
  g[5].x = X.x * sp;        g[5].y = X.y * sp;
  g[3] = g[1];
  g[6] = g[2];
  g[7] = g[5];
}

// Packed upper-triangle index of the unordered pair (i <= j).
__device__ __forceinline__ size_t somm_index(int i, int j, int n) {
  return (size_t)i * n - ((size_t)i * (i - 1)) / 2 + (size_t)(j - i);
}

// Record of the ordered pair (i, j): lattice key (da^2 + db^2, c_i + c_j)
// or the packed unordered-pair index.
struct SommIdx {
  int keyed;
  int n;
  int T;
  const int4* __restrict__ lidx;
  __device__ __forceinline__ size_t rec(int i, int j, int4 li, int4 lj) const {
    if (keyed) {
      const int da = li.x - lj.x, db = li.y - lj.y;
      return (size_t)(da * da + db * db) * T + (size_t)(li.z + lj.z);
    }
    return j >= i ? somm_index(i, j, n) : somm_index(j, i, n);
  }
};

__device__ __forceinline__ void somm_store(const SommInt& I, double2* __restrict__ rec,
                                           float2* __restrict__ rec32) {
  double2 v[4];
  somm_record(I, v);
  for (int c = 0; c < kSommRecordC; ++c) {
    rec[c] = v[c];
    if (rec32) rec32[c] = make_float2((float)v[c].x, (float)v[c].y);
  }
}

// Per unordered pair: one thread per (i = blockIdx.y, j >= i).
__global__ void __launch_bounds__(kSommBlock)
somm_table_pairs(int n, const double4* __restrict__ pos, SommDev S, double2* __restrict__ tab) {
  const int i = blockIdx.y;
  const int j = blockIdx.x * kSommBlock + threadIdx.x;
  if (j < i || j >= n) return;
  const double4 ri = pos[i], rj = pos[j];
  const double dz = (ri.z - S.z0) + (rj.z - S.z0);
  double2* rec = tab + kSommRecordC * somm_index(i, j, n);
  if (dz <= 0.0) {
    for (int c = 0; c < kSommRecordC; ++c) rec[c] = make_double2(0.0, 0.0);
    return;
  }
  const double dx = ri.x - rj.x, dy = ri.y - rj.y;
  somm_store(somm_integrals(S, sqrt(dx * dx + dy * dy), dz), rec, nullptr);
}

// Per lattice key: record q = s T + t, rho = d sqrt(s), dz = (zlo - z0) +
// (zlo - z0) + d t.
__global__ void __launch_bounds__(kSommBlock)
somm_table_keys(long long records, int T, double d, double zlo, SommDev S,
                double2* __restrict__ tab, float2* __restrict__ tab32) {
  const long long q = (long long)blockIdx.x * kSommBlock + threadIdx.x;
  if (q >= records) return;
  const long long s = q / T;
  const int t = (int)(q % T);
  const double dz = (zlo - S.z0) + (zlo - S.z0) + d * t;
  double2* rec = tab + kSommRecordC * (size_t)q;
  float2* rec32 = tab32 + kSommRecordC * (size_t)q;
  if (dz <= 0.0) {
    for (int c = 0; c < kSommRecordC; ++c) {
      rec[c] = make_double2(0.0, 0.0);
      rec32[c] = make_float2(0.f, 0.f);
    }
    return;
  }
  somm_store(somm_integrals(S, d * sqrt((double)s), dz), rec, rec32);
}

template <typename R> struct SommT;
template <> struct SommT<double> {
  typedef double2 R2;
  static __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
};
template <> struct SommT<float> {
  typedef float2 R2;
  static __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
};

// y_i -= sum_j G_refl(i, j) x_j: one warp per row, lanes over j, R
// arithmetic with the record type of R, fixed-order shuffle reduction
// (deterministic), the row's update in FP64.
constexpr int kSommRows = 8;
template <typename R>
__global__ void __launch_bounds__(32 * kSommRows)
somm_apply_rows(int n, const double4* __restrict__ pos, SommIdx K,
                const typename SommT<R>::R2* __restrict__ tab, const double2* __restrict__ x,
                double2* __restrict__ y, const int* __restrict__ skip) {
  typedef typename SommT<R>::R2 R2;
  if (skip && *skip) return;
  const int i = blockIdx.x * kSommRows + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const double4 ri = pos[i];
  const int4 li = K.keyed ? K.lidx[i] : make_int4(0, 0, 0, 0);
  R2 acc[3];
  for (int a = 0; a < 3; ++a) acc[a] = SommT<R>::mk(R(0), R(0));
  for (int j = lane; j < n; j += 32) {
    const int4 lj = K.keyed ? K.lidx[j] : make_int4(0, 0, 0, 0);
    const double4 rj = pos[j];
    R2 g[9];
    somm_block<R, R2>(tab + kSommRecordC * K.rec(i, j, li, lj), (R)(ri.x - rj.x),
                      (R)(ri.y - rj.y), g);
    const double2 xd0 = x[3 * (size_t)j], xd1 = x[3 * (size_t)j + 1],
                  xd2 = x[3 * (size_t)j + 2];
    const R2 x0 = SommT<R>::mk((R)xd0.x, (R)xd0.y), x1 = SommT<R>::mk((R)xd1.x, (R)xd1.y),
             x2 = SommT<R>::mk((R)xd2.x, (R)xd2.y);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const R2 g0 = g[3 * a], g1 = g[3 * a + 1], g2 = g[3 * a + 2];
      acc[a].x += g0.x * x0.x - g0.y * x0.y + g1.x * x1.x - g1.y * x1.y + g2.x * x2.x -
                  g2.y * x2.y;
      acc[a].y += g0.x * x0.y + g0.y * x0.x + g1.x * x1.y + g1.y * x1.x + g2.x * x2.y +
                  g2.y * x2.x;
    }
  }
  double ax[3], ay[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    ax[a] = (double)acc[a].x;
    ay[a] = (double)acc[a].y;
    for (int o = 16; o > 0; o >>= 1) {
      ax[a] += __shfl_xor_sync(0xffffffffu, ax[a], o);
      ay[a] += __shfl_xor_sync(0xffffffffu, ay[a], o);
    }
  }
  if (lane == 0)
    for (int a = 0; a < 3; ++a) {
      double2& e = y[3 * (size_t)i + a];
      e = make_double2(e.x - ax[a], e.y - ay[a]);
    }
}

// Lattice-keyed application: the block's eight rows share column tiles of
// lattice coordinates and x staged in shared memory; cos phi and sin phi come
// from the integer offsets (da, db) / sqrt(s), so a pair reads only its
// record (from L2) beyond the tile.
constexpr int kSommTile = 128;
template <typename R>
__global__ void __launch_bounds__(32 * kSommRows)
somm_apply_keyed(int n, const int4* __restrict__ lidx, int T,
                 const typename SommT<R>::R2* __restrict__ tab, const double2* __restrict__ x,
                 double2* __restrict__ y, const int* __restrict__ skip) {
  typedef typename SommT<R>::R2 R2;
  __shared__ int4 s_l[kSommTile];
  __shared__ R2 s_x[3][kSommTile];
  if (skip && *skip) return;  // the flag is the same for the whole block
  const int i = blockIdx.x * kSommRows + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const bool active = i < n;
  const int4 li = active ? lidx[i] : make_int4(0, 0, 0, 0);
  R2 acc[3];
  for (int a = 0; a < 3; ++a) acc[a] = SommT<R>::mk(R(0), R(0));
  for (int c0 = 0; c0 < n; c0 += kSommTile) {
    __syncthreads();
    if (threadIdx.x < kSommTile) {
      const int t = threadIdx.x, j = c0 + t;
      if (j < n) {
        s_l[t] = lidx[j];
        for (int c = 0; c < 3; ++c) {
          const double2 v = x[3 * (size_t)j + c];
          s_x[c][t] = SommT<R>::mk((R)v.x, (R)v.y);
        }
      }
    }
    __syncthreads();
    const int cmax = min(kSommTile, n - c0);
    if (active) {
#pragma unroll 2
      for (int t = lane; t < cmax; t += 32) {
        const int4 lj = s_l[t];
        const int da = li.x - lj.x, db = li.y - lj.y;
        const int sq = da * da + db * db;
        const R2* rec = tab + kSommRecordC * ((size_t)sq * T + (size_t)(li.z + lj.z));
        R2 A, B, Z, X;
        if constexpr (sizeof(R) == 4) {
          const float4 r0 = __ldg(reinterpret_cast<const float4*>(rec));
          const float4 r1 = __ldg(reinterpret_cast<const float4*>(rec) + 1);
          A = SommT<R>::mk(r0.x, r0.y);
          B = SommT<R>::mk(r0.z, r0.w);
          Z = SommT<R>::mk(r1.x, r1.y);
          X = SommT<R>::mk(r1.z, r1.w);
        } else {
          A = __ldg(rec);
          B = __ldg(rec + 1);
          Z = __ldg(rec + 2);
          X = __ldg(rec + 3);
        }
        R cp = R(1), sp = R(0);
        if (sq > 0) {
          const R inv = rsqrt((R)sq);
          cp = (R)da * inv;
          sp = (R)db * inv;
        }
        const R c2 = R(2) * cp * cp - R(1), s2 = R(2) * sp * cp;
        const R2 gxx = SommT<R>::mk(A.x - B.x * c2, A.y - B.y * c2);
        const R2 gyy = SommT<R>::mk(A.x + B.x * c2, A.y + B.y * c2);
        const R2 gxy = SommT<R>::mk(-B.x * s2, -B.y * s2);
        const R2 gxz = SommT<R>::mk(X.x * cp, X.y * cp);
        const R2 gyz = SommT<R>::mk(X.x * sp, X.y * sp);
        const R2 x0 = s_x[0][t], x1 = s_x[1][t], x2 = s_x[2][t];
        acc[0].x += gxx.x * x0.x - gxx.y * x0.y + gxy.x * x1.x - gxy.y * x1.y + gxz.x * x2.x -
                    gxz.y * x2.y;
        acc[0].y += gxx.x * x0.y + gxx.y * x0.x + gxy.x * x1.y + gxy.y * x1.x + gxz.x * x2.y +
                    gxz.y * x2.x;
        acc[1].x += gxy.x * x0.x - gxy.y * x0.y + gyy.x * x1.x - gyy.y * x1.y + gyz.x * x2.x -
                    gyz.y * x2.y;
        acc[1].y += gxy.x * x0.y + gxy.y * x0.x + gyy.x * x1.y + gyy.y * x1.x + gyz.x * x2.y +
                    gyz.y * x2.x;
        acc[2].x += gxz.x * x0.x - gxz.y * x0.y + gyz.x * x1.x - gyz.y * x1.y - Z.x * x2.x +
                    Z.y * x2.y;
        acc[2].y += gxz.x * x0.y + gxz.y * x0.x + gyz.x * x1.y + gyz.y * x1.x - Z.x * x2.y -
                    Z.y * x2.x;
      }
    }
  }
  if (!active) return;
  double ax[3], ay[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    ax[a] = (double)acc[a].x;
    ay[a] = (double)acc[a].y;
    for (int o = 16; o > 0; o >>= 1) {
      ax[a] += __shfl_xor_sync(0xffffffffu, ax[a], o);
      ay[a] += __shfl_xor_sync(0xffffffffu, ay[a], o);
    }
  }
  if (lane == 0)
    for (int a = 0; a < 3; ++a) {
      double2& e = y[3 * (size_t)i + a];
      e = make_double2(e.x - ax[a], e.y - ay[a]);
    }
}

template <typename T2> __device__ __forceinline__ T2 somm_mk(double re, double im);
template <> __device__ __forceinline__ float2 somm_mk<float2>(double re, double im) {
  return make_float2((float)re, (float)im);
}
template <> __device__ __forceinline__ double2 somm_mk<double2>(double re, double im) {
  return make_double2(re, im);
}

// A[i][j] -= G_refl(i, j) for every ordered pair (assembly.rs:157-166), from
// the FP64 records.
template <typename T2>
__global__ void __launch_bounds__(kSommBlock)
somm_assemble_pairs(int n, const double4* __restrict__ pos, SommIdx K,
                    const double2* __restrict__ tab, size_t ld, T2* __restrict__ A) {
  const int i = blockIdx.y;
  const int j = blockIdx.x * kSommBlock + threadIdx.x;
  if (j >= n) return;
  const double4 ri = pos[i], rj = pos[j];
  const int4 li = K.keyed ? K.lidx[i] : make_int4(0, 0, 0, 0);
  const int4 lj = K.keyed ? K.lidx[j] : make_int4(0, 0, 0, 0);
  double2 g[9];
  somm_block<double, double2>(tab + kSommRecordC * K.rec(i, j, li, lj), ri.x - rj.x,
                              ri.y - rj.y, g);
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      T2& e = A[(3 * (size_t)i + a) * ld + 3 * (size_t)j + b];
      e = somm_mk<T2>((double)e.x - g[3 * a + b].x, (double)e.y - g[3 * a + b].y);
    }
}

// evaluate() literally (sommerfeld.rs:254-300), one thread per pair.
__global__ void somm_evaluate(int npairs, SommDev S, const double* __restrict__ ri,
                              const double* __restrict__ rj, double2* __restrict__ out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npairs) return;
  const double* a = ri + 3 * (size_t)q;
  const double* b = rj + 3 * (size_t)q;
  double2* g = out + 9 * (size_t)q;
  const double dz = (a[2] - S.z0) + (b[2] - S.z0);
  if (dz <= 0.0) {
    for (int e = 0; e < 9; ++e) g[e] = make_double2(0.0, 0.0);
    return;
  }
  const double dx = a[0] - b[0], dy = a[1] - b[1];
  const double rho = sqrt(dx * dx + dy * dy);
  const double phi = atan2(dy, dx);
  double sp, cp;
  sincos(phi, &sp, &cp);
  const double c2 = 2.0 * cp * cp - 1.0, s2 = 2.0 * sp * cp;
  const SommInt I = somm_integrals(S, rho, dz);
  const double2 pre = make_double2(0.0, 1.0 / (8.0 * kPi));
  const double2 spv = cadd(I.s_j0, I.p_j0);
  g[0] = cmul(pre, make_double2(spv.x - I.j2.x * c2, spv.y - I.j2.y * c2));
  g[4] = cmul(pre, make_double2(spv.x + I.j2.x * c2, spv.y + I.j2.y * c2));
  g[8] = cmul(pre, make_double2(-I.zz.x, -I.zz.y));
  g[1] = g[3] = cmul(pre, make_double2(-I.j2.x * s2, -I.j2.y * s2));
  g[2] = g[6] = cmul(pre, cscale(I.xz, cp));
  g[5] = g[7] = cmul(pre, cscale(I.xz, sp));
}

// SommerfeldGreens::new (sommerfeld.rs:236-241).
lum_status somm_params(const lum_sommerfeld* s, SommDev* out) {
  if (!s) {
    set_error("Sommerfeld parameters must not be NULL");
    return LUM_ERR_INVALID;
  }
  if (!(s->wavelength_nm > 0.0) || !std::isfinite(s->wavelength_nm) || !(s->eps_env > 0.0) ||
      !std::isfinite(s->eps_env) || !std::isfinite(s->eps_sub_re) ||
      !std::isfinite(s->eps_sub_im) || !std::isfinite(s->z_interface)) {
    set_error("invalid Sommerfeld substrate (wavelength %g, eps_env %g)", s->wavelength_nm,
              s->eps_env);
    return LUM_ERR_INVALID;
  }
  const double k0 = 2.0 * kPi / s->wavelength_nm;
  SommDev S;
  S.z0 = s->z_interface;
  S.k_env = k0 * std::sqrt(s->eps_env);
  S.eps_env = s->eps_env;
  S.eps_sub = make_double2(s->eps_sub_re, s->eps_sub_im);
  // k_sub = csqrt_pos_im(eps_sub k0^2): principal root of a complex number
  // (the same algebraic branch as somm_csqrt, on the host)
  const double zr = s->eps_sub_re * k0 * k0, zi = s->eps_sub_im * k0 * k0;
  double sr, si;
  if (zi == 0.0) {
    if (!std::signbit(zr)) {
      sr = std::sqrt(zr);
      si = zi;
    } else {
      sr = 0.0;
      si = std::signbit(zi) ? -std::sqrt(-zr) : std::sqrt(-zr);
    }
  } else {
    const double r = std::hypot(zr, zi);
    const double t = std::sqrt(0.5 * (r + std::fabs(zr)));
    if (zr >= 0.0) {
      sr = t;
      si = zi / (2.0 * t);
    } else {
      sr = std::fabs(zi) / (2.0 * t);
      si = std::copysign(t, zi);
    }
  }
  if (si < 0.0) {
    sr = -sr;
    si = -si;
  }
  S.k_sub = make_double2(sr, si);
  *out = S;
  return LUM_OK;
}

// Integer lattice coordinates of every dipole when the positions lie on a
// cubic lattice to 1e-12 of its pitch (then the lattice key reproduces rho
// and dz of every pair to rounding); false otherwise.
static bool somm_lattice(const std::vector<double>& p4, int n, double cell, double* d_out,
                         double lo[3], std::vector<int>& idx, int mx[3]) {
  for (int c = 0; c < 3; ++c) lo[c] = 1e300;
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) lo[c] = std::min(lo[c], p4[4 * (size_t)i + c]);
  std::vector<double> cand;
  if (cell > 0.0) cand.push_back(cell);
  double step = 1e300;
  for (int i = 1; i < n && i < 4096; ++i)
    for (int c = 0; c < 3; ++c) {
      const double dl = std::fabs(p4[4 * (size_t)i + c] - p4[c]);
      if (dl > 1e-9) step = std::min(step, dl);
    }
  if (step < 1e300) cand.push_back(step);
  if (n == 1) cand.push_back(1.0);
  for (double d : cand) {
    idx.assign((size_t)4 * n, 0);
    mx[0] = mx[1] = mx[2] = 0;
    bool ok = true;
    for (int i = 0; i < n && ok; ++i)
      for (int c = 0; c < 3; ++c) {
        const double u = (p4[4 * (size_t)i + c] - lo[c]) / d;
        const double r = std::nearbyint(u);
        if (std::fabs(u - r) > 1e-12 * std::max(1.0, r) || r > 1e5) {
          ok = false;
          break;
        }
        idx[4 * (size_t)i + c] = (int)r;
        mx[c] = std::max(mx[c], (int)r);
      }
    if (ok) {
      *d_out = d;
      return true;
    }
  }
  return false;
}

lum_status OtfOperator::somm_build(const lum_sommerfeld* s, cudaStream_t st) {
  SommDev S;
  LUM_TRY(somm_params(s, &S));
  if (n > 65535) {
    set_error("Sommerfeld substrate: at most 65535 dipoles (got %d)", n);
    return LUM_ERR_INVALID;
  }
  const long long pairs = (long long)n * (n + 1) / 2;
  double d = 0.0, lo[3];
  std::vector<int> idx;
  int mx[3];
  int keyed = 0;
  long long records = pairs;
  int T = 0;
  if (somm_lattice(host_pos, n, cell, &d, lo, idx, mx)) {
    T = 2 * mx[2] + 1;
    const long long keys = ((long long)mx[0] * mx[0] + (long long)mx[1] * mx[1] + 1) * T;
    if (keys < pairs && keys <= (16ll << 20)) {
      keyed = 1;
      records = keys;
    }
  }
  const size_t bytes = (size_t)records * kSommRecordC * sizeof(double2);
  if (somm_tab.bytes != bytes) {
    somm_tab.release();
    size_t free_b = 0, total_b = 0;
    LUM_TRY_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (bytes + bytes / 2 + ((size_t)1 << 30) > free_b) {
      set_error("Sommerfeld table of %zu bytes does not fit (%zu bytes free)", bytes, free_b);
      return LUM_ERR_OOM;
    }
    LUM_TRY(somm_tab.alloc(bytes));
  }
  if (keyed) {
    LUM_TRY(somm_tab32.alloc(bytes / 2));
    LUM_TRY(somm_idx.alloc(sizeof(int) * idx.size()));
    LUM_TRY_CUDA(cudaMemcpyAsync(somm_idx.p, idx.data(), somm_idx.bytes, cudaMemcpyHostToDevice,
                                 st));
    somm_table_keys<<<(unsigned)((records + kSommBlock - 1) / kSommBlock), kSommBlock, 0, st>>>(
        records, T, d, lo[2], S, somm_tab.as<double2>(), somm_tab32.as<float2>());
  } else {
    somm_tab32.release();
    somm_idx.release();
    dim3 grid((n + kSommBlock - 1) / kSommBlock, n);
    somm_table_pairs<<<grid, kSommBlock, 0, st>>>(n, pos64.as<double4>(), S,
                                                  somm_tab.as<double2>());
  }
  LUM_CHECK_LAUNCH();
  // the idx upload above reads a host vector that dies with this frame
  LUM_TRY_CUDA(cudaStreamSynchronize(st));
  somm = S;
  somm_keyed = keyed;
  somm_T = T;
  somm_d = d;
  somm_zlo = keyed ? lo[2] : 0.0;
  somm_records = records;
  has_somm = 1;
  somm_stale = 0;
  return LUM_OK;
}

static SommIdx somm_indexer(const OtfOperator& g) {
  SommIdx K;
  K.keyed = g.somm_keyed;
  K.n = g.n;
  K.T = g.somm_T;
  K.lidx = g.somm_keyed ? g.somm_idx.as<int4>() : nullptr;
  return K;
}

lum_status OtfOperator::somm_apply(int precision, const double2* x, double2* y, cudaStream_t st,
                                   const int* skip) const {
  if (!has_somm) return LUM_OK;
  if (somm_stale) {
    set_error("the Sommerfeld table belongs to another wavelength: call "
              "lum_session_set_sommerfeld after lum_session_set_wavelength");
    return LUM_ERR_INVALID;
  }
  const SommIdx K = somm_indexer(*this);
  const unsigned blocks = (unsigned)((n + kSommRows - 1) / kSommRows);
  if (somm_keyed && precision == LUM_FP32)
    somm_apply_keyed<float><<<blocks, 32 * kSommRows, 0, st>>>(
        n, somm_idx.as<int4>(), somm_T, somm_tab32.as<float2>(), x, y, skip);
  else if (somm_keyed)
    somm_apply_keyed<double><<<blocks, 32 * kSommRows, 0, st>>>(
        n, somm_idx.as<int4>(), somm_T, somm_tab.as<double2>(), x, y, skip);
  else
    somm_apply_rows<double><<<blocks, 32 * kSommRows, 0, st>>>(
        n, pos64.as<double4>(), K, somm_tab.as<double2>(), x, y, skip);
  LUM_CHECK_LAUNCH();
  return LUM_OK;
}

lum_status somm_assemble(const OtfOperator& g, int precision, void* A, size_t ld,
                         cudaStream_t st) {
  if (!g.has_somm) return LUM_OK;
  const SommIdx K = somm_indexer(g);
  dim3 grid((g.n + kSommBlock - 1) / kSommBlock, g.n);
  if (precision == LUM_FP32)
    somm_assemble_pairs<float2><<<grid, kSommBlock, 0, st>>>(
        g.n, g.pos64.as<double4>(), K, g.somm_tab.as<double2>(), ld, (float2*)A);
  else
    somm_assemble_pairs<double2><<<grid, kSommBlock, 0, st>>>(
        g.n, g.pos64.as<double4>(), K, g.somm_tab.as<double2>(), ld, (double2*)A);
  LUM_CHECK_LAUNCH();
  return LUM_OK;
}

}  // namespace lum

using namespace lum;

int lum_sommerfeld_tensor(lum_ctx* ctx, const lum_sommerfeld* s, int npairs, const double* ri,
                          const double* rj, double* g) {
  if (!ctx) {
    set_error("null context");
    return LUM_ERR_INVALID;
  }
  SommDev S;
  LUM_TRY(somm_params(s, &S));
  if (npairs < 0 || (npairs > 0 && (!ri || !rj || !g))) {
    set_error("invalid pair arrays (npairs = %d)", npairs);
    return LUM_ERR_INVALID;
  }
  if (npairs == 0) return LUM_OK;
  for (size_t q = 0; q < 3 * (size_t)npairs; ++q)
    if (!std::isfinite(ri[q]) || !std::isfinite(rj[q])) {
      set_error("non-finite point in pair %zu", q / 3);
      return LUM_ERR_INVALID;
    }
  LUM_TRY_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = nullptr;
  LUM_TRY_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } guard{st};
  DevBuf da, db, dg;
  const size_t pb = sizeof(double) * 3 * (size_t)npairs;
  LUM_TRY(da.alloc(pb));
  LUM_TRY(db.alloc(pb));
  LUM_TRY(dg.alloc(sizeof(double2) * 9 * (size_t)npairs));
  LUM_TRY_CUDA(cudaMemcpyAsync(da.p, ri, pb, cudaMemcpyHostToDevice, st));
  LUM_TRY_CUDA(cudaMemcpyAsync(db.p, rj, pb, cudaMemcpyHostToDevice, st));
  somm_evaluate<<<(npairs + 127) / 128, 128, 0, st>>>(npairs, S, da.as<double>(),
                                                      db.as<double>(), dg.as<double2>());
  LUM_CHECK_LAUNCH();
  LUM_TRY_CUDA(cudaMemcpyAsync(g, dg.p, dg.bytes, cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));
  return LUM_OK;
}
