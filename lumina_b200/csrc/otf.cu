// otf.cu -- matrix-free (on-the-fly) CDA operator on sm_100a.
//
// y_i = alpha_i^-1 x_i - sum_{j != i} G(r_i - r_j) x_j      (assembly.rs:209-318)
//
// Decomposition: one thread owns one observer dipole i (3 complex outputs);
// a CTA owns 128*R observers and one chunk of source dipoles; sources are
// staged through shared memory in tiles of 128 and every thread of the CTA
// reads the same source (broadcast).  The j-range is split over grid.y so
// that the grid fills every SM; each split writes its own partial sums and
// the epilogue reduces them in a fixed order (deterministic result), adds the
// alpha^-1 block in FP64 and applies the FCD near-pair correction.
//
// The point-dipole interaction is written as
//   G x = A x + B' d (d . x),  d = r_i - r_j, u = 1/(kR),
//   A  = (k^3/4pi) u e^{ikR} (1 - u^2 + i u),
//   B' = (k^3/4pi) u e^{ikR} (3u^2 - 1 - 3iu) / R^2,
// which is the tensor of greens.rs:34-71 (a = 1 + (ikR-1)/(kR)^2,
// b = (3 - 3ikR - (kR)^2)/(kR)^2) applied without forming it:
// 1 rsqrt + 1 sincos + ~60 FMA-pipe instructions per pair.
//
// FCD (greens.rs:94-167): pairs with dist <= 2*cell use the 27-node
// Gauss-Legendre cell average instead of the point tensor.  The dense
// kernels evaluate the point tensor for every pair; the near pairs are
// listed once per geometry (FP64, the reference's own comparison) and the
// correction G_fcd - G_point is tabulated per wavelength in FP64 (and an
// FP32 copy), then applied by the epilogue.
#include "lumina_internal.cuh"
#include "device_physics.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>

namespace lum {

constexpr int kOtfBlock = 128;
}  // namespace lum
#include "pairs_f32x2.cuh"
#include "pairs_f32_sym.cuh"
#include "pairs_f64_sym.cuh"
namespace lum {

// ---------------------------------------------------------------------------
// FP64 dense pair kernel (same decomposition; sources as double4 + 3 double2)
// ---------------------------------------------------------------------------
// One CTA's work: rows [row0, row0 + 128) against sources [j_begin, j_end);
// out is this split's slice of the partial buffer (shared with the batched
// kernel).  NR == 2 also contracts the same tensors with x2 into out2.
template <bool IMAGE, int NR>
__device__ __forceinline__ void pairs_f64_cta(int n, const double4* __restrict__ pos,
                                              const double2* __restrict__ x,
                                              const double2* __restrict__ x2, double2 m0,
                                              double2 m1, double2 m2, double z_mirror, double k,
                                              double inv_k, double s0, int row0, int j_begin,
                                              int j_end, double2* __restrict__ out,
                                              double2* __restrict__ out2,
                                              const double2* __restrict__ sTab) {
  __shared__ double4 sP[kOtfBlock];
  __shared__ double2 sX[3 * NR * kOtfBlock];
  const int tid = threadIdx.x;
  const int i = row0 + tid;
  const double4 ri = pos[min(i, n - 1)];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  double acc2[6] = {0, 0, 0, 0, 0, 0};
  for (int jt = j_begin; jt < j_end; jt += kOtfBlock) {
    const int cnt = min(kOtfBlock, j_end - jt);
    __syncthreads();
    if (tid < cnt) {
      const int j = jt + tid;
      double4 p = pos[j];
      double2 a = x[3 * j], b = x[3 * j + 1], c = x[3 * j + 2];
      if (IMAGE) {  // image source (x, y, 2 z0 - z) with x' = m x (assembly.rs:278-293)
        p.z = z_mirror - p.z;
        a = make_double2(m0.x * a.x - m0.y * a.y, m0.x * a.y + m0.y * a.x);
        b = make_double2(m1.x * b.x - m1.y * b.y, m1.x * b.y + m1.y * b.x);
        c = make_double2(m2.x * c.x - m2.y * c.y, m2.x * c.y + m2.y * c.x);
      }
      sP[tid] = p;
      sX[3 * tid] = a;
      sX[3 * tid + 1] = b;
      sX[3 * tid + 2] = c;
      if constexpr (NR == 2) {
        double2 d = x2[3 * j], e = x2[3 * j + 1], f = x2[3 * j + 2];
        if (IMAGE) {
          d = make_double2(m0.x * d.x - m0.y * d.y, m0.x * d.y + m0.y * d.x);
          e = make_double2(m1.x * e.x - m1.y * e.y, m1.x * e.y + m1.y * e.x);
          f = make_double2(m2.x * f.x - m2.y * f.y, m2.x * f.y + m2.y * f.x);
        }
        sX[3 * kOtfBlock + 3 * tid] = d;
        sX[3 * kOtfBlock + 3 * tid + 1] = e;
        sX[3 * kOtfBlock + 3 * tid + 2] = f;
      }
    }
    __syncthreads();
    for (int jj = 0; jj < cnt; ++jj) {
      const double4 pj = sP[jj];
      const double2 xa = sX[3 * jj], xb = sX[3 * jj + 1], xc = sX[3 * jj + 2];
      double dx = ri.x - pj.x, dy = ri.y - pj.y, dz = ri.z - pj.z;
      double r2 = dx * dx + dy * dy + dz * dz;
      bool skip = IMAGE ? (r2 < 1e-20) : (jt + jj == i);
      if (skip) r2 = 1.0;
      double ir = rsqrt(r2);
      double Rr = r2 * ir;
      double u = ir * inv_k;
      double u2 = u * u;
      double sn, cs;
      sincos_tab(k * Rr, sTab, &sn, &cs);
      double su = skip ? 0.0 : s0 * u;
      double pr = su * cs, pi = su * sn;
      double ar = 1.0 - u2;
      double Ar = pr * ar - pi * u, Ai = pr * u + pi * ar;
      double br = 3.0 * u2 - 1.0, bi = -3.0 * u;
      double ir2 = ir * ir;
      double Br = (pr * br - pi * bi) * ir2, Bi = (pr * bi + pi * br) * ir2;
      double dxr = dx * xa.x + dy * xb.x + dz * xc.x;
      double dxi = dx * xa.y + dy * xb.y + dz * xc.y;
      double tr = Br * dxr - Bi * dxi, ti = Br * dxi + Bi * dxr;
      acc[0] += Ar * xa.x - Ai * xa.y + tr * dx;
      acc[1] += Ar * xa.y + Ai * xa.x + ti * dx;
      acc[2] += Ar * xb.x - Ai * xb.y + tr * dy;
      acc[3] += Ar * xb.y + Ai * xb.x + ti * dy;
      acc[4] += Ar * xc.x - Ai * xc.y + tr * dz;
      acc[5] += Ar * xc.y + Ai * xc.x + ti * dz;
      if constexpr (NR == 2) {
        const double2 ya = sX[3 * kOtfBlock + 3 * jj], yb = sX[3 * kOtfBlock + 3 * jj + 1],
                      yc = sX[3 * kOtfBlock + 3 * jj + 2];
        double dyr = dx * ya.x + dy * yb.x + dz * yc.x;
        double dyi = dx * ya.y + dy * yb.y + dz * yc.y;
        double ur = Br * dyr - Bi * dyi, ui = Br * dyi + Bi * dyr;
        acc2[0] += Ar * ya.x - Ai * ya.y + ur * dx;
        acc2[1] += Ar * ya.y + Ai * ya.x + ui * dx;
        acc2[2] += Ar * yb.x - Ai * yb.y + ur * dy;
        acc2[3] += Ar * yb.y + Ai * yb.x + ui * dy;
        acc2[4] += Ar * yc.x - Ai * yc.y + ur * dz;
        acc2[5] += Ar * yc.y + Ai * yc.x + ui * dz;
      }
    }
  }
  if (i < n) {
    out[3 * i + 0] = make_double2(acc[0], acc[1]);
    out[3 * i + 1] = make_double2(acc[2], acc[3]);
    out[3 * i + 2] = make_double2(acc[4], acc[5]);
    if constexpr (NR == 2) {
      out2[3 * i + 0] = make_double2(acc2[0], acc2[1]);
      out2[3 * i + 1] = make_double2(acc2[2], acc2[3]);
      out2[3 * i + 2] = make_double2(acc2[4], acc2[5]);
    }
  }
}

template <bool IMAGE>
__global__ void __launch_bounds__(kOtfBlock)
otf_pairs_f64(int n, const double4* __restrict__ pos, const double2* __restrict__ x,
              double2 m0, double2 m1, double2 m2, double z_mirror, double k, double inv_k,
              double s0, int chunk, double2* __restrict__ partial,
              const int* __restrict__ skip) {
  if (skip && *skip) return;
  __shared__ double2 sTab[kScTab];
  sincos_table_stage(sTab);  // the first source tile's barrier precedes its use
  const int j_begin = blockIdx.y * chunk;
  pairs_f64_cta<IMAGE, 1>(n, pos, x, nullptr, m0, m1, m2, z_mirror, k, inv_k, s0,
                          blockIdx.x * kOtfBlock, j_begin, min(n, j_begin + chunk),
                          partial + (size_t)blockIdx.y * (3 * (size_t)n), nullptr, sTab);
}

// Two right-hand sides (see otf_pairs_f32_x2).
template <bool IMAGE>
__global__ void __launch_bounds__(kOtfBlock)
otf_pairs_f64_x2(int n, const double4* __restrict__ pos, const double2* __restrict__ x,
                 const double2* __restrict__ x2, double2 m0, double2 m1, double2 m2,
                 double z_mirror, double k, double inv_k, double s0, int chunk,
                 double2* __restrict__ partial, double2* __restrict__ partial2,
                 const int* __restrict__ skip, const int* __restrict__ skip2) {
  const bool live = !(skip && *skip), live2 = !(skip2 && *skip2);
  if (!live && !live2) return;
  __shared__ double2 sTab[kScTab];
  sincos_table_stage(sTab);  // the first source tile's barrier precedes its use
  const int j_begin = blockIdx.y * chunk, j_end = min(n, j_begin + chunk);
  const size_t off = (size_t)blockIdx.y * (3 * (size_t)n);
  if (live && live2)
    pairs_f64_cta<IMAGE, 2>(n, pos, x, x2, m0, m1, m2, z_mirror, k, inv_k, s0,
                            blockIdx.x * kOtfBlock, j_begin, j_end, partial + off,
                            partial2 + off, sTab);
  else
    pairs_f64_cta<IMAGE, 1>(n, pos, live ? x : x2, nullptr, m0, m1, m2, z_mirror, k, inv_k, s0,
                            blockIdx.x * kOtfBlock, j_begin, j_end,
                            (live ? partial : partial2) + off, nullptr, sTab);
}

// ---------------------------------------------------------------------------
// Epilogue: y = alpha^-1 x - sum(partials) - sum_near C_ij x_j
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }
__device__ __forceinline__ double2 to_d2(double2 v) { return v; }

// kEpiTPR consecutive threads share one dipole: they split the pair partials
// and the near-pair slots between them (more loads in flight per row), then
// combine by shuffle in a fixed order; the first thread adds alpha^-1 x.
constexpr int kEpiTPR = 4;

template <typename TP, typename TC>
__global__ void __launch_bounds__(256)
otf_epilogue(int n, const double2* __restrict__ x, const double2* __restrict__ inv_alpha,
             const TP* __restrict__ partial, int nparts, int ell_w,
             const int* __restrict__ near_j, const TC* __restrict__ fcd,
             double2* __restrict__ y, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = min(gid / kEpiTPR, n - 1);
  const int sub = gid % kEpiTPR;
  const bool live = gid / kEpiTPR < n;
  double gr[3] = {0, 0, 0}, gi[3] = {0, 0, 0};
  const size_t stride = 3 * (size_t)n;
  for (int s = sub; s < nparts; s += kEpiTPR) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double2 p = to_d2(partial[s * stride + 3 * i + a]);
      gr[a] += p.x;
      gi[a] += p.y;
    }
  }
  for (int w = sub; w < ell_w; w += kEpiTPR) {
    const int j = near_j[(size_t)w * n + i];
    if (j < 0) break;  // lists are packed: the rest of this row is padding
    double2 xj[3] = {x[3 * j], x[3 * j + 1], x[3 * j + 2]};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        double2 c = to_d2(fcd[((size_t)w * 9 + 3 * a + b) * n + i]);
        gr[a] += c.x * xj[b].x - c.y * xj[b].y;
        gi[a] += c.x * xj[b].y + c.y * xj[b].x;
      }
  }
#pragma unroll
  for (int o = 1; o < kEpiTPR; o <<= 1)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      gr[a] += __shfl_xor_sync(0xffffffffu, gr[a], o);
      gi[a] += __shfl_xor_sync(0xffffffffu, gi[a], o);
    }
  if (!live || sub != 0) return;
  const double2 xi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      double2 m = inv_alpha[(size_t)(3 * a + b) * n + i];
      sr += m.x * xi[b].x - m.y * xi[b].y;
      si += m.x * xi[b].y + m.y * xi[b].x;
    }
    y[3 * i + a] = make_double2(sr - gr[a], si - gi[a]);
  }
}

// The epilogue of a two-vector application: the same sums for x and x2, with
// each FCD correction tensor read once for both vectors.  A vector whose
// skip flag is set is left untouched.
template <typename TP, typename TC>
__global__ void __launch_bounds__(256)
otf_epilogue2(int n, const double2* __restrict__ x, const double2* __restrict__ x2,
              const double2* __restrict__ inv_alpha, const TP* __restrict__ partial,
              const TP* __restrict__ partial2, int nparts, int ell_w,
              const int* __restrict__ near_j, const TC* __restrict__ fcd,
              double2* __restrict__ y, double2* __restrict__ y2, const int* __restrict__ skip,
              const int* __restrict__ skip2) {
  const bool l1 = !(skip && *skip), l2 = !(skip2 && *skip2);  // grid-uniform
  if (!l1 && !l2) return;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = min(gid / kEpiTPR, n - 1);
  const int sub = gid % kEpiTPR;
  const bool live = gid / kEpiTPR < n;
  double gr[3] = {0, 0, 0}, gi[3] = {0, 0, 0}, hr[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  const size_t stride = 3 * (size_t)n;
  for (int s = sub; s < nparts; s += kEpiTPR) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (l1) {
        const double2 p = to_d2(partial[s * stride + 3 * i + a]);
        gr[a] += p.x;
        gi[a] += p.y;
      }
      if (l2) {
        const double2 p = to_d2(partial2[s * stride + 3 * i + a]);
        hr[a] += p.x;
        hi[a] += p.y;
      }
    }
  }
  for (int w = sub; w < ell_w; w += kEpiTPR) {
    const int j = near_j[(size_t)w * n + i];
    if (j < 0) break;  // lists are packed: the rest of this row is padding
    double2 xj[3], zj[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      xj[b] = l1 ? x[3 * j + b] : make_double2(0.0, 0.0);
      zj[b] = l2 ? x2[3 * j + b] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const double2 c = to_d2(fcd[((size_t)w * 9 + 3 * a + b) * n + i]);
        gr[a] += c.x * xj[b].x - c.y * xj[b].y;
        gi[a] += c.x * xj[b].y + c.y * xj[b].x;
        hr[a] += c.x * zj[b].x - c.y * zj[b].y;
        hi[a] += c.x * zj[b].y + c.y * zj[b].x;
      }
  }
#pragma unroll
  for (int o = 1; o < kEpiTPR; o <<= 1)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      gr[a] += __shfl_xor_sync(0xffffffffu, gr[a], o);
      gi[a] += __shfl_xor_sync(0xffffffffu, gi[a], o);
      hr[a] += __shfl_xor_sync(0xffffffffu, hr[a], o);
      hi[a] += __shfl_xor_sync(0xffffffffu, hi[a], o);
    }
  if (!live || sub != 0) return;
  double2 m[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) m[e] = inv_alpha[(size_t)e * n + i];
  if (l1) {
    const double2 xi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double sr = 0.0, si = 0.0;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        sr += m[3 * a + b].x * xi[b].x - m[3 * a + b].y * xi[b].y;
        si += m[3 * a + b].x * xi[b].y + m[3 * a + b].y * xi[b].x;
      }
      y[3 * i + a] = make_double2(sr - gr[a], si - gi[a]);
    }
  }
  if (l2) {
    const double2 zi[3] = {x2[3 * i], x2[3 * i + 1], x2[3 * i + 2]};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double sr = 0.0, si = 0.0;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        sr += m[3 * a + b].x * zi[b].x - m[3 * a + b].y * zi[b].y;
        si += m[3 * a + b].x * zi[b].y + m[3 * a + b].y * zi[b].x;
      }
      y2[3 * i + a] = make_double2(sr - hr[a], si - hi[a]);
    }
  }
}

// ---------------------------------------------------------------------------
// Near-pair list (FCD).  The near test is the reference's, in FP64 without
// contraction: dist = sqrt((dx*dx + dy*dy) + dz*dz); near = !(dist > 2*cell)
// (greens.rs:100-108).  Coincident dipoles (r == 0, i != j) are flagged.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double ref_dist(double4 a, double4 b) {
  double dx = __dsub_rn(a.x, b.x), dy = __dsub_rn(a.y, b.y), dz = __dsub_rn(a.z, b.z);
  double s = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  return __dsqrt_rn(s);
}

template <bool FILL>
__global__ void __launch_bounds__(256)
near_scan(int n, const double4* __restrict__ pos, double two_cell, int use_fcd,
          int* __restrict__ count, int ell_w, int* __restrict__ near_j,
          int* __restrict__ coincident) {
  __shared__ double4 sP[256];
  const int tid = threadIdx.x;
  const int i = blockIdx.x * 256 + tid;
  const double4 ri = pos[min(i, n - 1)];
  int c = 0;
  for (int jt = 0; jt < n; jt += 256) {
    const int cnt = min(256, n - jt);
    __syncthreads();
    if (tid < cnt) sP[tid] = pos[jt + tid];
    __syncthreads();
    if (i < n) {
      for (int jj = 0; jj < cnt; ++jj) {
        const int j = jt + jj;
        if (j == i) continue;
        double d = ref_dist(ri, sP[jj]);
        if (d == 0.0) atomicOr(coincident, 1);
        if (use_fcd && !(d > two_cell)) {
          if (FILL && c < ell_w) near_j[(size_t)c * n + i] = j;
          ++c;
        }
      }
    }
  }
  if (i < n && !FILL) count[i] = c;
}

__device__ void fcd_correction(const double4* __restrict__ pos, int i, int j, double k,
                               double cell, double2 C[9]);

// FCD correction per near pair: C = G_fcd(r_i, r_j) - G_point(r_i, r_j).
// The 27-node rule, the r^2 < 1e-20 node skip and the weight
// normalisation follow greens.rs:110-164.
__global__ void __launch_bounds__(128)
fcd_table(int n, int ell_w, const double4* __restrict__ pos, const int* __restrict__ near_j,
          double k, double cell, double2* __restrict__ fcd64, float2* __restrict__ fcd32) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * ell_w) return;
  const int w = idx / n, i = idx % n;
  const int j = near_j[(size_t)w * n + i];
  double2 C[9];
  fcd_correction(pos, i, j, k, cell, C);
  for (int e = 0; e < 9; ++e) {
    fcd64[((size_t)w * 9 + e) * n + i] = C[e];
    fcd32[((size_t)w * 9 + e) * n + i] = make_float2((float)C[e].x, (float)C[e].y);
  }
}

// C = G_fcd(r_i, r_j) - G_point(r_i, r_j); zero when j < 0 (ELL padding).
__device__ void fcd_correction(const double4* __restrict__ pos, int i, int j, double k,
                               double cell, double2 C[9]) {
  for (int e = 0; e < 9; ++e) C[e] = make_double2(0.0, 0.0);
  if (j >= 0) {
    const double4 ro = pos[i], rs = pos[j];
    const double nodes[3] = {-sqrt(3.0 / 5.0), 0.0, sqrt(3.0 / 5.0)};
    const double wts[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    const double half_d = cell / 2.0;
    double tw = 0.0;
    double2 g[9];
    for (int ix = 0; ix < 3; ++ix)
      for (int iy = 0; iy < 3; ++iy)
        for (int iz = 0; iz < 3; ++iz) {
          double px = rs.x + half_d * nodes[ix];
          double py = rs.y + half_d * nodes[iy];
          double pz = rs.z + half_d * nodes[iz];
          double ddx = ro.x - px, ddy = ro.y - py, ddz = ro.z - pz;
          if (ddx * ddx + ddy * ddy + ddz * ddz < 1e-20) continue;
          double wt = wts[ix] * wts[iy] * wts[iz];
          greens_point_d(ddx, ddy, ddz, k, g);
          for (int e = 0; e < 9; ++e) {
            C[e].x += wt * g[e].x;
            C[e].y += wt * g[e].y;
          }
          tw += wt;
        }
    if (tw > 1e-30) {
      double inv = 1.0 / tw;
      for (int e = 0; e < 9; ++e) {
        C[e].x *= inv;
        C[e].y *= inv;
      }
    }
    greens_point_d(ro.x - rs.x, ro.y - rs.y, ro.z - rs.z, k, g);
    for (int e = 0; e < 9; ++e) {
      C[e].x -= g[e].x;
      C[e].y -= g[e].y;
    }
  }
}

// Lattice pair kernel: thread per observer, j over a chunk; FP64 throughout.
// Accumulates +G_ewald x_j (+ m G_ewald(img) x_j for a substrate) into the
// partial slice of its split.
__global__ void __launch_bounds__(128)
otf_pairs_ewald(int n, const double4* __restrict__ pos, const double2* __restrict__ x,
                LatticeDev L, const double4* __restrict__ lreal,
                const double4* __restrict__ lrecip, double kb0, double kb1, double kb2,
                double k, int has_sub, SubstrateDev sub, int chunk,
                double2* __restrict__ partial, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double kb[3] = {kb0, kb1, kb2};
  const double4 ri = pos[i];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const int j_begin = blockIdx.y * chunk;
  const int j_end = min(n, j_begin + chunk);
  const double2 rr = make_double2(sub.refl_re, sub.refl_im);
  const double2 mm[3] = {make_double2(-rr.x, -rr.y), make_double2(-rr.x, -rr.y), rr};
  double2 g[9];
  for (int j = j_begin; j < j_end; ++j) {
    const double4 rj = pos[j];
    const double2 xj[3] = {x[3 * j], x[3 * j + 1], x[3 * j + 2]};
    ewald_tensor(L, lreal, lrecip, ri.x - rj.x, ri.y - rj.y, ri.z - rj.z, kb, k, g);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double2 t = cmul(g[3 * a + b], xj[b]);
        acc[2 * a] += t.x;
        acc[2 * a + 1] += t.y;
      }
    if (has_sub) {
      double dx = ri.x - rj.x, dy = ri.y - rj.y, dz = ri.z - (2.0 * sub.z_interface - rj.z);
      if (dx * dx + dy * dy + dz * dz >= 1e-20) {
        ewald_tensor(L, lreal, lrecip, dx, dy, dz, kb, k, g);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) {
            double2 t = cmul(cmul(mm[b], g[3 * a + b]), xj[b]);
            acc[2 * a] += t.x;
            acc[2 * a + 1] += t.y;
          }
      }
    }
  }
  double2* out = partial + (size_t)blockIdx.y * (3 * (size_t)n);
  out[3 * i + 0] = make_double2(acc[0], acc[1]);
  out[3 * i + 1] = make_double2(acc[2], acc[3]);
  out[3 * i + 2] = make_double2(acc[4], acc[5]);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

int device_sms() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

// Split the source range so that row-blocks x splits fills whole waves.
int choose_nsplit(int rowblocks, int ntiles, int ctas_per_sm, int sms) {
  const int slots = std::max(1, ctas_per_sm * sms);
  int best = 1;
  double best_eff = -1.0;
  const int smax = std::max(1, std::min(64, ntiles));
  for (int s = 1; s <= smax; ++s) {
    long total = (long)rowblocks * s;
    long waves = (total + slots - 1) / slots;
    double eff = (double)total / (double)(waves * slots);
    // prefer at least one full wave, then the best wave efficiency, then fewer splits
    double score = eff + (total >= slots ? 1.0 : 0.0);
    if (score > best_eff + 1e-9) {
      best_eff = score;
      best = s;
    }
    if (total >= 2L * slots && eff > 0.97) break;
  }
  return best;
}

// FP32 pair-kernel variants the tuner chooses from: rows per thread (2*RP)
// and the register cap implied by MINB resident CTAs per SM.
struct F32Args {
  int n;
  const float4 *oh, *ol, *sh, *sl;
  const double2* x;
  float2 m0, m1, m2;
  float k, ik, s0;
  int chunk;
  float2* part;
  const int* skip;
};

template <int RP, int MINB>
struct F32Variant {
  template <bool IMAGE>
  static void launch(int fast, int lofree, dim3 grid, cudaStream_t st, const F32Args& a) {
#define LUM_F32_LAUNCH(F, L)                                                                  \
  otf_pairs_f32<F, IMAGE, L, RP, MINB><<<grid, kOtfBlock, 0, st>>>(                           \
      a.n, a.oh, a.ol, a.sh, a.sl, a.x, a.m0, a.m1, a.m2, a.k, a.ik, a.s0, a.chunk, a.part, \
      a.skip)
    if (fast && lofree)
      LUM_F32_LAUNCH(true, true);
    else if (fast)
      LUM_F32_LAUNCH(true, false);
    else if (lofree)
      LUM_F32_LAUNCH(false, true);
    else
      LUM_F32_LAUNCH(false, false);
#undef LUM_F32_LAUNCH
  }
  static int occupancy(int fast, int lofree) {
    int occ = 1;
    if (fast && lofree)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, otf_pairs_f32<true, false, true, RP, MINB>, kOtfBlock, 0);
    else if (fast)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, otf_pairs_f32<true, false, false, RP, MINB>, kOtfBlock, 0);
    else if (lofree)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, otf_pairs_f32<false, false, true, RP, MINB>, kOtfBlock, 0);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, otf_pairs_f32<false, false, false, RP, MINB>, kOtfBlock, 0);
    return std::max(1, occ);
  }
};

struct F32VariantEntry {
  const char* name;
  int rows;  // observer rows per thread
  void (*direct)(int, int, dim3, cudaStream_t, const F32Args&);
  void (*image)(int, int, dim3, cudaStream_t, const F32Args&);
  int (*occupancy)(int, int);
};

const F32VariantEntry kF32Variants[] = {
    {"rows2_minb1", 2, F32Variant<1, 1>::launch<false>, F32Variant<1, 1>::launch<true>, F32Variant<1, 1>::occupancy},
    {"rows2_minb6", 2, F32Variant<1, 6>::launch<false>, F32Variant<1, 6>::launch<true>, F32Variant<1, 6>::occupancy},
    {"rows2_minb8", 2, F32Variant<1, 8>::launch<false>, F32Variant<1, 8>::launch<true>, F32Variant<1, 8>::occupancy},
    {"rows4_minb3", 4, F32Variant<2, 3>::launch<false>, F32Variant<2, 3>::launch<true>, F32Variant<2, 3>::occupancy},
    {"rows4_minb4", 4, F32Variant<2, 4>::launch<false>, F32Variant<2, 4>::launch<true>, F32Variant<2, 4>::occupancy},
};
constexpr int kNumF32Variants = sizeof(kF32Variants) / sizeof(kF32Variants[0]);

// Two-vector variants (otf_pairs_f32_x2): the second accumulator set needs
// more registers, so the register caps are looser.
struct F32X2Args {
  int n;
  const float4 *oh, *ol, *sh, *sl;
  const double2 *x, *x2;
  float2 m0, m1, m2;
  float k, ik, s0;
  int chunk;
  float2 *part, *part2;
  const int *skip, *skip2;
};

template <int RP, int MINB>
struct F32X2Variant {
  template <bool IMAGE>
  static void launch(int fast, int lofree, dim3 grid, cudaStream_t st, const F32X2Args& a) {
#define LUM_F32X2_LAUNCH(F, L)                                                                \
  otf_pairs_f32_x2<F, IMAGE, L, RP, MINB><<<grid, kOtfBlock, 0, st>>>(                         \
      a.n, a.oh, a.ol, a.sh, a.sl, a.x, a.x2, a.m0, a.m1, a.m2, a.k, a.ik, a.s0, a.chunk,      \
      a.part, a.part2, a.skip, a.skip2)
    if (fast && lofree)
      LUM_F32X2_LAUNCH(true, true);
    else if (fast)
      LUM_F32X2_LAUNCH(true, false);
    else if (lofree)
      LUM_F32X2_LAUNCH(false, true);
    else
      LUM_F32X2_LAUNCH(false, false);
#undef LUM_F32X2_LAUNCH
  }
  static int occupancy(int fast, int lofree) {
    int occ = 1;
    if (fast && lofree)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, otf_pairs_f32_x2<true, false, true, RP, MINB>, kOtfBlock, 0);
    else if (fast)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, otf_pairs_f32_x2<true, false, false, RP, MINB>, kOtfBlock, 0);
    else if (lofree)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, otf_pairs_f32_x2<false, false, true, RP, MINB>, kOtfBlock, 0);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, otf_pairs_f32_x2<false, false, false, RP, MINB>, kOtfBlock, 0);
    return std::max(1, occ);
  }
};

struct F32X2VariantEntry {
  const char* name;
  int rows;
  void (*direct)(int, int, dim3, cudaStream_t, const F32X2Args&);
  void (*image)(int, int, dim3, cudaStream_t, const F32X2Args&);
  int (*occupancy)(int, int);
};

const F32X2VariantEntry kF32X2Variants[] = {
    {"x2_rows2_minb4", 2, F32X2Variant<1, 4>::launch<false>, F32X2Variant<1, 4>::launch<true>, F32X2Variant<1, 4>::occupancy},
    {"x2_rows4_minb2", 4, F32X2Variant<2, 2>::launch<false>, F32X2Variant<2, 2>::launch<true>, F32X2Variant<2, 2>::occupancy},
    {"x2_rows4_minb3", 4, F32X2Variant<2, 3>::launch<false>, F32X2Variant<2, 3>::launch<true>, F32X2Variant<2, 3>::occupancy},
};
constexpr int kNumF32X2Variants = sizeof(kF32X2Variants) / sizeof(kF32X2Variants[0]);

}  // namespace

const char* f32_variant_name(int v) {
  return (v >= 0 && v < kNumF32Variants) ? kF32Variants[v].name : "none";
}

const char* f32x2_variant_name(int v) {
  return (v >= 0 && v < kNumF32X2Variants) ? kF32X2Variants[v].name : "none";
}

lum_status OtfOperator::build_geometry(const double* pos_host, int n_, cudaStream_t st) {
  n = n_;
  if (n <= 0) {
    set_error("No dipoles provided");
    return LUM_ERR_INVALID;
  }
  std::vector<double> p4((size_t)4 * n);
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c) {
      double v = pos_host[3 * (size_t)i + c];
      if (!std::isfinite(v)) {
        set_error("non-finite dipole position at index %d", i);
        return LUM_ERR_INVALID;
      }
      p4[4 * (size_t)i + c] = v;
      lo[c] = std::min(lo[c], v);
      hi[c] = std::max(hi[c], v);
    }
    p4[4 * (size_t)i + 3] = 0.0;
  }
  for (int c = 0; c < 3; ++c) center[c] = 0.5 * (lo[c] + hi[c]);
  extent = std::sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                     (hi[2] - lo[2]) * (hi[2] - lo[2]));
  std::vector<float> h4((size_t)4 * n), l4((size_t)4 * n);
  for (int i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c) {
      double v = p4[4 * (size_t)i + c] - center[c];
      float h = (float)v;
      h4[4 * (size_t)i + c] = h;
      l4[4 * (size_t)i + c] = (float)(v - (double)h);
    }
    h4[4 * (size_t)i + 3] = 0.f;
    l4[4 * (size_t)i + 3] = 0.f;
  }
  LUM_TRY(pos64.alloc(sizeof(double) * 4 * (size_t)n));
  LUM_TRY(pos_hi.alloc(sizeof(float) * 4 * (size_t)n));
  LUM_TRY(pos_lo.alloc(sizeof(float) * 4 * (size_t)n));
  // ordered on the session stream with every later kernel (pageable sources
  // are staged before the call returns)
  LUM_TRY_CUDA(cudaMemcpyAsync(pos64.p, p4.data(), pos64.bytes, cudaMemcpyHostToDevice, st));
  LUM_TRY_CUDA(cudaMemcpyAsync(pos_hi.p, h4.data(), pos_hi.bytes, cudaMemcpyHostToDevice, st));
  LUM_TRY_CUDA(cudaMemcpyAsync(pos_lo.p, l4.data(), pos_lo.bytes, cudaMemcpyHostToDevice, st));
  host_pos.swap(p4);
  lofree = 1;
  for (float v : l4)
    if (v != 0.0f) {
      lofree = 0;
      break;
    }
  return LUM_OK;
}

static lum_status build_near_list(OtfOperator& op, cudaStream_t st) {
  const int n = op.n;
  DevBuf cnt, flag;
  LUM_TRY(cnt.alloc(sizeof(int) * (size_t)n));
  LUM_TRY(flag.alloc(sizeof(int)));
  LUM_TRY_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
  const double two_cell = 2.0 * op.cell;
  dim3 grid((n + 255) / 256);
  near_scan<false><<<grid, 256, 0, st>>>(n, op.pos64.as<double4>(), two_cell, op.use_fcd,
                                         cnt.as<int>(), 0, nullptr, flag.as<int>());
  LUM_CHECK_LAUNCH();
  std::vector<int> hc(n);
  int hflag = 0;
  LUM_TRY_CUDA(cudaMemcpyAsync(hc.data(), cnt.p, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaMemcpyAsync(&hflag, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));
  if (hflag) {
    set_error("Self-interaction: two dipoles share a position");
    return LUM_ERR_INVALID;
  }
  int w = 0;
  for (int v : hc) w = std::max(w, v);
  op.ell_w = w;
  if (w > 0) {
    LUM_TRY(op.near_j.alloc(sizeof(int) * (size_t)w * n));
    LUM_TRY_CUDA(cudaMemsetAsync(op.near_j.p, 0xff, op.near_j.bytes, st));
    near_scan<true><<<grid, 256, 0, st>>>(n, op.pos64.as<double4>(), two_cell, op.use_fcd,
                                          nullptr, w, op.near_j.as<int>(), flag.as<int>());
    LUM_CHECK_LAUNCH();
    LUM_TRY(op.fcd64.alloc(sizeof(double2) * 9 * (size_t)w * n));
    LUM_TRY(op.fcd32.alloc(sizeof(float2) * 9 * (size_t)w * n));
  }
  LUM_TRY_CUDA(cudaStreamSynchronize(st));
  return LUM_OK;
}

static void lattice_points(const lum_lattice& L, std::vector<double>& real,
                           std::vector<double>& recip, LatticeDev& D) {
  // lattice.rs:75-233
  D.is_2d = L.is_2d;
  if (L.is_2d) {
    double cx = L.a1[1] * L.a2[2] - L.a1[2] * L.a2[1];
    double cy = L.a1[2] * L.a2[0] - L.a1[0] * L.a2[2];
    double cz = L.a1[0] * L.a2[1] - L.a1[1] * L.a2[0];
    D.area = std::sqrt(cx * cx + cy * cy + cz * cz);
  } else {
    D.area = std::sqrt(L.a1[0] * L.a1[0] + L.a1[1] * L.a1[1] + L.a1[2] * L.a1[2]);
  }
  D.eta = L.has_eta ? L.eta : std::sqrt(kPi / D.area);
  int ns = L.is_2d ? L.truncation_real : std::max(L.truncation_real, 20);
  real.clear();
  recip.clear();
  if (L.is_2d) {
    for (int m1 = -ns; m1 <= ns; ++m1)
      for (int m2 = -ns; m2 <= ns; ++m2) {
        real.push_back(m1 * L.a1[0] + m2 * L.a2[0]);
        real.push_back(m1 * L.a1[1] + m2 * L.a2[1]);
        real.push_back(m1 * L.a1[2] + m2 * L.a2[2]);
        real.push_back(0.0);
      }
    const double two_pi = 2.0 * kPi;
    const double* a1 = L.a1;
    const double* a2 = L.a2;
    double a2xz[2] = {a2[1], -a2[0]};
    double d1 = a1[0] * a2xz[0] + a1[1] * a2xz[1];
    double b1[2] = {two_pi * a2xz[0] / d1, two_pi * a2xz[1] / d1};
    double zxa1[2] = {-a1[1], a1[0]};
    double d2 = a2[0] * zxa1[0] + a2[1] * zxa1[1];
    double b2[2] = {two_pi * zxa1[0] / d2, two_pi * zxa1[1] / d2};
    int nr = L.truncation_recip;
    for (int n1 = -nr; n1 <= nr; ++n1)
      for (int n2 = -nr; n2 <= nr; ++n2) {
        recip.push_back(n1 * b1[0] + n2 * b2[0]);
        recip.push_back(n1 * b1[1] + n2 * b2[1]);
        recip.push_back(0.0);
        recip.push_back(0.0);
      }
  } else {
    for (int m1 = -ns; m1 <= ns; ++m1) {
      real.push_back(m1 * L.a1[0]);
      real.push_back(m1 * L.a1[1]);
      real.push_back(m1 * L.a1[2]);
      real.push_back(0.0);
    }
    D.a1_len = D.area;
    for (int c = 0; c < 3; ++c) D.e_hat[c] = L.a1[c] / D.a1_len;
    recip.assign(4, 0.0);
  }
  for (int c = 0; c < 3; ++c) D.a1[c] = L.a1[c];
  D.n_real = (int)(real.size() / 4);
  D.n_recip = L.is_2d ? (int)(recip.size() / 4) : 0;
}

lum_status OtfOperator::set_physics(double k_, const double* inv_alpha_host, int use_fcd_,
                                    double cell_, const lum_lattice* lat, const double* kb,
                                    const lum_substrate* sub, cudaStream_t st) {
  const bool first = (inv_alpha.p == nullptr);
  if (!(k_ > 0.0) || !std::isfinite(k_)) {
    set_error("wavenumber must be positive and finite (got %g)", k_);
    return LUM_ERR_INVALID;
  }
  k = k_;
  if (first) {
    LUM_TRY(sincos_table_ready());  // the FP64 symmetric kernels' sin / cos table
    use_fcd = use_fcd_;
    cell = cell_;
    has_lattice = lat != nullptr;
    if (has_lattice) {
      lattice = *lat;
      use_fcd = 0;  // the Ewald branch wins over FCD (assembly.rs:94-104)
    }
    if (kb) {
      kbloch[0] = kb[0];
      kbloch[1] = kb[1];
      kbloch[2] = kb[2];
    }
    if (use_fcd && !(cell > 0.0)) {
      set_error("FCD needs a positive cell size (got %g)", cell);
      return LUM_ERR_INVALID;
    }
    LUM_TRY(build_near_list(*this, st));
    if (has_lattice) {
      std::vector<double> re, rc;
      lattice_points(lattice, re, rc, latdev);
      LUM_TRY(lat_real.alloc(sizeof(double) * re.size()));
      LUM_TRY(lat_recip.alloc(sizeof(double) * rc.size()));
      LUM_TRY_CUDA(cudaMemcpyAsync(lat_real.p, re.data(), lat_real.bytes, cudaMemcpyHostToDevice, st));
      LUM_TRY_CUDA(cudaMemcpyAsync(lat_recip.p, rc.data(), lat_recip.bytes, cudaMemcpyHostToDevice, st));
      LUM_TRY(table_detect(st));
    }
  }
  if (has_lattice && !latdev.is_2d)
    latdev.m_max = std::min((long)std::ceil(k * latdev.a1_len / (2.0 * kPi) + 10.0), 50L);
  has_substrate = sub != nullptr;
  if (has_substrate) {
    substrate.z_interface = sub->z_interface;
    substrate.refl_re = sub->refl_re;
    substrate.refl_im = sub->refl_im;
    // image positions for the FP32 kernel (centred like the observers)
    const std::vector<double>& p4 = host_pos;
    std::vector<float> h4((size_t)4 * n), l4((size_t)4 * n);
    for (int i = 0; i < n; ++i) {
      double im[3] = {p4[4 * (size_t)i], p4[4 * (size_t)i + 1],
                      2.0 * substrate.z_interface - p4[4 * (size_t)i + 2]};
      for (int c = 0; c < 3; ++c) {
        double v = im[c] - center[c];
        float h = (float)v;
        h4[4 * (size_t)i + c] = h;
        l4[4 * (size_t)i + c] = (float)(v - (double)h);
      }
      h4[4 * (size_t)i + 3] = 0.f;
      l4[4 * (size_t)i + 3] = 0.f;
    }
    if (!img_hi.p) {
      LUM_TRY(img_hi.alloc(sizeof(float) * 4 * (size_t)n));
      LUM_TRY(img_lo.alloc(sizeof(float) * 4 * (size_t)n));
    }
    img_lofree = 1;
    for (float v : l4)
      if (v != 0.0f) {
        img_lofree = 0;
        break;
      }
    LUM_TRY_CUDA(cudaMemcpyAsync(img_hi.p, h4.data(), img_hi.bytes, cudaMemcpyHostToDevice, st));
    LUM_TRY_CUDA(cudaMemcpyAsync(img_lo.p, l4.data(), img_lo.bytes, cudaMemcpyHostToDevice, st));
  }
  // alpha^-1, element-major
  std::vector<double> ia((size_t)18 * n);
  for (int i = 0; i < n; ++i)
    for (int e = 0; e < 9; ++e) {
      ia[2 * ((size_t)e * n + i)] = inv_alpha_host[18 * (size_t)i + 2 * e];
      ia[2 * ((size_t)e * n + i) + 1] = inv_alpha_host[18 * (size_t)i + 2 * e + 1];
    }
  if (first) LUM_TRY(inv_alpha.alloc(sizeof(double) * ia.size()));
  LUM_TRY_CUDA(cudaMemcpyAsync(inv_alpha.p, ia.data(), inv_alpha.bytes, cudaMemcpyHostToDevice, st));
  // periodic tensor tables for this wavelength / Bloch vector / substrate
  if (has_lattice && table_ok) LUM_TRY(table_build(st));
  // FCD corrections for this wavelength
  if (ell_w > 0) {
    int total = ell_w * n;
    fcd_table<<<(total + 127) / 128, 128, 0, st>>>(n, ell_w, pos64.as<double4>(),
                                                   near_j.as<int>(), k, cell,
                                                   fcd64.as<double2>(), fcd32.as<float2>());
    LUM_CHECK_LAUNCH();
  }
  const int old_fast = fast_trig;
  fast_trig = (k * extent < 3.0) ? 1 : 0;
  // partial-sum scratch, sized for the largest split of any FP32 variant
  if (first) {
    const int sms = device_sms();
    const int ntiles = (n + kOtfBlock - 1) / kOtfBlock;
    size_t max_parts32 = 1;
    for (int v = 0; v < kNumF32Variants; ++v) {
      const int rows = kF32Variants[v].rows;
      const int occ = kF32Variants[v].occupancy(1, lofree);
      const int rb = (n + kOtfBlock * rows - 1) / (kOtfBlock * rows);
      nsplit_v[v] = choose_nsplit(rb, ntiles, occ, sms);
      max_parts32 = std::max<size_t>(max_parts32, nsplit_v[v]);
    }
    int occ64 = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ64, otf_pairs_f64<false>, kOtfBlock, 0);
    nsplit64 = choose_nsplit(ntiles, ntiles, std::max(1, occ64), sms);
    nsplit64 = std::max(nsplit64, table_ok ? nsplit_tab : 1);
    const size_t bytes = std::max(sizeof(float2) * max_parts32 * 2,
                                  sizeof(double2) * (size_t)nsplit64 * 2) * 3 * (size_t)n;
    LUM_TRY(partial.alloc(bytes));
  }
  if (first) LUM_TRY(tune_f64(st));
  if (first || old_fast != fast_trig) {
    LUM_TRY(tune_f32(st));
    f32x2_variant = -1;  // the two-vector variant is tuned again on first use
  }
  return LUM_OK;
}

// Autotuner of the pair kernels: every build of the FP32 kernel (split
// variants: rows per thread x register cap, each with its own wave-filling
// split; symmetric variants) and both FP64 schemes are timed on this
// geometry -- one warm launch, then the best of three -- and the fastest is
// kept.  Choices are cached in memory and in the tuner's JSON file
// (tune_cache.cu) per (device, kernel build, N, trig flavour, flags);
// LUMINA_TUNE=0 keeps the first split variant and the split FP64 kernel.
namespace {
const char kKernelBuild[] = __DATE__ "_" __TIME__;

std::string tune_key(const char* family, int n, int trig, int flags) {
  std::string build(kKernelBuild);
  for (char& c : build)
    if (c == ' ') c = '_';
  return std::string(family) + "|" + tune_device_tag() + "|" + build + "|n=" +
         std::to_string(n) + "|trig=" + std::to_string(trig) + "|flags=" + std::to_string(flags);
}

// One warm launch, then the best of three timed launches.
template <typename F>
lum_status time_best(F&& launch, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1,
                     const char* what, float* best_ms) {
  launch();
  float best = 1e30f;
  for (int rep = 0; rep < 3; ++rep) {
    cudaEventRecord(e0, st);
    launch();
    cudaEventRecord(e1, st);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, what, __FILE__, __LINE__);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    best = std::min(best, ms);
  }
  g_launches.fetch_add(4, std::memory_order_relaxed);
  *best_ms = best;
  return LUM_OK;
}

struct EventPair {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ~EventPair() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
  lum_status create() {
    LUM_TRY_CUDA(cudaEventCreate(&e0));
    LUM_TRY_CUDA(cudaEventCreate(&e1));
    return LUM_OK;
  }
};
}  // namespace

// Superblock pairs (I <= J) and the per-superblock partial sums of the
// symmetric scheme (sized once per geometry).
lum_status OtfOperator::sym_prepare(cudaStream_t st) {
  const int nb = (n + kSymRows - 1) / kSymRows;
  if (nb == sym_nb && sym_items.p) return LUM_OK;
  std::vector<int2> items;
  items.reserve((size_t)nb * (nb + 1) / 2);
  for (int I = 0; I < nb; ++I)
    for (int J = I; J < nb; ++J) items.push_back(make_int2(I, J));
  LUM_TRY(sym_items.alloc(sizeof(int2) * items.size()));
  LUM_TRY_CUDA(cudaMemcpyAsync(sym_items.p, items.data(), sizeof(int2) * items.size(),
                               cudaMemcpyHostToDevice, st));
  // sized for the FP64 scheme; the FP32 scheme uses the first half (or both
  // halves for two vectors)
  LUM_TRY(sym_slots.alloc(sizeof(double2) * (size_t)nb * 3 * (size_t)n));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));  // items is freed on return
  sym_nb = nb;
  sym_nitems = (int)items.size();
  return LUM_OK;
}

template <int MINB, int RP, int UNR = 1>
static void sym_launch_t(const OtfOperator& o, const double2* x, const int* skip,
                         cudaStream_t st) {
  const float kf = (float)o.k, s0f = (float)(o.k * o.k * o.k / (4.0 * kPi));
#define LUM_SYM_LAUNCH(F, L)                                                                  \
  otf_pairs_f32_sym<F, L, MINB, RP, UNR><<<o.sym_nitems, SymShape<RP>::kThreads, 0, st>>>(    \
      o.n, o.pos_hi.as<float4>(), o.pos_lo.as<float4>(), x, kf, s0f, o.sym_items.as<int2>(), \
      o.sym_slots.as<float2>(), skip)
  if (o.fast_trig && o.lofree)
    LUM_SYM_LAUNCH(true, true);
  else if (o.fast_trig)
    LUM_SYM_LAUNCH(true, false);
  else if (o.lofree)
    LUM_SYM_LAUNCH(false, true);
  else
    LUM_SYM_LAUNCH(false, false);
#undef LUM_SYM_LAUNCH
}

template <int MINB, int RP, int UNR = 1>
static void sym2_launch_t(const OtfOperator& o, const double2* x, const double2* x2,
                          const int* skip, const int* skip2, cudaStream_t st) {
  const float kf = (float)o.k, s0f = (float)(o.k * o.k * o.k / (4.0 * kPi));
  float2* s1 = o.sym_slots.as<float2>();
  float2* s2 = s1 + (size_t)o.sym_nb * 3 * (size_t)o.n;
#define LUM_SYM2_LAUNCH(F, L)                                                                 \
  otf_pairs_f32_sym2<F, L, MINB, RP, UNR><<<o.sym_nitems, SymShape<RP>::kThreads, 0, st>>>(   \
      o.n, o.pos_hi.as<float4>(), o.pos_lo.as<float4>(), x, x2, kf, s0f,                     \
      o.sym_items.as<int2>(), s1, s2, skip, skip2)
  if (o.fast_trig && o.lofree)
    LUM_SYM2_LAUNCH(true, true);
  else if (o.fast_trig)
    LUM_SYM2_LAUNCH(true, false);
  else if (o.lofree)
    LUM_SYM2_LAUNCH(false, true);
  else
    LUM_SYM2_LAUNCH(false, false);
#undef LUM_SYM2_LAUNCH
}

namespace {
// Builds of the symmetric FP32 scheme the tuner chooses from: rows per
// thread (2, 4 or 8) x CTAs per SM (the register cap) x unroll of the step
// loop.  f32_sym is 1 + the index into this table, 0 for the split kernels.
struct SymVariantEntry {
  const char* name;
  void (*launch)(const OtfOperator&, const double2*, const int*, cudaStream_t);
};
const SymVariantEntry kSymVariants[] = {
    {"sym_rows2_minb2", sym_launch_t<2, 1>},
    {"sym_rows2_minb3", sym_launch_t<3, 1>},
    {"sym_rows4_minb4", sym_launch_t<4, 2>},
    {"sym_rows4_minb3", sym_launch_t<3, 2>},
    {"sym_rows2_minb2_unroll2", sym_launch_t<2, 1, 2>},
    {"sym_rows4_minb3_unroll2", sym_launch_t<3, 2, 2>},
    {"sym_rows8_minb4", sym_launch_t<4, 4>},
    {"sym_rows8_minb5", sym_launch_t<5, 4>},
    {"sym_rows4_minb4_unroll2", sym_launch_t<4, 2, 2>},
    {"sym_rows4_minb3_unroll4", sym_launch_t<3, 2, 4>},
    {"sym_rows8_minb4_unroll2", sym_launch_t<4, 4, 2>},
    {"sym_rows4_minb4_unroll4", sym_launch_t<4, 2, 4>},
    {"sym_rows4_minb3_unroll8", sym_launch_t<3, 2, 8>},
};
constexpr int kNumSymVariants = sizeof(kSymVariants) / sizeof(kSymVariants[0]);

// Two-vector builds of the symmetric scheme; f32x2_sym is 1 + the index.
struct Sym2VariantEntry {
  const char* name;
  void (*launch)(const OtfOperator&, const double2*, const double2*, const int*, const int*,
                 cudaStream_t);
};
const Sym2VariantEntry kSym2Variants[] = {
    {"sym2_rows2_minb2", sym2_launch_t<2, 1>},
    {"sym2_rows2_minb1", sym2_launch_t<1, 1>},
    {"sym2_rows4_minb2", sym2_launch_t<2, 2>},
    {"sym2_rows4_minb2_unroll2", sym2_launch_t<2, 2, 2>},
};
constexpr int kNumSym2Variants = sizeof(kSym2Variants) / sizeof(kSym2Variants[0]);
}  // namespace

const char* sym_variant_name(int v) {
  return (v >= 1 && v <= kNumSymVariants) ? kSymVariants[v - 1].name : "none";
}

const char* sym2_variant_name(int v) {
  return (v >= 1 && v <= kNumSym2Variants) ? kSym2Variants[v - 1].name : "none";
}

void OtfOperator::sym_launch(int variant, const double2* x, const int* skip, cudaStream_t st) {
  kSymVariants[std::min(std::max(variant, 1), kNumSymVariants) - 1].launch(*this, x, skip, st);
}

void OtfOperator::sym2_launch(int variant, const double2* x, const double2* x2, const int* skip,
                              const int* skip2, cudaStream_t st) {
  kSym2Variants[std::min(std::max(variant, 1), kNumSym2Variants) - 1].launch(*this, x, x2, skip,
                                                                            skip2, st);
}

void OtfOperator::sym64_launch(const double2* x, const int* skip, cudaStream_t st) {
  otf_pairs_f64_sym<<<sym_nitems, kSym64Threads, 0, st>>>(
      n, pos64.as<double4>(), x, k, 1.0 / k, k * k * k / (4.0 * kPi), sym_items.as<int2>(),
      sym_slots.as<double2>(), skip);
}

lum_status OtfOperator::tune_f32(cudaStream_t st) {
  f32_variant = 0;
  f32_sym = 0;
  nsplit32 = nsplit_v[0];
  const bool isolated = !has_lattice && !has_substrate;
  // LUMINA_F32_SYM=v (1..kNumSymVariants) forces symmetric build v on
  // isolated systems (no lattice, no substrate image); =0 excludes the
  // symmetric scheme.
  const char* sym_env = std::getenv("LUMINA_F32_SYM");
  const int sym_forced = sym_env ? std::atoi(sym_env) : 0;
  if (isolated && sym_forced >= 1) {
    f32_sym = std::min(sym_forced, kNumSymVariants);
    return sym_prepare(st);
  }
  const bool sym_allowed = isolated && !(sym_env && sym_env[0] == '0');
  const char* env = std::getenv("LUMINA_TUNE");
  if ((env && env[0] == '0') || n < 2048) return LUM_OK;
  const std::string key = tune_key("f32", n, fast_trig,
                                   lofree + 2 * (isolated ? 0 : 1) + 4 * (sym_allowed ? 0 : 1));
  int choice = 0;
  if (tune_lookup(key, &choice)) {
    f32_variant = std::min(std::max(choice % 100, 0), kNumF32Variants - 1);
    f32_sym = sym_allowed ? std::min(choice / 100, kNumSymVariants) : 0;
    nsplit32 = nsplit_v[f32_variant];
    return f32_sym ? sym_prepare(st) : LUM_OK;
  }
  DevBuf xz;
  LUM_TRY(xz.alloc(sizeof(double2) * 3 * (size_t)n));
  LUM_TRY_CUDA(cudaMemsetAsync(xz.p, 0, xz.bytes, st));
  EventPair ev;
  LUM_TRY(ev.create());
  const int ntiles = (n + kOtfBlock - 1) / kOtfBlock;
  const double s0 = k * k * k / (4.0 * kPi);
  float best = 1e30f;
  for (int v = 0; v < kNumF32Variants; ++v) {
    const int rows = kF32Variants[v].rows, ns = nsplit_v[v];
    const int chunk = ((ntiles + ns - 1) / ns) * kOtfBlock;
    dim3 grid((n + kOtfBlock * rows - 1) / (kOtfBlock * rows), ns);
    F32Args a{n, pos_hi.as<float4>(), pos_lo.as<float4>(), pos_hi.as<float4>(),
              pos_lo.as<float4>(), xz.as<double2>(), make_float2(1.f, 0.f),
              make_float2(1.f, 0.f), make_float2(1.f, 0.f), (float)k, (float)(1.0 / k),
              (float)s0, chunk, partial.as<float2>(), nullptr};
    float ms = 0.f;
    LUM_TRY(time_best([&] { kF32Variants[v].direct(fast_trig, lofree, grid, st, a); }, st,
                      ev.e0, ev.e1, "pair-kernel tuning", &ms));
    if (ms < best) {
      best = ms;
      f32_variant = v;
    }
  }
  // the symmetric scheme (isolated systems: no lattice, no substrate image)
  if (sym_allowed) {
    LUM_TRY(sym_prepare(st));
    tuned_sym_ms = 1e30f;
    for (int v = 1; v <= kNumSymVariants; ++v) {
      float ms = 0.f;
      LUM_TRY(time_best([&] { sym_launch(v, xz.as<double2>(), nullptr, st); }, st, ev.e0,
                        ev.e1, "symmetric pair-kernel tuning", &ms));
      tuned_sym_ms = std::min(tuned_sym_ms, ms);
      if (ms < best) {
        best = ms;
        f32_sym = v;
      }
    }
  }
  nsplit32 = nsplit_v[f32_variant];
  tuned_ms = best;
  tune_store(key, f32_variant + 100 * f32_sym);
  return LUM_OK;
}

// FP64 scheme: the split kernel (otf_pairs_f64) or, on isolated systems, the
// symmetric one (otf_pairs_f64_sym); LUMINA_F64_SYM=1 forces the symmetric
// scheme there, =0 excludes it.
lum_status OtfOperator::tune_f64(cudaStream_t st) {
  f64_sym = 0;
  const bool isolated = !has_lattice && !has_substrate;
  if (!isolated) return LUM_OK;
  const char* sym_env = std::getenv("LUMINA_F64_SYM");
  if (sym_env && sym_env[0] == '0') return LUM_OK;
  if (sym_env && sym_env[0] == '1') {
    f64_sym = 1;
    return sym_prepare(st);
  }
  const char* env = std::getenv("LUMINA_TUNE");
  if ((env && env[0] == '0') || n < 2048) return LUM_OK;
  const std::string key = tune_key("f64", n, 0, 0);
  int choice = 0;
  if (tune_lookup(key, &choice)) {
    f64_sym = choice ? 1 : 0;
    return f64_sym ? sym_prepare(st) : LUM_OK;
  }
  LUM_TRY(sym_prepare(st));
  DevBuf xz;
  LUM_TRY(xz.alloc(sizeof(double2) * 3 * (size_t)n));
  LUM_TRY_CUDA(cudaMemsetAsync(xz.p, 0, xz.bytes, st));
  EventPair ev;
  LUM_TRY(ev.create());
  const int ntiles = (n + kOtfBlock - 1) / kOtfBlock;
  const int ns = nsplit64;
  const int chunk = ((ntiles + ns - 1) / ns) * kOtfBlock;
  const double2 one = make_double2(1.0, 0.0);
  float ms_split = 0.f, ms_sym = 0.f;
  LUM_TRY(time_best(
      [&] {
        otf_pairs_f64<false><<<dim3(ntiles, ns), kOtfBlock, 0, st>>>(
            n, pos64.as<double4>(), xz.as<double2>(), one, one, one, 0.0, k, 1.0 / k,
            k * k * k / (4.0 * kPi), chunk, partial.as<double2>(), nullptr);
      },
      st, ev.e0, ev.e1, "FP64 pair-kernel tuning", &ms_split));
  LUM_TRY(time_best([&] { sym64_launch(xz.as<double2>(), nullptr, st); }, st, ev.e0, ev.e1,
                    "FP64 symmetric pair-kernel tuning", &ms_sym));
  tuned_f64_ms = std::min(ms_split, ms_sym);
  f64_sym = ms_sym < ms_split ? 1 : 0;
  tune_store(key, f64_sym);
  return LUM_OK;
}

lum_status OtfOperator::apply(int precision, const double2* x, double2* y, cudaStream_t st,
                              cudaEvent_t ev0, cudaEvent_t ev1, const int* skip) {
  const int ntiles = (n + kOtfBlock - 1) / kOtfBlock;
  const double s0 = k * k * k / (4.0 * kPi);
  const int epi_blocks = (int)(((size_t)n * kEpiTPR + 255) / 256);
  if (has_lattice && table_ok) {
    // Periodic operator on a dipole lattice: gather from the FP32 or FP64 table.
    int nparts = 1;
    if (ev0) cudaEventRecord(ev0, st);
    LUM_TRY(table_apply(precision, x, partial.as<double2>(), st, skip, &nparts));
    if (ev1) cudaEventRecord(ev1, st);
    if (precision == LUM_FP32)
      otf_epilogue<float2, float2><<<epi_blocks, 256, 0, st>>>(
          n, x, inv_alpha.as<double2>(), partial.as<float2>(), nparts, 0, nullptr, nullptr, y,
          skip);
    else
      otf_epilogue<double2, double2><<<epi_blocks, 256, 0, st>>>(
          n, x, inv_alpha.as<double2>(), partial.as<double2>(), nparts, 0, nullptr, nullptr, y,
          skip);
    LUM_CHECK_LAUNCH();
    return LUM_OK;
  }
  if (has_lattice) {
    // Off-lattice periodic geometry: per-pair Ewald kernel (FP64) for either precision.
    const int ns = nsplit64;
    const int chunk = ((n + ns - 1) / ns);
    dim3 grid(ntiles, ns);
    if (ev0) cudaEventRecord(ev0, st);
    otf_pairs_ewald<<<grid, kOtfBlock, 0, st>>>(
        n, pos64.as<double4>(), x, latdev, lat_real.as<double4>(), lat_recip.as<double4>(),
        kbloch[0], kbloch[1], kbloch[2], k, has_substrate, substrate, chunk,
        partial.as<double2>(), skip);
    LUM_CHECK_LAUNCH();
    if (ev1) cudaEventRecord(ev1, st);
    otf_epilogue<double2, double2><<<epi_blocks, 256, 0, st>>>(
        n, x, inv_alpha.as<double2>(), partial.as<double2>(), ns, 0, nullptr, nullptr, y, skip);
    LUM_CHECK_LAUNCH();
    return LUM_OK;
  }
  const double2 rr = make_double2(substrate.refl_re, substrate.refl_im);
  if (precision == LUM_FP32 && f32_sym) {
    if (ev0) cudaEventRecord(ev0, st);
    sym_launch(f32_sym, x, skip, st);
    LUM_CHECK_LAUNCH();
    if (ev1) cudaEventRecord(ev1, st);
    otf_epilogue<float2, float2><<<epi_blocks, 256, 0, st>>>(
        n, x, inv_alpha.as<double2>(), sym_slots.as<float2>(), sym_nb, ell_w, near_j.as<int>(),
        fcd32.as<float2>(), y, skip);
    LUM_CHECK_LAUNCH();
    return LUM_OK;
  }
  if (precision == LUM_FP32) {
    const F32VariantEntry& V = kF32Variants[f32_variant];
    const int ns = nsplit32;
    const int chunk = ((ntiles + ns - 1) / ns) * kOtfBlock;
    const int rb = (n + kOtfBlock * V.rows - 1) / (kOtfBlock * V.rows);
    dim3 grid(rb, ns);
    const float kf = (float)k, ikf = (float)(1.0 / k), s0f = (float)s0;
    const float2 one = make_float2(1.f, 0.f);
    float2* part = partial.as<float2>();
    F32Args a{n, pos_hi.as<float4>(), pos_lo.as<float4>(), pos_hi.as<float4>(),
              pos_lo.as<float4>(), x, one, one, one, kf, ikf, s0f, chunk, part, skip};
    if (ev0) cudaEventRecord(ev0, st);
    V.direct(fast_trig, lofree, grid, st, a);
    LUM_CHECK_LAUNCH();
    if (ev1) cudaEventRecord(ev1, st);
    int nparts = ns;
    if (has_substrate) {
      const float2 mneg = make_float2((float)-rr.x, (float)-rr.y);
      const float2 mpos = make_float2((float)rr.x, (float)rr.y);
      F32Args b = a;
      b.sh = img_hi.as<float4>();
      b.sl = img_lo.as<float4>();
      b.m0 = mneg;
      b.m1 = mneg;
      b.m2 = mpos;
      b.part = part + (size_t)ns * 3 * n;
      V.image(fast_trig, lofree && img_lofree, grid, st, b);
      LUM_CHECK_LAUNCH();
      nparts = 2 * ns;
    }
    otf_epilogue<float2, float2><<<epi_blocks, 256, 0, st>>>(
        n, x, inv_alpha.as<double2>(), part, nparts, ell_w, near_j.as<int>(),
        fcd32.as<float2>(), y, skip);
    LUM_CHECK_LAUNCH();
    return LUM_OK;
  }
  // FP64
  if (f64_sym && !has_substrate) {
    if (ev0) cudaEventRecord(ev0, st);
    sym64_launch(x, skip, st);
    LUM_CHECK_LAUNCH();
    if (ev1) cudaEventRecord(ev1, st);
    otf_epilogue<double2, double2><<<epi_blocks, 256, 0, st>>>(
        n, x, inv_alpha.as<double2>(), sym_slots.as<double2>(), sym_nb, ell_w,
        near_j.as<int>(), fcd64.as<double2>(), y, skip);
    LUM_CHECK_LAUNCH();
    return LUM_OK;
  }
  const int ns = nsplit64;
  const int chunk = ((ntiles + ns - 1) / ns) * kOtfBlock;
  dim3 grid(ntiles, ns);
  const double2 one = make_double2(1.0, 0.0);
  double2* part = partial.as<double2>();
  if (ev0) cudaEventRecord(ev0, st);
  otf_pairs_f64<false><<<grid, kOtfBlock, 0, st>>>(n, pos64.as<double4>(), x, one, one, one, 0.0,
                                                   k, 1.0 / k, s0, chunk, part, skip);
  LUM_CHECK_LAUNCH();
  if (ev1) cudaEventRecord(ev1, st);
  int nparts = ns;
  if (has_substrate) {
    const double2 mneg = make_double2(-rr.x, -rr.y);
    otf_pairs_f64<true><<<grid, kOtfBlock, 0, st>>>(
        n, pos64.as<double4>(), x, mneg, mneg, rr, 2.0 * substrate.z_interface, k, 1.0 / k, s0,
        chunk, part + (size_t)ns * 3 * n, skip);
    LUM_CHECK_LAUNCH();
    nparts = 2 * ns;
  }
  otf_epilogue<double2, double2><<<epi_blocks, 256, 0, st>>>(
      n, x, inv_alpha.as<double2>(), part, nparts, ell_w, near_j.as<int>(),
      fcd64.as<double2>(), y, skip);
  LUM_CHECK_LAUNCH();
  return LUM_OK;
}


// ---------------------------------------------------------------------------
// Two right-hand sides per application (multi-RHS solves, forward + adjoint)
// ---------------------------------------------------------------------------
lum_status OtfOperator::tune_f32_x2(cudaStream_t st) {
  const int sms = device_sms();
  const int ntiles = (n + kOtfBlock - 1) / kOtfBlock;
  // room for the direct and image splits of each vector in partial / partial2
  const int cap = std::max(1, (int)(partial.bytes / (sizeof(float2) * 3 * (size_t)n * 2)));
  int ns_v[kNumF32X2Variants];
  for (int v = 0; v < kNumF32X2Variants; ++v) {
    const int rows = kF32X2Variants[v].rows;
    const int rb = (n + kOtfBlock * rows - 1) / (kOtfBlock * rows);
    ns_v[v] = std::min(cap, choose_nsplit(rb, ntiles, kF32X2Variants[v].occupancy(fast_trig, lofree),
                                          sms));
  }
  f32x2_variant = 0;
  f32x2_sym = 0;
  nsplit_x2 = ns_v[0];
  const bool isolated = !has_lattice && !has_substrate;
  // LUMINA_F32_SYM=v forces symmetric build v here too (the two-vector build
  // of that number, capped at the last), =0 excludes the symmetric scheme
  const char* sym_env = std::getenv("LUMINA_F32_SYM");
  const int sym_forced = sym_env ? std::atoi(sym_env) : 0;
  if (isolated && sym_forced >= 1) {
    f32x2_sym = std::min(sym_forced, kNumSym2Variants);
    return sym_prepare(st);
  }
  const bool sym_allowed = isolated && !(sym_env && sym_env[0] == '0');
  const char* env = std::getenv("LUMINA_TUNE");
  if ((env && env[0] == '0') || n < 2048) return LUM_OK;
  const std::string key = tune_key("f32x2", n, fast_trig,
                                   lofree + 2 * (isolated ? 0 : 1) + 4 * (sym_allowed ? 0 : 1));
  int choice = 0;
  if (tune_lookup(key, &choice)) {
    f32x2_variant = std::min(std::max(choice % 100, 0), kNumF32X2Variants - 1);
    f32x2_sym = sym_allowed ? std::min(choice / 100, kNumSym2Variants) : 0;
    nsplit_x2 = ns_v[f32x2_variant];
    return f32x2_sym ? sym_prepare(st) : LUM_OK;
  }
  DevBuf xz;
  LUM_TRY(xz.alloc(sizeof(double2) * 3 * (size_t)n));
  LUM_TRY_CUDA(cudaMemsetAsync(xz.p, 0, xz.bytes, st));
  EventPair ev;
  LUM_TRY(ev.create());
  const double s0 = k * k * k / (4.0 * kPi);
  float best = 1e30f;
  for (int v = 0; v < kNumF32X2Variants; ++v) {
    const int rows = kF32X2Variants[v].rows, ns = ns_v[v];
    const int chunk = ((ntiles + ns - 1) / ns) * kOtfBlock;
    dim3 grid((n + kOtfBlock * rows - 1) / (kOtfBlock * rows), ns);
    const float2 one = make_float2(1.f, 0.f);
    F32X2Args a{n, pos_hi.as<float4>(), pos_lo.as<float4>(), pos_hi.as<float4>(),
                pos_lo.as<float4>(), xz.as<double2>(), xz.as<double2>(), one, one, one,
                (float)k, (float)(1.0 / k), (float)s0, chunk, partial.as<float2>(),
                partial2.as<float2>(), nullptr, nullptr};
    float ms = 0.f;
    LUM_TRY(time_best([&] { kF32X2Variants[v].direct(fast_trig, lofree, grid, st, a); }, st,
                      ev.e0, ev.e1, "two-vector pair-kernel tuning", &ms));
    if (ms < best) {
      best = ms;
      f32x2_variant = v;
    }
  }
  if (sym_allowed) {
    LUM_TRY(sym_prepare(st));
    for (int v = 1; v <= kNumSym2Variants; ++v) {
      float ms = 0.f;
      LUM_TRY(time_best(
          [&] { sym2_launch(v, xz.as<double2>(), xz.as<double2>(), nullptr, nullptr, st); }, st,
          ev.e0, ev.e1, "two-vector symmetric pair-kernel tuning", &ms));
      if (ms < best) {
        best = ms;
        f32x2_sym = v;
      }
    }
  }
  nsplit_x2 = ns_v[f32x2_variant];
  tuned_x2_ms = best;
  tune_store(key, f32x2_variant + 100 * f32x2_sym);
  return LUM_OK;
}

lum_status OtfOperator::apply2(int precision, const double2* x, const double2* x2, double2* y,
                               double2* y2, cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1,
                               const int* skip, const int* skip2) {
  if (has_lattice) {  // tabulated / per-pair Ewald operators: one vector at a time
    LUM_TRY(apply(precision, x, y, st, ev0, ev1, skip));
    return apply(precision, x2, y2, st, nullptr, nullptr, skip2);
  }
  if (!partial2.p) LUM_TRY(partial2.alloc(partial.bytes));
  const int ntiles = (n + kOtfBlock - 1) / kOtfBlock;
  const double s0 = k * k * k / (4.0 * kPi);
  const int epi_blocks = (int)(((size_t)n * kEpiTPR + 255) / 256);
  const double2 rr = make_double2(substrate.refl_re, substrate.refl_im);
  const size_t slice = 3 * (size_t)n;
  if (precision == LUM_FP32) {
    if (f32x2_variant < 0) LUM_TRY(tune_f32_x2(st));
    if (f32x2_sym && !has_substrate) {
      if (ev0) cudaEventRecord(ev0, st);
      sym2_launch(f32x2_sym, x, x2, skip, skip2, st);
      LUM_CHECK_LAUNCH();
      if (ev1) cudaEventRecord(ev1, st);
      float2* s1 = sym_slots.as<float2>();
      otf_epilogue2<float2, float2><<<epi_blocks, 256, 0, st>>>(
          n, x, x2, inv_alpha.as<double2>(), s1, s1 + (size_t)sym_nb * slice, sym_nb, ell_w,
          near_j.as<int>(), fcd32.as<float2>(), y, y2, skip, skip2);
      LUM_CHECK_LAUNCH();
      return LUM_OK;
    }
    const F32X2VariantEntry& V = kF32X2Variants[f32x2_variant];
    const int ns = nsplit_x2;
    const int chunk = ((ntiles + ns - 1) / ns) * kOtfBlock;
    dim3 grid((n + kOtfBlock * V.rows - 1) / (kOtfBlock * V.rows), ns);
    const float2 one = make_float2(1.f, 0.f);
    float2 *part = partial.as<float2>(), *part2 = partial2.as<float2>();
    F32X2Args a{n, pos_hi.as<float4>(), pos_lo.as<float4>(), pos_hi.as<float4>(),
                pos_lo.as<float4>(), x, x2, one, one, one, (float)k, (float)(1.0 / k),
                (float)s0, chunk, part, part2, skip, skip2};
    if (ev0) cudaEventRecord(ev0, st);
    V.direct(fast_trig, lofree, grid, st, a);
    LUM_CHECK_LAUNCH();
    if (ev1) cudaEventRecord(ev1, st);
    int nparts = ns;
    if (has_substrate) {
      F32X2Args b = a;
      b.sh = img_hi.as<float4>();
      b.sl = img_lo.as<float4>();
      b.m0 = b.m1 = make_float2((float)-rr.x, (float)-rr.y);
      b.m2 = make_float2((float)rr.x, (float)rr.y);
      b.part = part + (size_t)ns * slice;
      b.part2 = part2 + (size_t)ns * slice;
      V.image(fast_trig, lofree && img_lofree, grid, st, b);
      LUM_CHECK_LAUNCH();
      nparts = 2 * ns;
    }
    otf_epilogue2<float2, float2><<<epi_blocks, 256, 0, st>>>(
        n, x, x2, inv_alpha.as<double2>(), part, part2, nparts, ell_w, near_j.as<int>(),
        fcd32.as<float2>(), y, y2, skip, skip2);
    LUM_CHECK_LAUNCH();
    return LUM_OK;
  }
  if (f64_sym && !has_substrate) {
    if (!sym_slots2.p) LUM_TRY(sym_slots2.alloc(sym_slots.bytes));
    double2 *s1 = sym_slots.as<double2>(), *s2 = sym_slots2.as<double2>();
    if (ev0) cudaEventRecord(ev0, st);
    otf_pairs_f64_sym2<<<sym_nitems, kSym64Threads, 0, st>>>(
        n, pos64.as<double4>(), x, x2, k, 1.0 / k, s0, sym_items.as<int2>(), s1, s2, skip, skip2);
    LUM_CHECK_LAUNCH();
    if (ev1) cudaEventRecord(ev1, st);
    otf_epilogue2<double2, double2><<<epi_blocks, 256, 0, st>>>(
        n, x, x2, inv_alpha.as<double2>(), s1, s2, sym_nb, ell_w, near_j.as<int>(),
        fcd64.as<double2>(), y, y2, skip, skip2);
    LUM_CHECK_LAUNCH();
    return LUM_OK;
  }
  const int ns = nsplit64;
  const int chunk = ((ntiles + ns - 1) / ns) * kOtfBlock;
  dim3 grid(ntiles, ns);
  const double2 one = make_double2(1.0, 0.0);
  double2 *part = partial.as<double2>(), *part2 = partial2.as<double2>();
  if (ev0) cudaEventRecord(ev0, st);
  otf_pairs_f64_x2<false><<<grid, kOtfBlock, 0, st>>>(n, pos64.as<double4>(), x, x2, one, one, one,
                                                      0.0, k, 1.0 / k, s0, chunk, part, part2,
                                                      skip, skip2);
  LUM_CHECK_LAUNCH();
  if (ev1) cudaEventRecord(ev1, st);
  int nparts = ns;
  if (has_substrate) {
    const double2 mneg = make_double2(-rr.x, -rr.y);
    otf_pairs_f64_x2<true><<<grid, kOtfBlock, 0, st>>>(
        n, pos64.as<double4>(), x, x2, mneg, mneg, rr, 2.0 * substrate.z_interface, k, 1.0 / k,
        s0, chunk, part + (size_t)ns * slice, part2 + (size_t)ns * slice, skip, skip2);
    LUM_CHECK_LAUNCH();
    nparts = 2 * ns;
  }
  otf_epilogue2<double2, double2><<<epi_blocks, 256, 0, st>>>(
      n, x, x2, inv_alpha.as<double2>(), part, part2, nparts, ell_w, near_j.as<int>(),
      fcd64.as<double2>(), y, y2, skip, skip2);
  LUM_CHECK_LAUNCH();
  return LUM_OK;
}

// ---------------------------------------------------------------------------
// Batched systems: K independent clusters concatenated into one dipole range
// (BatchGeom).  Each pair kernel is one persistent launch over a work list of
// (system, row tile, source split) items ordered by decreasing cost, drawn
// through an atomic counter so uneven cluster sizes balance across the SMs.
// Items of systems that have converged (or whose restart cycle has ended)
// are skipped at draw time.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool batch_skipped(const BatchFlags* flags, int s, int mode) {
  if (mode == 0) return false;
  const BatchFlags f = flags[s];
  return f.frozen || (mode == 1 && f.done);
}

// Next item for the whole CTA, or -1 once the list is exhausted.  When the
// list is exhausted the last CTA to leave resets both counters, so the same
// launch can be replayed (CUDA graph) without a memset.
__device__ __forceinline__ int batch_draw(unsigned* counters, int nitems, int* s_item) {
  __syncthreads();
  if (threadIdx.x == 0) *s_item = (int)atomicAdd(&counters[0], 1u);
  __syncthreads();
  const int it = *s_item;
  if (it < nitems) return it;
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&counters[1], 1u) == gridDim.x - 1) {
      counters[0] = 0u;
      counters[1] = 0u;
    }
  }
  return -1;
}

// MINB 6: 80 registers, 24 warps per SM (some spill); MINB 4: no spills,
// 16 warps per SM.
template <bool FAST, bool LOFREE, int MINB>
__global__ void __launch_bounds__(kOtfBlock, MINB)
batch_pairs_f32(BatchGeom g, const double2* __restrict__ x, const int4* __restrict__ items,
                int nitems, unsigned* counters, const BatchFlags* __restrict__ flags,
                int skip_mode, float2* __restrict__ partial) {
  __shared__ int s_item;
  const size_t stride = 3 * (size_t)g.N;
  const float2 one = make_float2(1.f, 0.f);
  for (int it; (it = batch_draw(counters, nitems, &s_item)) >= 0;) {
    const int4 item = items[it];
    const int s = item.x;
    if (batch_skipped(flags, s, skip_mode)) continue;  // CTA-uniform
    const int off = g.sys_off[s], n = g.sys_off[s + 1] - off;
    const int chunk = g.sys_chunk32[s];
    const int j0 = item.z * chunk, j1 = min(n, j0 + chunk);
    const double k = g.sys_k[s];
    pairs_f32_cta<FAST, false, LOFREE, 1, 1>(
        n, g.hi + off, g.lo + off, g.hi + off, g.lo + off, x + 3 * (size_t)off, nullptr, one,
        one, one, (float)k, (float)(1.0 / k), (float)(k * k * k / (4.0 * kPi)), item.y, j0, j1,
        partial + (size_t)item.z * stride + 3 * (size_t)off, nullptr);
  }
}

// The symmetric scheme over the batch: items (system, I, J), I <= J, the
// superblock pairs of each system (pairs_f32_sym.cuh), written to per-system
// slots laid out like the split partials, [superblock][3N] over the global
// dipole range, so the batch epilogue sums sys_nb[s] of them per row.
template <bool FAST, bool LOFREE, int MINB, int RP, int UNR = 1>
__global__ void __launch_bounds__(SymShape<RP>::kThreads, MINB)
batch_pairs_f32_sym(BatchGeom g, const double2* __restrict__ x, const int4* __restrict__ items,
                    int nitems, unsigned* counters, const BatchFlags* __restrict__ flags,
                    int skip_mode, float2* __restrict__ slots) {
  __shared__ int s_item;
  __shared__ float4 sS[6][32];
  __shared__ float2 sAcc[SymShape<RP>::kWarps * 32 * 6];
  __shared__ float sRed[32 * 6];
  const size_t stride = 3 * (size_t)g.N;
  for (int it; (it = batch_draw(counters, nitems, &s_item)) >= 0;) {
    const int4 item = items[it];
    const int s = item.x;
    if (batch_skipped(flags, s, skip_mode)) continue;  // CTA-uniform
    const int off = g.sys_off[s], n = g.sys_off[s + 1] - off;
    const double k = g.sys_k[s];
    sym_superblock_pair<FAST, LOFREE, RP, 1, UNR>(
        n, g.hi + off, g.lo + off, x + 3 * (size_t)off, nullptr, (float)k,
        (float)(k * k * k / (4.0 * kPi)), item.y, item.z, slots + 3 * (size_t)off, nullptr,
        stride, sS, sAcc, sRed);
  }
}

__global__ void __launch_bounds__(kOtfBlock)
batch_pairs_f64(BatchGeom g, const double2* __restrict__ x, const int4* __restrict__ items,
                int nitems, unsigned* counters, const BatchFlags* __restrict__ flags,
                int skip_mode, double2* __restrict__ partial) {
  __shared__ int s_item;
  __shared__ double2 sTab[kScTab];
  sincos_table_stage(sTab);  // staged once; the first tile's barrier precedes its use
  const size_t stride = 3 * (size_t)g.N;
  const double2 one = make_double2(1.0, 0.0);
  for (int it; (it = batch_draw(counters, nitems, &s_item)) >= 0;) {
    const int4 item = items[it];
    const int s = item.x;
    if (batch_skipped(flags, s, skip_mode)) continue;  // CTA-uniform
    const int off = g.sys_off[s], n = g.sys_off[s + 1] - off;
    const int chunk = g.sys_chunk64[s];
    const int j0 = item.z * chunk, j1 = min(n, j0 + chunk);
    const double k = g.sys_k[s];
    pairs_f64_cta<false, 1>(n, g.pos64 + off, x + 3 * (size_t)off, nullptr, one, one, one, 0.0,
                            k, 1.0 / k, k * k * k / (4.0 * kPi), item.y, j0, j1,
                            partial + (size_t)item.z * stride + 3 * (size_t)off, nullptr, sTab);
  }
}

// y = alpha^-1 x - sum(partials of the row's system) - sum_near C_ij x_j,
// the epilogue above with per-system split counts and skip flags.
template <typename TP, typename TC>
__global__ void __launch_bounds__(256)
batch_epilogue(BatchGeom g, const double2* __restrict__ x, const TP* __restrict__ partial,
               const int* __restrict__ sys_ns, const TC* __restrict__ fcd,
               const BatchFlags* __restrict__ flags, int skip_mode, double2* __restrict__ y) {
  const int N = g.N;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = min(gid / kEpiTPR, N - 1);
  const int sub = gid % kEpiTPR;
  const int s = g.row_sys[i];
  const bool live = gid / kEpiTPR < N && !batch_skipped(flags, s, skip_mode);
  const int nparts = live ? sys_ns[s] : 0;
  const int ell_w = live ? g.ell_w : 0;
  double gr[3] = {0, 0, 0}, gi[3] = {0, 0, 0};
  const size_t stride = 3 * (size_t)N;
  for (int p = sub; p < nparts; p += kEpiTPR) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double2 v = to_d2(partial[p * stride + 3 * (size_t)i + a]);
      gr[a] += v.x;
      gi[a] += v.y;
    }
  }
  for (int w = sub; w < ell_w; w += kEpiTPR) {
    const int j = g.near_j[(size_t)w * N + i];
    if (j < 0) break;  // lists are packed: the rest of this row is padding
    double2 xj[3] = {x[3 * (size_t)j], x[3 * (size_t)j + 1], x[3 * (size_t)j + 2]};
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        double2 c = to_d2(fcd[((size_t)w * 9 + 3 * a + b) * N + i]);
        gr[a] += c.x * xj[b].x - c.y * xj[b].y;
        gi[a] += c.x * xj[b].y + c.y * xj[b].x;
      }
  }
#pragma unroll
  for (int o = 1; o < kEpiTPR; o <<= 1)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      gr[a] += __shfl_xor_sync(0xffffffffu, gr[a], o);
      gi[a] += __shfl_xor_sync(0xffffffffu, gi[a], o);
    }
  if (!live || sub != 0) return;
  const double2 xi[3] = {x[3 * (size_t)i], x[3 * (size_t)i + 1], x[3 * (size_t)i + 2]};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      double2 m = g.inv_alpha[(size_t)(3 * a + b) * N + i];
      sr += m.x * xi[b].x - m.y * xi[b].y;
      si += m.x * xi[b].y + m.y * xi[b].x;
    }
    y[3 * (size_t)i + a] = make_double2(sr - gr[a], si - gi[a]);
  }
}

// Near-pair scan within each dipole's own system (same FP64 test as
// near_scan); thread per dipole, sources read through L1 (a warp's dipoles
// share a system, so the loads broadcast).
template <bool FILL>
__global__ void __launch_bounds__(256)
batch_near_scan(BatchGeom g, int use_fcd, int* __restrict__ count, int ell_w,
                int* __restrict__ near_j, int* __restrict__ coincident) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const int s = g.row_sys[i];
  const int jb = g.sys_off[s], je = g.sys_off[s + 1];
  const double two_cell = 2.0 * g.sys_cell[s];
  const double4 ri = g.pos64[i];
  int c = 0;
  for (int j = jb; j < je; ++j) {
    if (j == i) continue;
    const double d = ref_dist(ri, g.pos64[j]);
    if (d == 0.0) atomicOr(coincident, 1);
    if (use_fcd && !(d > two_cell)) {
      if (FILL && c < ell_w) near_j[(size_t)c * g.N + i] = j;
      ++c;
    }
  }
  if (!FILL) count[i] = c;
}

__global__ void __launch_bounds__(128)
batch_fcd_table(BatchGeom g, double2* __restrict__ fcd64, float2* __restrict__ fcd32) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int N = g.N;
  if (idx >= (size_t)N * g.ell_w) return;
  const int w = (int)(idx / N), i = (int)(idx % N);
  const int j = g.near_j[(size_t)w * N + i];
  const int s = g.row_sys[i];
  double2 C[9];
  fcd_correction(g.pos64, i, j, g.sys_k[s], g.sys_cell[s], C);
  for (int e = 0; e < 9; ++e) {
    fcd64[((size_t)w * 9 + e) * N + i] = C[e];
    fcd32[((size_t)w * 9 + e) * N + i] = make_float2((float)C[e].x, (float)C[e].y);
  }
}

lum_status batch_near_fcd(BatchGeom& g, int use_fcd, DevBuf& near_j, DevBuf& fcd64,
                          DevBuf& fcd32, cudaStream_t st) {
  const int N = g.N;
  DevBuf cnt, flag;
  LUM_TRY(cnt.alloc(sizeof(int) * (size_t)N));
  LUM_TRY(flag.alloc(sizeof(int)));
  LUM_TRY_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
  const int blocks = (N + 255) / 256;
  batch_near_scan<false><<<blocks, 256, 0, st>>>(g, use_fcd, cnt.as<int>(), 0, nullptr,
                                                 flag.as<int>());
  LUM_CHECK_LAUNCH();
  std::vector<int> hc(N);
  int hflag = 0;
  LUM_TRY_CUDA(cudaMemcpyAsync(hc.data(), cnt.p, sizeof(int) * (size_t)N,
                               cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaMemcpyAsync(&hflag, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));
  if (hflag) {
    set_error("Self-interaction: two dipoles of one system share a position");
    return LUM_ERR_INVALID;
  }
  int w = 0;
  for (int v : hc) w = std::max(w, v);
  g.ell_w = w;
  if (w == 0) {
    near_j.release();
    fcd64.release();
    fcd32.release();
    g.near_j = nullptr;
    g.fcd64 = nullptr;
    g.fcd32 = nullptr;
    return LUM_OK;
  }
  LUM_TRY(near_j.alloc(sizeof(int) * (size_t)w * N));
  LUM_TRY_CUDA(cudaMemsetAsync(near_j.p, 0xff, near_j.bytes, st));
  batch_near_scan<true><<<blocks, 256, 0, st>>>(g, use_fcd, nullptr, w, near_j.as<int>(),
                                                flag.as<int>());
  LUM_CHECK_LAUNCH();
  g.near_j = near_j.as<int>();
  LUM_TRY(fcd64.alloc(sizeof(double2) * 9 * (size_t)w * N));
  LUM_TRY(fcd32.alloc(sizeof(float2) * 9 * (size_t)w * N));
  const size_t total = (size_t)w * N;
  batch_fcd_table<<<(unsigned)((total + 127) / 128), 128, 0, st>>>(g, fcd64.as<double2>(),
                                                                   fcd32.as<float2>());
  LUM_CHECK_LAUNCH();
  g.fcd64 = fcd64.as<double2>();
  g.fcd32 = fcd32.as<float2>();
  // the counts and flag buffers are freed on return: finish their users first
  LUM_TRY_CUDA(cudaStreamSynchronize(st));
  return LUM_OK;
}

// Builds of the batched symmetric kernel (g.sym32 = 1 + index): 2 rows per
// thread at 2 CTAs per SM, 4 rows per thread at 4 CTAs per SM, and 4 rows
// with the step loop unrolled (4 CTAs by two, 3 CTAs by four).
template <int MINB, int RP, int UNR = 1>
static void batch_sym_launch_t(const BatchGeom& g, const double2* x, const BatchQueue& q,
                               const BatchFlags* flags, int skip_mode, float2* slots,
                               cudaStream_t st) {
#define LUM_BSYM(F, L)                                                                       \
  batch_pairs_f32_sym<F, L, MINB, RP, UNR><<<q.grid, SymShape<RP>::kThreads, 0, st>>>(       \
      g, x, q.items.as<int4>(), q.nitems, q.counters.as<unsigned>(), flags, skip_mode, slots)
  if (g.fast && g.lofree)
    LUM_BSYM(true, true);
  else if (g.fast)
    LUM_BSYM(true, false);
  else if (g.lofree)
    LUM_BSYM(false, true);
  else
    LUM_BSYM(false, false);
#undef LUM_BSYM
}

template <int MINB, int RP, int UNR = 1>
static int batch_sym_occupancy_t(const BatchGeom& g) {
  int occ = 1;
  if (g.fast && g.lofree)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_pairs_f32_sym<true, true, MINB, RP, UNR>,
                                                  SymShape<RP>::kThreads, 0);
  else if (g.fast)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_pairs_f32_sym<true, false, MINB, RP, UNR>,
                                                  SymShape<RP>::kThreads, 0);
  else if (g.lofree)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_pairs_f32_sym<false, true, MINB, RP, UNR>,
                                                  SymShape<RP>::kThreads, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &occ, batch_pairs_f32_sym<false, false, MINB, RP, UNR>, SymShape<RP>::kThreads, 0);
  return std::max(1, occ);
}

namespace {
struct BatchSymVariant {
  const char* name;
  void (*launch)(const BatchGeom&, const double2*, const BatchQueue&, const BatchFlags*, int,
                 float2*, cudaStream_t);
  int (*occupancy)(const BatchGeom&);
};
const BatchSymVariant kBatchSym[] = {
    {"batch_sym_rows2_minb2", batch_sym_launch_t<2, 1>, batch_sym_occupancy_t<2, 1>},
    {"batch_sym_rows4_minb4", batch_sym_launch_t<4, 2>, batch_sym_occupancy_t<4, 2>},
    {"batch_sym_rows4_minb4_unroll2", batch_sym_launch_t<4, 2, 2>,
     batch_sym_occupancy_t<4, 2, 2>},
    {"batch_sym_rows4_minb3_unroll4", batch_sym_launch_t<3, 2, 4>,
     batch_sym_occupancy_t<3, 2, 4>},
};
constexpr int kNumBatchSym = sizeof(kBatchSym) / sizeof(kBatchSym[0]);
}  // namespace

int batch_sym_variants() { return kNumBatchSym; }
const char* batch_sym_name(int v) {
  return (v >= 1 && v <= kNumBatchSym) ? kBatchSym[v - 1].name : "none";
}
int batch_sym_occupancy(const BatchGeom& g, int v) {
  return kBatchSym[std::min(std::max(v, 1), kNumBatchSym) - 1].occupancy(g);
}

static_assert(kSymRows == kBatchSymRows, "one superblock size for the batch and its kernels");

// The FP64 sin / cos table of this file's kernels, for callers outside it
// (a cluster batch has no OtfOperator).
lum_status otf_sincos_ready() { return sincos_table_ready(); }

// Work list of the symmetric scheme: every superblock pair (I <= J) of every
// system, ordered by decreasing cost (diagonal pairs count half).
lum_status batch_queue_sym(const std::vector<int>& off, int slots, BatchQueue& q,
                           std::vector<int>& nb, cudaStream_t st) {
  const int K = (int)off.size() - 1;
  nb.assign(K, 1);
  struct It {
    long cost;
    int s, I, J;
  };
  std::vector<It> list;
  for (int s = 0; s < K; ++s) {
    const int n = off[s + 1] - off[s];
    nb[s] = (n + kSymRows - 1) / kSymRows;
    for (int I = 0; I < nb[s]; ++I)
      for (int J = I; J < nb[s]; ++J) {
        const long ri = std::min(kSymRows, n - I * kSymRows);
        const long cj = std::min(kSymRows, n - J * kSymRows);
        list.push_back({I == J ? ri * ri / 2 : ri * cj, s, I, J});
      }
  }
  std::stable_sort(list.begin(), list.end(), [](const It& a, const It& b) { return a.cost > b.cost; });
  std::vector<int4> items(list.size());
  for (size_t t = 0; t < list.size(); ++t)
    items[t] = make_int4(list[t].s, list[t].I, list[t].J, 0);
  q.nitems = (int)items.size();
  q.grid = std::max(1, std::min(q.nitems, slots));
  LUM_TRY(q.items.alloc(sizeof(int4) * items.size()));
  LUM_TRY(q.counters.alloc(2 * sizeof(unsigned)));
  LUM_TRY_CUDA(cudaMemcpyAsync(q.items.p, items.data(), q.items.bytes, cudaMemcpyHostToDevice, st));
  LUM_TRY_CUDA(cudaMemsetAsync(q.counters.p, 0, q.counters.bytes, st));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));  // the host item list is freed on return
  return LUM_OK;
}

int batch_occupancy(const BatchGeom& g, int precision) {
  int occ = 1;
  if (precision == LUM_FP32) {
#define LUM_BATCH_OCC(F, L)                                                                  \
  (g.minb32 == 4                                                                           \
       ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_pairs_f32<F, L, 4>,      \
                                                       kOtfBlock, 0)                       \
       : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_pairs_f32<F, L, 6>,      \
                                                       kOtfBlock, 0))
    if (g.fast && g.lofree)
      LUM_BATCH_OCC(true, true);
    else if (g.fast)
      LUM_BATCH_OCC(true, false);
    else if (g.lofree)
      LUM_BATCH_OCC(false, true);
    else
      LUM_BATCH_OCC(false, false);
#undef LUM_BATCH_OCC
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_pairs_f64, kOtfBlock, 0);
  }
  return std::max(1, occ);
}

// Work list for one precision.  Rows per item: 256 (FP32) or 128 (FP64).
// Every system is split into source chunks of about 512 dipoles, so that a
// large system still spreads over many CTAs once the systems around it have
// converged; a batch whose row tiles alone leave the persistent grid short
// of four items per slot is split further.
lum_status batch_queue(int precision, const std::vector<int>& off, int slots, BatchQueue& q,
                       std::vector<int>& ns, std::vector<int>& chunk, cudaStream_t st) {
  const int K = (int)off.size() - 1;
  const int rows = (precision == LUM_FP32) ? 2 * kOtfBlock : kOtfBlock;
  long tiles = 0;
  for (int s = 0; s < K; ++s) tiles += (off[s + 1] - off[s] + rows - 1) / rows;
  const long want = 4L * slots;
  const int split = tiles >= want ? 1 : (int)std::min<long>(16, (want + tiles - 1) / tiles);
  constexpr int kChunk = 512;
  ns.assign(K, 1);
  chunk.assign(K, kOtfBlock);
  struct It {
    long cost;
    int s, r, p;
  };
  std::vector<It> list;
  for (int s = 0; s < K; ++s) {
    const int n = off[s + 1] - off[s];
    const int sp = std::max(1, std::min(std::min(16, std::max(split, (n + kChunk - 1) / kChunk)),
                                        (n + 2 * kOtfBlock - 1) / (2 * kOtfBlock)));
    const int c = ((n + sp - 1) / sp + kOtfBlock - 1) / kOtfBlock * kOtfBlock;
    ns[s] = (n + c - 1) / c;
    chunk[s] = c;
    for (int r = 0; r < n; r += rows)
      for (int p = 0; p < ns[s]; ++p)
        list.push_back({(long)std::min(rows, n - r) * std::min(c, n - p * c), s, r, p});
  }
  std::stable_sort(list.begin(), list.end(), [](const It& a, const It& b) { return a.cost > b.cost; });
  std::vector<int4> items(list.size());
  for (size_t t = 0; t < list.size(); ++t) items[t] = make_int4(list[t].s, list[t].r, list[t].p, 0);
  q.nitems = (int)items.size();
  q.grid = std::max(1, std::min(q.nitems, slots));
  LUM_TRY(q.items.alloc(sizeof(int4) * items.size()));
  LUM_TRY(q.counters.alloc(2 * sizeof(unsigned)));
  LUM_TRY_CUDA(cudaMemcpyAsync(q.items.p, items.data(), q.items.bytes, cudaMemcpyHostToDevice, st));
  LUM_TRY_CUDA(cudaMemsetAsync(q.counters.p, 0, q.counters.bytes, st));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));  // the host item list is freed on return
  return LUM_OK;
}

lum_status batch_apply(const BatchGeom& g, int precision, const double2* x, double2* y,
                       void* partial, BatchQueue& q, const BatchFlags* flags, int skip_mode,
                       cudaStream_t st) {
  const int epi_blocks = (int)(((size_t)g.N * kEpiTPR + 255) / 256);
  const int4* items = q.items.as<int4>();
  unsigned* cnt = q.counters.as<unsigned>();
  if (precision == LUM_FP32 && g.sym32 && g.qsym) {
    float2* part = static_cast<float2*>(partial);
    kBatchSym[std::min(g.sym32, kNumBatchSym) - 1].launch(g, x, *g.qsym, flags, skip_mode, part,
                                                           st);
    LUM_CHECK_LAUNCH();
    batch_epilogue<float2, float2><<<epi_blocks, 256, 0, st>>>(g, x, part, g.sys_nb, g.fcd32,
                                                               flags, skip_mode, y);
    LUM_CHECK_LAUNCH();
    return LUM_OK;
  }
  if (precision == LUM_FP32) {
    float2* part = static_cast<float2*>(partial);
#define LUM_BATCH_F32(F, L)                                                                 \
  do {                                                                                       \
    if (g.minb32 == 4)                                                                       \
      batch_pairs_f32<F, L, 4><<<q.grid, kOtfBlock, 0, st>>>(g, x, items, q.nitems, cnt,     \
                                                             flags, skip_mode, part);        \
    else                                                                                     \
      batch_pairs_f32<F, L, 6><<<q.grid, kOtfBlock, 0, st>>>(g, x, items, q.nitems, cnt,     \
                                                             flags, skip_mode, part);        \
  } while (0)
    if (g.fast && g.lofree)
      LUM_BATCH_F32(true, true);
    else if (g.fast)
      LUM_BATCH_F32(true, false);
    else if (g.lofree)
      LUM_BATCH_F32(false, true);
    else
      LUM_BATCH_F32(false, false);
#undef LUM_BATCH_F32
    LUM_CHECK_LAUNCH();
    batch_epilogue<float2, float2><<<epi_blocks, 256, 0, st>>>(g, x, part, g.sys_ns32, g.fcd32,
                                                               flags, skip_mode, y);
    LUM_CHECK_LAUNCH();
    return LUM_OK;
  }
  double2* part = static_cast<double2*>(partial);
  batch_pairs_f64<<<q.grid, kOtfBlock, 0, st>>>(g, x, items, q.nitems, cnt, flags, skip_mode,
                                                part);
  LUM_CHECK_LAUNCH();
  batch_epilogue<double2, double2><<<epi_blocks, 256, 0, st>>>(g, x, part, g.sys_ns64, g.fcd64,
                                                               flags, skip_mode, y);
  LUM_CHECK_LAUNCH();
  return LUM_OK;
}

}  // namespace lum
