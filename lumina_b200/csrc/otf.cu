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

namespace lum {

constexpr int kOtfBlock = 128;

// ---------------------------------------------------------------------------
// FP32 dense pair kernel
// ---------------------------------------------------------------------------
// Source tile entry: P0 = (hx, hy, hz, lx), P1 = (ly, lz, x0r, x0i),
// P2 = (x1r, x1i, x2r, x2i)  -- 3 x LDS.128 per source.
template <bool FAST, bool IMAGE, int R>
__global__ void __launch_bounds__(kOtfBlock)
otf_pairs_f32(int n, const float4* __restrict__ obs_hi, const float4* __restrict__ obs_lo,
              const float4* __restrict__ src_hi, const float4* __restrict__ src_lo,
              const double2* __restrict__ x, float2 m0, float2 m1, float2 m2, float k,
              float inv_k, float s0, int chunk, float2* __restrict__ partial) {
  __shared__ float4 sP0[kOtfBlock], sP1[kOtfBlock], sP2[kOtfBlock];
  const int tid = threadIdx.x;
  int irow[R];
  float ohx[R], ohy[R], ohz[R], olx[R], oly[R], olz[R];
  float acc[R][6];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    int i = blockIdx.x * (kOtfBlock * R) + r * kOtfBlock + tid;
    irow[r] = i;
    int ic = min(i, n - 1);
    float4 h = obs_hi[ic], l = obs_lo[ic];
    ohx[r] = h.x; ohy[r] = h.y; ohz[r] = h.z;
    olx[r] = l.x; oly[r] = l.y; olz[r] = l.z;
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[r][c] = 0.f;
  }
  const int j_begin = blockIdx.y * chunk;
  const int j_end = min(n, j_begin + chunk);
  for (int jt = j_begin; jt < j_end; jt += kOtfBlock) {
    const int cnt = min(kOtfBlock, j_end - jt);
    __syncthreads();
    if (tid < cnt) {
      const int j = jt + tid;
      float4 h = src_hi[j], l = src_lo[j];
      double2 a = x[3 * j], b = x[3 * j + 1], c = x[3 * j + 2];
      float2 xa = make_float2((float)a.x, (float)a.y);
      float2 xb = make_float2((float)b.x, (float)b.y);
      float2 xc = make_float2((float)c.x, (float)c.y);
      if (IMAGE) {  // x'_b = m_b x_b, m = (-r, -r, +r)  (assembly.rs:288-292)
        xa = make_float2(m0.x * xa.x - m0.y * xa.y, m0.x * xa.y + m0.y * xa.x);
        xb = make_float2(m1.x * xb.x - m1.y * xb.y, m1.x * xb.y + m1.y * xb.x);
        xc = make_float2(m2.x * xc.x - m2.y * xc.y, m2.x * xc.y + m2.y * xc.x);
      }
      sP0[tid] = make_float4(h.x, h.y, h.z, l.x);
      sP1[tid] = make_float4(l.y, l.z, xa.x, xa.y);
      sP2[tid] = make_float4(xb.x, xb.y, xc.x, xc.y);
    }
    __syncthreads();
#pragma unroll 2
    for (int jj = 0; jj < cnt; ++jj) {
      const float4 P0 = sP0[jj], P1 = sP1[jj], P2 = sP2[jj];
      const int j = jt + jj;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        float dx = (ohx[r] - P0.x) + (olx[r] - P0.w);
        float dy = (ohy[r] - P0.y) + (oly[r] - P1.x);
        float dz = (ohz[r] - P0.z) + (olz[r] - P1.y);
        float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        bool skip = IMAGE ? (r2 < 1e-20f) : (j == irow[r]);
        if (skip) r2 = 1.0f;
        float ir = rsqrtf(r2);
        float Rr = r2 * ir;
        float u = ir * inv_k;
        float u2 = u * u;
        float sn, cs;
        if (FAST)
          __sincosf(k * Rr, &sn, &cs);
        else
          sincosf(k * Rr, &sn, &cs);
        float su = skip ? 0.f : s0 * u;
        float pr = su * cs, pi = su * sn;
        float ar = 1.0f - u2;
        float Ar = fmaf(pr, ar, -pi * u), Ai = fmaf(pr, u, pi * ar);
        float br = fmaf(3.0f, u2, -1.0f), bi = -3.0f * u;
        float ir2 = ir * ir;
        float Br = fmaf(pr, br, -pi * bi) * ir2, Bi = fmaf(pr, bi, pi * br) * ir2;
        float dxr = fmaf(dx, P1.z, fmaf(dy, P2.x, dz * P2.z));
        float dxi = fmaf(dx, P1.w, fmaf(dy, P2.y, dz * P2.w));
        float tr = fmaf(Br, dxr, -Bi * dxi), ti = fmaf(Br, dxi, Bi * dxr);
        acc[r][0] = fmaf(tr, dx, fmaf(Ar, P1.z, fmaf(-Ai, P1.w, acc[r][0])));
        acc[r][1] = fmaf(ti, dx, fmaf(Ar, P1.w, fmaf(Ai, P1.z, acc[r][1])));
        acc[r][2] = fmaf(tr, dy, fmaf(Ar, P2.x, fmaf(-Ai, P2.y, acc[r][2])));
        acc[r][3] = fmaf(ti, dy, fmaf(Ar, P2.y, fmaf(Ai, P2.x, acc[r][3])));
        acc[r][4] = fmaf(tr, dz, fmaf(Ar, P2.z, fmaf(-Ai, P2.w, acc[r][4])));
        acc[r][5] = fmaf(ti, dz, fmaf(Ar, P2.w, fmaf(Ai, P2.z, acc[r][5])));
      }
    }
  }
  float2* out = partial + (size_t)blockIdx.y * (3 * (size_t)n);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (irow[r] < n) {
      out[3 * irow[r] + 0] = make_float2(acc[r][0], acc[r][1]);
      out[3 * irow[r] + 1] = make_float2(acc[r][2], acc[r][3]);
      out[3 * irow[r] + 2] = make_float2(acc[r][4], acc[r][5]);
    }
  }
}

// ---------------------------------------------------------------------------
// FP64 dense pair kernel (same decomposition; sources as double4 + 3 double2)
// ---------------------------------------------------------------------------
template <bool IMAGE>
__global__ void __launch_bounds__(kOtfBlock)
otf_pairs_f64(int n, const double4* __restrict__ pos, const double2* __restrict__ x,
              double2 m0, double2 m1, double2 m2, double z_mirror, double k, double inv_k,
              double s0, int chunk, double2* __restrict__ partial) {
  __shared__ double4 sP[kOtfBlock];
  __shared__ double2 sX[3 * kOtfBlock];
  const int tid = threadIdx.x;
  const int i = blockIdx.x * kOtfBlock + tid;
  const double4 ri = pos[min(i, n - 1)];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const int j_begin = blockIdx.y * chunk;
  const int j_end = min(n, j_begin + chunk);
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
      sincos(k * Rr, &sn, &cs);
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
    }
  }
  if (i < n) {
    double2* out = partial + (size_t)blockIdx.y * (3 * (size_t)n);
    out[3 * i + 0] = make_double2(acc[0], acc[1]);
    out[3 * i + 1] = make_double2(acc[2], acc[3]);
    out[3 * i + 2] = make_double2(acc[4], acc[5]);
  }
}

// ---------------------------------------------------------------------------
// Epilogue: y = alpha^-1 x - sum(partials) - sum_near C_ij x_j
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }
__device__ __forceinline__ double2 to_d2(double2 v) { return v; }

template <typename TP, typename TC>
__global__ void __launch_bounds__(256)
otf_epilogue(int n, const double2* __restrict__ x, const double2* __restrict__ inv_alpha,
             const TP* __restrict__ partial, int nparts, int ell_w,
             const int* __restrict__ near_j, const TC* __restrict__ fcd,
             double2* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double2 xi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
  double yr[3], yi[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      double2 m = inv_alpha[(size_t)(3 * a + b) * n + i];
      sr += m.x * xi[b].x - m.y * xi[b].y;
      si += m.x * xi[b].y + m.y * xi[b].x;
    }
    yr[a] = sr;
    yi[a] = si;
  }
  double gr[3] = {0, 0, 0}, gi[3] = {0, 0, 0};
  const size_t stride = 3 * (size_t)n;
  for (int s = 0; s < nparts; ++s) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double2 p = to_d2(partial[s * stride + 3 * i + a]);
      gr[a] += p.x;
      gi[a] += p.y;
    }
  }
  for (int w = 0; w < ell_w; ++w) {
    const int j = near_j[(size_t)w * n + i];
    if (j < 0) break;
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
  for (int a = 0; a < 3; ++a) y[3 * i + a] = make_double2(yr[a] - gr[a], yi[a] - gi[a]);
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
  for (int e = 0; e < 9; ++e) {
    fcd64[((size_t)w * 9 + e) * n + i] = C[e];
    fcd32[((size_t)w * 9 + e) * n + i] = make_float2((float)C[e].x, (float)C[e].y);
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
                double2* __restrict__ partial) {
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

constexpr int kRowsF32 = 2;

}  // namespace

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
  // FCD corrections for this wavelength
  if (ell_w > 0) {
    int total = ell_w * n;
    fcd_table<<<(total + 127) / 128, 128, 0, st>>>(n, ell_w, pos64.as<double4>(),
                                                   near_j.as<int>(), k, cell,
                                                   fcd64.as<double2>(), fcd32.as<float2>());
    LUM_CHECK_LAUNCH();
  }
  fast_trig = (k * extent < 3.0) ? 1 : 0;
  // partial-sum scratch
  if (first) {
    int sms = device_sms();
    int occ32 = 1, occ64 = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ32, otf_pairs_f32<true, false, kRowsF32>,
                                                  kOtfBlock, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ64, otf_pairs_f64<false>, kOtfBlock, 0);
    int ntiles = (n + kOtfBlock - 1) / kOtfBlock;
    int rb32 = (n + kOtfBlock * kRowsF32 - 1) / (kOtfBlock * kRowsF32);
    int rb64 = ntiles;
    nsplit32 = choose_nsplit(rb32, ntiles, std::max(1, occ32), sms);
    nsplit64 = choose_nsplit(rb64, ntiles, std::max(1, occ64), sms);
    int parts = std::max(nsplit32 * 2, nsplit64 * 2 + 0);
    if (has_lattice) parts = std::max(parts, nsplit64);
    size_t bytes = std::max(sizeof(float2) * (size_t)nsplit32 * 2, sizeof(double2) * (size_t)nsplit64 * 2) *
                   3 * (size_t)n;
    (void)parts;
    LUM_TRY(partial.alloc(bytes));
  }
  return LUM_OK;
}

lum_status OtfOperator::apply(int precision, const double2* x, double2* y, cudaStream_t st,
                              cudaEvent_t ev0, cudaEvent_t ev1) {
  const int ntiles = (n + kOtfBlock - 1) / kOtfBlock;
  const double s0 = k * k * k / (4.0 * kPi);
  const int epi_blocks = (n + 255) / 256;
  if (has_lattice) {
    // Ewald path: FP64 pair kernel for either precision.
    const int ns = nsplit64;
    const int chunk = ((n + ns - 1) / ns);
    dim3 grid(ntiles, ns);
    if (ev0) cudaEventRecord(ev0, st);
    otf_pairs_ewald<<<grid, kOtfBlock, 0, st>>>(
        n, pos64.as<double4>(), x, latdev, lat_real.as<double4>(), lat_recip.as<double4>(),
        kbloch[0], kbloch[1], kbloch[2], k, has_substrate, substrate, chunk,
        partial.as<double2>());
    LUM_CHECK_LAUNCH();
    if (ev1) cudaEventRecord(ev1, st);
    otf_epilogue<double2, double2><<<epi_blocks, 256, 0, st>>>(
        n, x, inv_alpha.as<double2>(), partial.as<double2>(), ns, 0, nullptr, nullptr, y);
    LUM_CHECK_LAUNCH();
    return LUM_OK;
  }
  const double2 rr = make_double2(substrate.refl_re, substrate.refl_im);
  if (precision == LUM_FP32) {
    const int ns = nsplit32;
    const int chunk = ((ntiles + ns - 1) / ns) * kOtfBlock;
    const int rb = (n + kOtfBlock * kRowsF32 - 1) / (kOtfBlock * kRowsF32);
    dim3 grid(rb, ns);
    const float kf = (float)k, ikf = (float)(1.0 / k), s0f = (float)s0;
    const float2 one = make_float2(1.f, 0.f);
    float2* part = partial.as<float2>();
    if (ev0) cudaEventRecord(ev0, st);
    if (fast_trig)
      otf_pairs_f32<true, false, kRowsF32><<<grid, kOtfBlock, 0, st>>>(
          n, pos_hi.as<float4>(), pos_lo.as<float4>(), pos_hi.as<float4>(), pos_lo.as<float4>(),
          x, one, one, one, kf, ikf, s0f, chunk, part);
    else
      otf_pairs_f32<false, false, kRowsF32><<<grid, kOtfBlock, 0, st>>>(
          n, pos_hi.as<float4>(), pos_lo.as<float4>(), pos_hi.as<float4>(), pos_lo.as<float4>(),
          x, one, one, one, kf, ikf, s0f, chunk, part);
    LUM_CHECK_LAUNCH();
    if (ev1) cudaEventRecord(ev1, st);
    int nparts = ns;
    if (has_substrate) {
      const float2 mneg = make_float2((float)-rr.x, (float)-rr.y);
      const float2 mpos = make_float2((float)rr.x, (float)rr.y);
      float2* part2 = part + (size_t)ns * 3 * n;
      if (fast_trig)
        otf_pairs_f32<true, true, kRowsF32><<<grid, kOtfBlock, 0, st>>>(
            n, pos_hi.as<float4>(), pos_lo.as<float4>(), img_hi.as<float4>(),
            img_lo.as<float4>(), x, mneg, mneg, mpos, kf, ikf, s0f, chunk, part2);
      else
        otf_pairs_f32<false, true, kRowsF32><<<grid, kOtfBlock, 0, st>>>(
            n, pos_hi.as<float4>(), pos_lo.as<float4>(), img_hi.as<float4>(),
            img_lo.as<float4>(), x, mneg, mneg, mpos, kf, ikf, s0f, chunk, part2);
      LUM_CHECK_LAUNCH();
      nparts = 2 * ns;
    }
    otf_epilogue<float2, float2><<<epi_blocks, 256, 0, st>>>(
        n, x, inv_alpha.as<double2>(), part, nparts, ell_w, near_j.as<int>(),
        fcd32.as<float2>(), y);
    LUM_CHECK_LAUNCH();
    return LUM_OK;
  }
  // FP64
  const int ns = nsplit64;
  const int chunk = ((ntiles + ns - 1) / ns) * kOtfBlock;
  dim3 grid(ntiles, ns);
  const double2 one = make_double2(1.0, 0.0);
  double2* part = partial.as<double2>();
  if (ev0) cudaEventRecord(ev0, st);
  otf_pairs_f64<false><<<grid, kOtfBlock, 0, st>>>(n, pos64.as<double4>(), x, one, one, one, 0.0,
                                                   k, 1.0 / k, s0, chunk, part);
  LUM_CHECK_LAUNCH();
  if (ev1) cudaEventRecord(ev1, st);
  int nparts = ns;
  if (has_substrate) {
    const double2 mneg = make_double2(-rr.x, -rr.y);
    otf_pairs_f64<true><<<grid, kOtfBlock, 0, st>>>(
        n, pos64.as<double4>(), x, mneg, mneg, rr, 2.0 * substrate.z_interface, k, 1.0 / k, s0,
        chunk, part + (size_t)ns * 3 * n);
    LUM_CHECK_LAUNCH();
    nparts = 2 * ns;
  }
  otf_epilogue<double2, double2><<<epi_blocks, 256, 0, st>>>(
      n, x, inv_alpha.as<double2>(), part, nparts, ell_w, near_j.as<int>(),
      fcd64.as<double2>(), y);
  LUM_CHECK_LAUNCH();
  return LUM_OK;
}

}  // namespace lum
