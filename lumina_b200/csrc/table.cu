// table.cu -- periodic (Ewald) operator on a dipole lattice.
//
// With a lattice set, the reference evaluates EwaldGreens::evaluate for every
// ordered pair in every matvec (assembly.rs:244-250): 121 real-space plus 121
// spectral terms per pair at truncation 5/5, and again for the substrate
// image (:283-284).  On a dipole lattice (positions o + d*(ia, ib, ic)) the
// displacement r_i - r_j only takes (2A-1)(2B-1)(2C-1) values, and the image
// displacement r_i - r~_j = (d da, d db, z_i + z_j - 2 z0) only
// (2A-1)(2B-1)(2C-1) more.  Both periodic tensors are tabulated once per
// wavelength / Bloch vector in FP64 (real and reciprocal sums accumulated in
// FP64, an FP32 copy for the FP32 operator), and the matvec becomes a table
// gather:
//   partial_i += sum_j T[ia-ja, ib-jb, ic-jc] x_j + sum_j T~[ia-ja, ib-jb, ic+jc] (m o x_j)
// with m = (-r, -r, +r) and the self term (i == j) included, as the
// reference's periodic branch does.  The epilogue (otf.cu) adds alpha^-1 x.
//
// The periodic tensor is symmetric, so an entry holds its six distinct
// components (xx xy xz yy yz zz; kSym below maps (p, q) to a slot): an FP32
// entry is three 16-byte loads, an FP64 entry six.  The tables are O(N) in
// size and stay L2-resident.
#include "lumina_internal.cuh"
#include "device_physics.cuh"

#include <algorithm>
#include <cmath>
#include <type_traits>

namespace lum {

constexpr int kTabBlock = 128;
// The periodic tensor (like the point tensor) is symmetric, so an entry holds
// its six distinct components xx xy xz yy yz zz: 48 B in FP32 (three 16-byte
// loads), 96 B in FP64.  kSym[p][q] is the slot of component (p, q).
constexpr int kEntry = 6;
__device__ __constant__ int kSym[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};

__global__ void tab_build(int count, int Db, int Dc, int oa, int ob, int oc, double d,
                          int image, double zbase, LatticeDev L,
                          const double4* __restrict__ lreal, const double4* __restrict__ lrecip,
                          double kb0, double kb1, double kb2, double k,
                          double2* __restrict__ t64, float2* __restrict__ t32) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  const int c = e % Dc;
  const int b = (e / Dc) % Db;
  const int a = e / (Dc * Db);
  const double rx = (a - oa) * d, ry = (b - ob) * d;
  // direct: rz = (c - oc) d; image: rz = z_i + z_j - 2 z0 = zbase + c d
  const double rz = image ? zbase + c * d : (c - oc) * d;
  double2 g[9];
  const double kb[3] = {kb0, kb1, kb2};
  if (image && rx * rx + ry * ry + rz * rz < 1e-20) {
    for (int q = 0; q < 9; ++q) g[q] = make_double2(0.0, 0.0);  // assembly.rs:281-282
  } else {
    ewald_tensor(L, lreal, lrecip, rx, ry, rz, kb, k, g);
  }
  const int upper[6] = {0, 1, 2, 4, 5, 8};
  for (int q = 0; q < kEntry; ++q) {
    const double2 v = g[upper[q]];
    t64[(size_t)e * kEntry + q] = v;
    t32[(size_t)e * kEntry + q] = make_float2((float)v.x, (float)v.y);
  }
}

// The six components of an entry in registers (FP32: three 16-byte loads).
template <typename T2>
__device__ __forceinline__ void tab_load(const T2* __restrict__ t, T2 c[6]);
template <>
__device__ __forceinline__ void tab_load<float2>(const float2* __restrict__ t, float2 c[6]) {
  const float4* t4 = reinterpret_cast<const float4*>(t);
#pragma unroll
  for (int h = 0; h < 3; ++h) {
    const float4 v = __ldg(t4 + h);
    c[2 * h] = make_float2(v.x, v.y);
    c[2 * h + 1] = make_float2(v.z, v.w);
  }
}
template <>
__device__ __forceinline__ void tab_load<double2>(const double2* __restrict__ t, double2 c[6]) {
#pragma unroll
  for (int h = 0; h < 6; ++h) c[h] = __ldg(t + h);
}

template <typename R> struct C2;
template <> struct C2<float> {
  typedef float2 T;
  __device__ static float2 mk(double a, double b) { return make_float2((float)a, (float)b); }
};
template <> struct C2<double> {
  typedef double2 T;
  __device__ static double2 mk(double a, double b) { return make_double2(a, b); }
};

// thread per observer dipole, the source range split over grid.y
template <typename R, bool IMG>
__global__ void __launch_bounds__(kTabBlock)
tab_pairs(int n, const int4* __restrict__ lidx, const double2* __restrict__ x,
          const typename C2<R>::T* __restrict__ tab, const typename C2<R>::T* __restrict__ img,
          int Db, int Dc, int oa, int ob, int oc, int Dcs, double2 m0, double2 m1, double2 m2,
          int chunk, typename C2<R>::T* __restrict__ partial, const int* __restrict__ skip) {
  typedef typename C2<R>::T T2;
  if (skip && *skip) return;
  __shared__ int4 sI[kTabBlock];
  __shared__ T2 sX[3 * kTabBlock];
  __shared__ T2 sM[3 * kTabBlock];
  const int tid = threadIdx.x;
  const int i = blockIdx.x * kTabBlock + tid;
  const int4 li = lidx[min(i, n - 1)];
  R acc[6] = {0, 0, 0, 0, 0, 0};
  const int j_begin = blockIdx.y * chunk;
  const int j_end = min(n, j_begin + chunk);
  for (int jt = j_begin; jt < j_end; jt += kTabBlock) {
    const int cnt = min(kTabBlock, j_end - jt);
    __syncthreads();
    if (tid < cnt) {
      const int j = jt + tid;
      sI[tid] = lidx[j];
      const double2 a = x[3 * j], b = x[3 * j + 1], c = x[3 * j + 2];
      sX[3 * tid] = C2<R>::mk(a.x, a.y);
      sX[3 * tid + 1] = C2<R>::mk(b.x, b.y);
      sX[3 * tid + 2] = C2<R>::mk(c.x, c.y);
      if (IMG) {  // m_b x_b, m = (-r, -r, +r)
        sM[3 * tid] = C2<R>::mk(m0.x * a.x - m0.y * a.y, m0.x * a.y + m0.y * a.x);
        sM[3 * tid + 1] = C2<R>::mk(m1.x * b.x - m1.y * b.y, m1.x * b.y + m1.y * b.x);
        sM[3 * tid + 2] = C2<R>::mk(m2.x * c.x - m2.y * c.y, m2.x * c.y + m2.y * c.x);
      }
    }
    __syncthreads();
    for (int jj = 0; jj < cnt; ++jj) {
      const int4 lj = sI[jj];
      const int ab = ((li.x - lj.x + oa) * Db + (li.y - lj.y + ob));
      T2 c[6];
      tab_load<T2>(tab + ((size_t)ab * Dc + (li.z - lj.z + oc)) * kEntry, c);
      constexpr int sym[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
#pragma unroll
      for (int p = 0; p < 3; ++p)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const T2 g = c[sym[p][q]];
          const T2 xv = sX[3 * jj + q];
          acc[2 * p] += g.x * xv.x - g.y * xv.y;
          acc[2 * p + 1] += g.x * xv.y + g.y * xv.x;
        }
      if (IMG) {
        tab_load<T2>(img + ((size_t)ab * Dcs + (li.z + lj.z)) * kEntry, c);
#pragma unroll
        for (int p = 0; p < 3; ++p)
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            const T2 g = c[sym[p][q]];
            const T2 xv = sM[3 * jj + q];
            acc[2 * p] += g.x * xv.x - g.y * xv.y;
            acc[2 * p + 1] += g.x * xv.y + g.y * xv.x;
          }
      }
    }
  }
  if (i < n) {
    T2* out = partial + (size_t)blockIdx.y * (3 * (size_t)n);
    out[3 * i + 0] = C2<R>::mk(acc[0], acc[1]);
    out[3 * i + 1] = C2<R>::mk(acc[2], acc[3]);
    out[3 * i + 2] = C2<R>::mk(acc[4], acc[5]);
  }
}

int table_split(int n);

// Lattice test: every position equals org + d * integer within 1e-9 d.
lum_status OtfOperator::table_detect(cudaStream_t st) {
  table_ok = 0;
  if (n <= 0) return LUM_OK;
  double lo[3] = {1e300, 1e300, 1e300};
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) lo[c] = std::min(lo[c], host_pos[4 * (size_t)i + c]);
  // candidate spacing: the cell size, else the smallest positive axis step
  std::vector<double> cand;
  if (cell > 0.0) cand.push_back(cell);
  double step = 1e300;
  for (int i = 1; i < n && i < 4096; ++i)
    for (int c = 0; c < 3; ++c) {
      double dlt = std::fabs(host_pos[4 * (size_t)i + c] - host_pos[c]);
      if (dlt > 1e-9) step = std::min(step, dlt);
    }
  if (step < 1e300) cand.push_back(step);
  for (double d : cand) {
    std::vector<int> idx((size_t)4 * n, 0);
    int mx[3] = {0, 0, 0};
    bool ok = true;
    for (int i = 0; i < n && ok; ++i)
      for (int c = 0; c < 3; ++c) {
        const double u = (host_pos[4 * (size_t)i + c] - lo[c]) / d;
        const double r = std::nearbyint(u);
        if (std::fabs(u - r) > 1e-9 || r > 1e6) {
          ok = false;
          break;
        }
        idx[4 * (size_t)i + c] = (int)r;
        mx[c] = std::max(mx[c], (int)r);
      }
    if (!ok) continue;
    const double entries = (2.0 * mx[0] + 1) * (2.0 * mx[1] + 1) * (2.0 * mx[2] + 1);
    if (entries > 2.0e7) return LUM_OK;  // table would exceed ~3 GB: per-pair path
    lat_d = d;
    for (int c = 0; c < 3; ++c) {
      lat_org[c] = lo[c];
      tdim[c] = 2 * mx[c] + 1;
    }
    tsdim = 2 * mx[2] + 1;
    LUM_TRY(lidx.alloc(sizeof(int) * idx.size()));
    LUM_TRY_CUDA(cudaMemcpyAsync(lidx.p, idx.data(), lidx.bytes, cudaMemcpyHostToDevice, st));
    nsplit_tab = table_split(n);
    table_ok = 1;
    return LUM_OK;
  }
  return LUM_OK;
}

lum_status OtfOperator::table_build(cudaStream_t st) {
  const size_t count = (size_t)tdim[0] * tdim[1] * tdim[2];
  const size_t scount = (size_t)tdim[0] * tdim[1] * tsdim;
  if (!tab64.p) {
    LUM_TRY(tab64.alloc(sizeof(double2) * kEntry * count));
    LUM_TRY(tab32.alloc(sizeof(float2) * kEntry * count));
  }
  const int oa = tdim[0] / 2, ob = tdim[1] / 2, oc = tdim[2] / 2;
  tab_build<<<(unsigned)((count + 127) / 128), 128, 0, st>>>(
      (int)count, tdim[1], tdim[2], oa, ob, oc, lat_d, 0, 0.0, latdev, lat_real.as<double4>(),
      lat_recip.as<double4>(), kbloch[0], kbloch[1], kbloch[2], k, tab64.as<double2>(),
      tab32.as<float2>());
  LUM_CHECK_LAUNCH();
  if (has_substrate) {
    if (!img64.p) {
      LUM_TRY(img64.alloc(sizeof(double2) * kEntry * scount));
      LUM_TRY(img32.alloc(sizeof(float2) * kEntry * scount));
    }
    const double zbase = 2.0 * lat_org[2] - 2.0 * substrate.z_interface;
    tab_build<<<(unsigned)((scount + 127) / 128), 128, 0, st>>>(
        (int)scount, tdim[1], tsdim, oa, ob, 0, lat_d, 1, zbase, latdev, lat_real.as<double4>(),
        lat_recip.as<double4>(), kbloch[0], kbloch[1], kbloch[2], k, img64.as<double2>(),
        img32.as<float2>());
    LUM_CHECK_LAUNCH();
  }
  return LUM_OK;
}

lum_status OtfOperator::table_apply(int precision, const double2* x, double2* part_d,
                                    cudaStream_t st, const int* skip, int* nparts) {
  const int ntiles = (n + kTabBlock - 1) / kTabBlock;
  const int ns = nsplit_tab;
  const int chunk = ((ntiles + ns - 1) / ns) * kTabBlock;
  dim3 grid(ntiles, ns);
  const int oa = tdim[0] / 2, ob = tdim[1] / 2, oc = tdim[2] / 2;
  const double2 rr = make_double2(substrate.refl_re, substrate.refl_im);
  const double2 mneg = make_double2(-rr.x, -rr.y);
  const int4* li = lidx.as<int4>();
  if (precision == LUM_FP32) {
    float2* part = reinterpret_cast<float2*>(part_d);
    if (has_substrate)
      tab_pairs<float, true><<<grid, kTabBlock, 0, st>>>(
          n, li, x, tab32.as<float2>(), img32.as<float2>(), tdim[1], tdim[2], oa, ob, oc, tsdim,
          mneg, mneg, rr, chunk, part, skip);
    else
      tab_pairs<float, false><<<grid, kTabBlock, 0, st>>>(
          n, li, x, tab32.as<float2>(), nullptr, tdim[1], tdim[2], oa, ob, oc, tsdim, mneg, mneg,
          rr, chunk, part, skip);
  } else {
    if (has_substrate)
      tab_pairs<double, true><<<grid, kTabBlock, 0, st>>>(
          n, li, x, tab64.as<double2>(), img64.as<double2>(), tdim[1], tdim[2], oa, ob, oc,
          tsdim, mneg, mneg, rr, chunk, part_d, skip);
    else
      tab_pairs<double, false><<<grid, kTabBlock, 0, st>>>(
          n, li, x, tab64.as<double2>(), nullptr, tdim[1], tdim[2], oa, ob, oc, tsdim, mneg, mneg,
          rr, chunk, part_d, skip);
  }
  LUM_CHECK_LAUNCH();
  *nparts = ns;
  return LUM_OK;
}

// Dense assembly from the tables: block (i, j) = alpha_i^-1 delta_ij - T - T~ m
// (assembly.rs:45-175 with the periodic branch), one thread per pair.
template <typename T2>
__global__ void __launch_bounds__(128)
assemble_table(int n, const int4* __restrict__ lidx, const double2* __restrict__ inv_alpha,
               const double2* __restrict__ tab, const double2* __restrict__ img, int Db, int Dc,
               int oa, int ob, int oc, int Dcs, double2 rr, size_t ld, T2* __restrict__ A) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * n) return;
  const int i = (int)(idx / n), j = (int)(idx % n);
  const int4 li = lidx[i], lj = lidx[j];
  const int ab = (li.x - lj.x + oa) * Db + (li.y - lj.y + ob);
  const double2* t = tab + ((size_t)ab * Dc + (li.z - lj.z + oc)) * kEntry;
  const double2* s = img ? img + ((size_t)ab * Dcs + (li.z + lj.z)) * kEntry : nullptr;
  const double2 m[3] = {make_double2(-rr.x, -rr.y), make_double2(-rr.x, -rr.y), rr};
  for (int p = 0; p < 3; ++p)
    for (int q = 0; q < 3; ++q) {
      double2 v = make_double2(0.0, 0.0);
      if (i == j) v = inv_alpha[(size_t)(3 * p + q) * n + i];
      const double2 g = t[kSym[p][q]];
      v.x -= g.x;
      v.y -= g.y;
      if (s) {
        const double2 h = s[kSym[p][q]];
        v.x -= m[q].x * h.x - m[q].y * h.y;
        v.y -= m[q].x * h.y + m[q].y * h.x;
      }
      A[(3 * (size_t)i + p) * ld + 3 * (size_t)j + q] = C2<typename std::conditional<
          sizeof(T2) == sizeof(float2), float, double>::type>::mk(v.x, v.y);
    }
}

lum_status assemble_from_table(const OtfOperator& g, int precision, void* A, size_t ld,
                               cudaStream_t st) {
  const long long npairs = (long long)g.n * g.n;
  const unsigned blocks = (unsigned)((npairs + 127) / 128);
  const int oa = g.tdim[0] / 2, ob = g.tdim[1] / 2, oc = g.tdim[2] / 2;
  const double2* img = g.has_substrate ? g.img64.as<double2>() : nullptr;
  const double2 rr = make_double2(g.substrate.refl_re, g.substrate.refl_im);
  if (precision == LUM_FP32)
    assemble_table<float2><<<blocks, 128, 0, st>>>(
        g.n, g.lidx.as<int4>(), g.inv_alpha.as<double2>(), g.tab64.as<double2>(), img, g.tdim[1],
        g.tdim[2], oa, ob, oc, g.tsdim, rr, ld, static_cast<float2*>(A));
  else
    assemble_table<double2><<<blocks, 128, 0, st>>>(
        g.n, g.lidx.as<int4>(), g.inv_alpha.as<double2>(), g.tab64.as<double2>(), img, g.tdim[1],
        g.tdim[2], oa, ob, oc, g.tsdim, rr, ld, static_cast<double2*>(A));
  LUM_CHECK_LAUNCH();
  return LUM_OK;
}

int table_split(int n) {
  int dev = 0, sms = 148, occ = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, tab_pairs<float, true>, kTabBlock, 0);
  const int ntiles = (n + kTabBlock - 1) / kTabBlock;
  const int want = std::max(1, 2 * std::max(1, occ) * sms);
  return std::max(1, std::min(ntiles, std::min(64, (want + ntiles - 1) / ntiles)));
}

}  // namespace lum
