// fft.cu -- block-Toeplitz operator through a 3D FFT convolution.
//
// The reference's FftMatvecPlan (crates/lumina-core/src/solver/cda/
// fft_matvec.rs:77-258) applies A = alpha^-1 - G for dipoles on a full cubic
// grid without FCD: G(r_i - r_j) depends only on the integer displacement,
// so -G x is a convolution, evaluated by embedding the grid in a circulant
// of twice its size (fft_matvec.rs:127-165) and three forward / three
// inverse 3D FFTs per product (fft_matvec.rs:211-258).
//
// Here the same embedding is built on the device, and widened in two ways:
//  * FCD: the filtered tensor of greens.rs:94-167 is also a function of the
//    displacement alone (27-node average over the source cell), so the
//    kernel table holds it for every displacement with |d| <= 2 cell and the
//    point tensor beyond -- the product equals the on-the-fly FCD operator;
//  * any set of lattice nodes: empty nodes carry x = 0 and are not read
//    back, so spheres, cylinders and helices on a cubic lattice qualify, not
//    only full boxes (fft_matvec.rs:63-70 requires a full box).
// Padded dimensions are powers of two >= 2 n - 1 per axis.  The tensor is
// symmetric (greens.rs:34-71), so six kernel spectra are stored.
//
// A planar substrate adds R(r_i, r_j), a function of (x_i - x_j, y_i - y_j,
// z_i + z_j): the Fresnel image tensor G(r_i - rbar_j) with column factors m
// (assembly.rs:129-156, :274-295) or the Sommerfeld G_refl (sommerfeld.rs).
// With c' = -c_j it is a convolution in the z-mirrored coordinate: on the
// circulant, x~(c) = x(-c mod Mz) has the spectrum X(kx, ky, -kz), so the
// reflected term is R^(k) . (m o X)(kx, ky, -kz) -- six more spectra and no
// further FFT.  The table holds R at height sums t = c + c' in [0, 2 n_z - 2]
// and lateral displacements as for G.
//
// FFTs are hand-written: batched Stockham passes (the autosort formulation of
// Govindaraju et al., "High Performance Discrete Fourier Transforms on
// Graphics Processors", SC 2008; radix-4 stages, one radix-2 stage when
// log2 L is odd) along one axis at a time,
// each CTA transforming B lines in shared memory, all three vector
// components in one launch.  Forward passes skip the lines that the zero
// padding keeps empty and mask the padding of the lines they do transform
// (it is never written); inverse passes skip the lines no dipole reads.  The
// first forward pass reads x through the node map and the last inverse pass
// writes y, so no scatter or gather kernel runs (except for single layers).
// FP64 and FP32 variants: the FP32 product (FP32 FFTs against FP32 copies
// of the FP64 kernel spectra) is the refinement inner operator, the FP64
// one the residual operator.
#include "sommerfeld.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace lum {
namespace {

constexpr int kFftThreads = 256;

template <typename R> struct Cx;
template <> struct Cx<float> { using T = float2; };
template <> struct Cx<double> { using T = double2; };

template <typename T2> __device__ __forceinline__ T2 cadd(T2 a, T2 b) {
  T2 r;
  r.x = a.x + b.x;
  r.y = a.y + b.y;
  return r;
}
template <typename T2> __device__ __forceinline__ T2 csub(T2 a, T2 b) {
  T2 r;
  r.x = a.x - b.x;
  r.y = a.y - b.y;
  return r;
}
template <typename T2> __device__ __forceinline__ T2 cmulT(T2 a, T2 b) {
  T2 r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}

// One pass of batched 1D FFTs of length L = 2^log2L.  Line (o, i) starts at
// comp * comp_stride + o * outer_stride + i * inner_stride and its element t
// is at + t * elem_stride; blockIdx.x covers n_outer x ceil(n_inner / B)
// groups of B lines, blockIdx.z the vector component.  tw[q] =
// exp(-2 pi i q / L), q < L/2 (conjugated for the inverse).
// Line I/O of a pass.  mode 0 reads and writes the buffer; mode 1 (the first
// forward pass) reads x through the node map instead of a scattered buffer;
// mode 2 (the last inverse pass) writes y_i = alpha_i^-1 x_i - line / mtot at
// the dipole nodes instead of the buffer.  Elements t >= valid of a line are
// read as zero: the padding of the circulant is never written, only masked.
struct FftIO {
  int mode;
  int valid;
  const int* node_dip;       // [mtot] dipole on each node, -1 if none
  const double2* x;          // [3n]
  const double2* inv_alpha;  // [9][n]
  double2* y;                // [3n]
  int n;
  double scale;              // 1 / mtot
};

template <typename R, bool INV>
__global__ void __launch_bounds__(kFftThreads)
fft_lines(typename Cx<R>::T* __restrict__ data, size_t comp_stride, int L, int B,
          long long elem_stride, int n_outer, long long outer_stride, int n_inner,
          long long inner_stride, const typename Cx<R>::T* __restrict__ tw,
          const int* __restrict__ skip, FftIO io) {
  using T2 = typename Cx<R>::T;
  if (skip && *skip) return;
  extern __shared__ unsigned char fft_smem[];
  const int LP = L + 1;  // padded line pitch: strided fills avoid bank conflicts
  T2* s0 = reinterpret_cast<T2*>(fft_smem);
  T2* s1 = s0 + (size_t)B * LP;
  T2* stw = s1 + (size_t)B * LP;
  const int chunks = (n_inner + B - 1) / B;
  const int outer = blockIdx.x / chunks;
  const int i0 = (blockIdx.x % chunks) * B;
  const int nb = min(B, n_inner - i0);
  if (outer >= n_outer) return;
  const size_t line0 = (size_t)outer * outer_stride + (size_t)i0 * inner_stride;
  const int comp = blockIdx.z;
  T2* base = data + comp * comp_stride + line0;
  const int half = L >> 1;
  for (int q = threadIdx.x; q < half; q += blockDim.x) {
    T2 w = tw[q];
    if (INV) w.y = -w.y;
    stw[q] = w;
  }
  for (int q = threadIdx.x; q < nb * L; q += blockDim.x) {
    int b, t;
    if (elem_stride == 1) {
      t = q % L;
      b = q / L;
    } else {
      b = q % nb;
      t = q / nb;
    }
    const size_t off = (size_t)b * inner_stride + (size_t)t * elem_stride;
    T2 v;
    v.x = 0;
    v.y = 0;
    if (t < io.valid) {
      if (io.mode == 1) {
        const int i = io.node_dip[line0 + off];
        if (i >= 0) {
          const double2 xv = io.x[3 * (size_t)i + comp];
          v.x = (R)xv.x;
          v.y = (R)xv.y;
        }
      } else {
        v = base[off];
      }
    }
    s0[b * LP + t] = v;
  }
  __syncthreads();
  T2* a = s0;
  T2* c = s1;
  // Stockham stages: one radix-2 stage when log2 L is odd, then radix-4
  // stages (each one shared-memory round trip for two radix-2 levels).
  int ns = 1;
  if ((__ffs(L) - 1) & 1) {
    for (int q = threadIdx.x; q < nb * half; q += blockDim.x) {
      const int b = q / half, j = q % half;
      const T2 v0 = a[b * LP + j], v1 = a[b * LP + j + half];
      c[b * LP + 2 * j] = cadd(v0, v1);
      c[b * LP + 2 * j + 1] = csub(v0, v1);
    }
    __syncthreads();
    T2* t = a;
    a = c;
    c = t;
    ns = 2;
  }
  const int quarter = L >> 2;
  for (; ns < L; ns <<= 2) {
    // x_m = a[j + m L/4] w^(m r), w = exp(-+2 pi i / (4 ns)), r = j mod ns;
    // tw index of w^t is t L / (4 ns); indices >= L/2 use w(t + L/2) = -w(t)
    const int step = quarter / ns;
    for (int q = threadIdx.x; q < nb * quarter; q += blockDim.x) {
      const int b = q / quarter, j = q % quarter;
      const int r = j & (ns - 1);
      const T2* ab = a + b * LP + j;
      const T2 x0 = ab[0];
      T2 x1 = ab[quarter], x2 = ab[2 * quarter], x3 = ab[3 * quarter];
      if (r) {
        const int t1 = r * step, t2 = 2 * t1, t3 = 3 * t1;
        x1 = cmulT(x1, stw[t1]);
        x2 = cmulT(x2, stw[t2]);
        T2 w3 = stw[t3 < half ? t3 : t3 - half];
        if (t3 >= half) {
          w3.x = -w3.x;
          w3.y = -w3.y;
        }
        x3 = cmulT(x3, w3);
      }
      // 4-point DFT with kernel exp(-+ i pi m q / 2): -i (forward) or +i (inverse)
      const T2 s02 = cadd(x0, x2), d02 = csub(x0, x2);
      const T2 s13 = cadd(x1, x3), d13 = csub(x1, x3);
      T2 jd13;  // (-i) d13 forward, (+i) d13 inverse
      if (INV) {
        jd13.x = -d13.y;
        jd13.y = d13.x;
      } else {
        jd13.x = d13.y;
        jd13.y = -d13.x;
      }
      T2* cb = c + b * LP + ((j - r) << 2) + r;
      cb[0] = cadd(s02, s13);
      cb[ns] = cadd(d02, jd13);
      cb[2 * ns] = csub(s02, s13);
      cb[3 * ns] = csub(d02, jd13);
    }
    __syncthreads();
    T2* t = a;
    a = c;
    c = t;
  }
  for (int q = threadIdx.x; q < nb * L; q += blockDim.x) {
    int b, t;
    if (elem_stride == 1) {
      t = q % L;
      b = q / L;
    } else {
      b = q % nb;
      t = q / nb;
    }
    const size_t off = (size_t)b * inner_stride + (size_t)t * elem_stride;
    if (io.mode == 2) {
      const int i = io.node_dip[line0 + off];
      if (i >= 0) {
        double sr = 0.0, si = 0.0;
#pragma unroll
        for (int e = 0; e < 3; ++e) {
          const double2 m = io.inv_alpha[(size_t)(3 * comp + e) * io.n + i];
          const double2 xe = io.x[3 * (size_t)i + e];
          sr += m.x * xe.x - m.y * xe.y;
          si += m.x * xe.y + m.y * xe.x;
        }
        const T2 v = a[b * LP + t];
        io.y[3 * (size_t)i + comp] =
            make_double2(sr - (double)v.x * io.scale, si - (double)v.y * io.scale);
      }
    } else {
      base[off] = a[b * LP + t];
    }
  }
}

// buf[c][g] = x[3 node_dip[g] + c] (zero on empty nodes), c < 3.
template <typename R>
__global__ void fft_scatter(size_t mtot, const int* __restrict__ node_dip,
                            const double2* __restrict__ x, typename Cx<R>::T* __restrict__ buf,
                            const int* __restrict__ skip) {
  using T2 = typename Cx<R>::T;
  if (skip && *skip) return;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < mtot;
       g += (size_t)gridDim.x * blockDim.x) {
    const int i = node_dip[g];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T2 v;
      v.x = 0;
      v.y = 0;
      if (i >= 0) {
        const double2 xv = x[3 * (size_t)i + c];
        v.x = (R)xv.x;
        v.y = (R)xv.y;
      }
      buf[c * mtot + g] = v;
    }
  }
}

// Y_a = sum_b K_ab X_b at every frequency; K symmetric: xx xy xz yy yz zz.
template <typename R>
__global__ void fft_spectral_product(size_t mtot, const typename Cx<R>::T* __restrict__ kern,
                                     typename Cx<R>::T* __restrict__ buf,
                                     const int* __restrict__ skip) {
  using T2 = typename Cx<R>::T;
  if (skip && *skip) return;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < mtot;
       g += (size_t)gridDim.x * blockDim.x) {
    const T2 x0 = buf[g], x1 = buf[mtot + g], x2 = buf[2 * mtot + g];
    const T2 kxx = kern[g], kxy = kern[mtot + g], kxz = kern[2 * mtot + g];
    const T2 kyy = kern[3 * mtot + g], kyz = kern[4 * mtot + g], kzz = kern[5 * mtot + g];
    buf[g] = cadd(cadd(cmulT(kxx, x0), cmulT(kxy, x1)), cmulT(kxz, x2));
    buf[mtot + g] = cadd(cadd(cmulT(kxy, x0), cmulT(kyy, x1)), cmulT(kyz, x2));
    buf[2 * mtot + g] = cadd(cadd(cmulT(kxz, x0), cmulT(kyz, x1)), cmulT(kzz, x2));
  }
}

// With a substrate: Y(k) = K(k) X(k) + R(k) (m o X)(kx, ky, -kz).  One thread
// takes the frequency pair (kz, Mz - kz) of a (kx, ky) line, so both inputs
// are read before either output is written.
template <typename R>
__global__ void fft_spectral_product_refl(int lines, int mz, size_t mtot,
                                          const typename Cx<R>::T* __restrict__ kern,
                                          const typename Cx<R>::T* __restrict__ refl,
                                          typename Cx<R>::T m0, typename Cx<R>::T m1,
                                          typename Cx<R>::T m2,
                                          typename Cx<R>::T* __restrict__ buf,
                                          const int* __restrict__ skip) {
  using T2 = typename Cx<R>::T;
  if (skip && *skip) return;
  const int half = mz / 2 + 1;
  const size_t count = (size_t)lines * half;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < count;
       q += (size_t)gridDim.x * blockDim.x) {
    const size_t line = q / half;
    const int nz = (int)(q % half);
    const int nz2 = (mz - nz) % mz;
    const size_t g[2] = {line * mz + nz, line * mz + nz2};
    const int cnt = (nz2 == nz) ? 1 : 2;
    T2 X[2][3];
    for (int h = 0; h < cnt; ++h)
      for (int c = 0; c < 3; ++c) X[h][c] = buf[c * mtot + g[h]];
    for (int h = 0; h < cnt; ++h) {
      const size_t gg = g[h];
      const int o = (cnt == 2) ? 1 - h : 0;   // the mirrored frequency
      const T2 xm[3] = {cmulT(m0, X[o][0]), cmulT(m1, X[o][1]), cmulT(m2, X[o][2])};
      const T2 kxx = kern[gg], kxy = kern[mtot + gg], kxz = kern[2 * mtot + gg];
      const T2 kyy = kern[3 * mtot + gg], kyz = kern[4 * mtot + gg], kzz = kern[5 * mtot + gg];
      const T2 rxx = refl[gg], rxy = refl[mtot + gg], rxz = refl[2 * mtot + gg];
      const T2 ryy = refl[3 * mtot + gg], ryz = refl[4 * mtot + gg], rzz = refl[5 * mtot + gg];
      const T2* x = X[h];
      buf[gg] = cadd(cadd(cadd(cmulT(kxx, x[0]), cmulT(kxy, x[1])), cmulT(kxz, x[2])),
                     cadd(cadd(cmulT(rxx, xm[0]), cmulT(rxy, xm[1])), cmulT(rxz, xm[2])));
      buf[mtot + gg] = cadd(cadd(cadd(cmulT(kxy, x[0]), cmulT(kyy, x[1])), cmulT(kyz, x[2])),
                            cadd(cadd(cmulT(rxy, xm[0]), cmulT(ryy, xm[1])), cmulT(ryz, xm[2])));
      buf[2 * mtot + gg] =
          cadd(cadd(cadd(cmulT(kxz, x[0]), cmulT(kyz, x[1])), cmulT(kzz, x[2])),
               cadd(cadd(cmulT(rxz, xm[0]), cmulT(ryz, xm[1])), cmulT(rzz, xm[2])));
    }
  }
}

// y_i = alpha_i^-1 x_i - (G x)_i, (G x)_i = buf[.][grid_of[i]] / mtot (FP64).
template <typename R>
__global__ void fft_gather(int n, size_t mtot, const int* __restrict__ grid_of,
                           const double2* __restrict__ inv_alpha, const double2* __restrict__ x,
                           const typename Cx<R>::T* __restrict__ buf, double2* __restrict__ y,
                           const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t g = (size_t)grid_of[i];
  const double scale = 1.0 / (double)mtot;
  const double2 xi[3] = {x[3 * (size_t)i], x[3 * (size_t)i + 1], x[3 * (size_t)i + 2]};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const double2 m = inv_alpha[(size_t)(3 * a + b) * n + i];
      sr += m.x * xi[b].x - m.y * xi[b].y;
      si += m.x * xi[b].y + m.y * xi[b].x;
    }
    const auto v = buf[a * mtot + g];
    y[3 * (size_t)i + a] = make_double2(sr - (double)v.x * scale, si - (double)v.y * scale);
  }
}

// Kernel table: the tensor at every lattice displacement of the circulant
// embedding (fft_matvec.rs:137-165), FCD-filtered within 2 cells when enabled
// (greens.rs:94-167: the near test without contraction, the 27-node
// Gauss-Legendre average with the r^2 < 1e-20 node skip).
__global__ void fft_kernel_table(int mx, int my, int mz, int gx, int gy, int gz,
                                 double spacing, double k, int use_fcd, double cell,
                                 double2* __restrict__ kern) {
  const size_t mtot = (size_t)mx * my * mz;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < mtot;
       g += (size_t)gridDim.x * blockDim.x) {
    const int l = (int)(g / ((size_t)my * mz)), m = (int)((g / mz) % my), nn = (int)(g % mz);
    // displacement of this circulant entry, or none (entries between n-1 and
    // M-(n-1) never meet a dipole pair)
    auto disp = [](int v, int M, int n, bool& ok) {
      if (v <= n - 1) return v;
      if (v >= M - (n - 1)) return v - M;
      ok = false;
      return 0;
    };
    bool ok = true;
    const int dl = disp(l, mx, gx, ok), dm = disp(m, my, gy, ok), dn = disp(nn, mz, gz, ok);
    double2 t[9];
    for (int e = 0; e < 9; ++e) t[e] = make_double2(0.0, 0.0);
    if (ok && (dl | dm | dn) != 0) {
      const double dx = dl * spacing, dy = dm * spacing, dz = dn * spacing;
      const double dist = __dsqrt_rn(
          __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
      if (use_fcd && !(dist > 2.0 * cell)) {
        const double nodes[3] = {-sqrt(3.0 / 5.0), 0.0, sqrt(3.0 / 5.0)};
        const double wts[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
        const double h = cell / 2.0;
        double tw = 0.0;
        double2 gq[9];
        for (int ix = 0; ix < 3; ++ix)
          for (int iy = 0; iy < 3; ++iy)
            for (int iz = 0; iz < 3; ++iz) {
              const double ex = dx - h * nodes[ix], ey = dy - h * nodes[iy],
                           ez = dz - h * nodes[iz];
              if (ex * ex + ey * ey + ez * ez < 1e-20) continue;
              const double wt = wts[ix] * wts[iy] * wts[iz];
              greens_point_d(ex, ey, ez, k, gq);
              for (int e = 0; e < 9; ++e) {
                t[e].x += wt * gq[e].x;
                t[e].y += wt * gq[e].y;
              }
              tw += wt;
            }
        if (tw > 1e-30)
          for (int e = 0; e < 9; ++e) {
            t[e].x /= tw;
            t[e].y /= tw;
          }
      } else {
        greens_point_d(dx, dy, dz, k, t);
      }
    }
    const int sym[6] = {0, 1, 2, 4, 5, 8};  // xx xy xz yy yz zz
    for (int c = 0; c < 6; ++c) kern[c * mtot + g] = t[sym[c]];
  }
}

// Reflected table: R at lateral displacement (dl, dm) and height sum t = nn
// (zero for t > 2 gz - 2).  mode 1: the Fresnel image tensor
// G(dl d, dm d, 2 (z_lo - z0) + t d), skipped below r^2 = 1e-20
// (assembly.rs:129-156); mode 2: the Sommerfeld G_refl with rho = d |(dl, dm)|,
// dz = 2 (z_lo - z0) + t d, zero for dz <= 0 (sommerfeld.rs:254-300).
__global__ void fft_refl_table(int mx, int my, int mz, int gx, int gy, int gz, double spacing,
                               double zlo, double z0, int mode, double k, SommDev S,
                               double2* __restrict__ kern) {
  const size_t mtot = (size_t)mx * my * mz;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < mtot;
       g += (size_t)gridDim.x * blockDim.x) {
    const int l = (int)(g / ((size_t)my * mz)), m = (int)((g / mz) % my), nn = (int)(g % mz);
    auto disp = [](int v, int M, int n, bool& ok) {
      if (v <= n - 1) return v;
      if (v >= M - (n - 1)) return v - M;
      ok = false;
      return 0;
    };
    bool ok = nn <= 2 * gz - 2;
    const int dl = disp(l, mx, gx, ok), dm = disp(m, my, gy, ok);
    double2 t[9];
    for (int e = 0; e < 9; ++e) t[e] = make_double2(0.0, 0.0);
    if (ok) {
      const double dx = dl * spacing, dy = dm * spacing;
      const double dz = (zlo - z0) + (zlo - z0) + nn * spacing;
      if (mode == 1) {
        if (dx * dx + dy * dy + dz * dz >= 1e-20) greens_point_d(dx, dy, dz, k, t);
      } else if (dz > 0.0) {
        const int sq = dl * dl + dm * dm;
        double2 v[4];
        somm_record(somm_integrals(S, spacing * sqrt((double)sq), dz), v);
        double cp = 1.0, sp = 0.0;
        if (sq > 0) {
          const double inv = rsqrt((double)sq);
          cp = dl * inv;
          sp = dm * inv;
        }
        const double c2 = 2.0 * cp * cp - 1.0, s2 = 2.0 * sp * cp;
        t[0] = make_double2(v[0].x - v[1].x * c2, v[0].y - v[1].y * c2);
        t[4] = make_double2(v[0].x + v[1].x * c2, v[0].y + v[1].y * c2);
        t[8] = make_double2(-v[2].x, -v[2].y);
        t[1] = make_double2(-v[1].x * s2, -v[1].y * s2);
        t[2] = make_double2(v[3].x * cp, v[3].y * cp);
        t[5] = make_double2(v[3].x * sp, v[3].y * sp);
      }
    }
    const int sym[6] = {0, 1, 2, 4, 5, 8};  // xx xy xz yy yz zz
    for (int c = 0; c < 6; ++c) kern[c * mtot + g] = t[sym[c]];
  }
}

__global__ void fft_twiddles(int L, double2* __restrict__ t64, float2* __restrict__ t32) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= L / 2) return;
  double s, c;
  sincospi(-2.0 * (double)q / (double)L, &s, &c);
  t64[q] = make_double2(c, s);
  t32[q] = make_float2((float)c, (float)s);
}

__global__ void narrow_spectra(size_t count, const double2* __restrict__ src,
                               float2* __restrict__ dst) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < count;
       q += (size_t)gridDim.x * blockDim.x)
    dst[q] = make_float2((float)src[q].x, (float)src[q].y);
}

unsigned grid_for(size_t count) {
  return (unsigned)std::max<size_t>(1, std::min<size_t>((count + 255) / 256, 148 * 16));
}

}  // namespace

// One FFT pass over the lines of axis `ax` (0 = x, 1 = y, 2 = z), restricted
// to outer / inner index ranges [0, n_outer) x [0, n_inner).
template <typename R>
static lum_status fft_pass(const FftOperator& op, typename Cx<R>::T* data, int ncomp, int ax,
                           bool inverse, int n_outer, int n_inner, const int* skip,
                           cudaStream_t st, FftIO io = FftIO{0, -1, nullptr, nullptr, nullptr,
                                                             nullptr, 0, 0.0}) {
  using T2 = typename Cx<R>::T;
  const int L = op.M[ax];
  if (L <= 1 || n_outer <= 0 || n_inner <= 0) return LUM_OK;
  const long long sz = 1, sy = op.M[2], sx = (long long)op.M[1] * op.M[2];
  long long elem, outer, inner;
  if (ax == 2) {  // z lines: outer x, inner y
    elem = sz;
    outer = sx;
    inner = sy;
  } else if (ax == 1) {  // y lines: outer x, inner z
    elem = sy;
    outer = sx;
    inner = sz;
  } else {  // x lines: outer y, inner z
    elem = sx;
    outer = sy;
    inner = sz;
  }
  const int cap = (sizeof(R) == 8) ? 1024 : 2048;  // B * L per CTA
  int B = std::max(1, std::min(n_inner, cap / L));
  // fill the GPU: halve the lines per CTA while the grid has fewer than four
  // CTAs per SM; strided lines keep at least 8 per CTA (coalesced loads)
  const int bmin = (elem == 1) ? 1 : 8;
  while (B > bmin && (long long)n_outer * ((n_inner + B - 1) / B) * ncomp < 4LL * 148)
    B = std::max(bmin, B / 2);
  const size_t smem = sizeof(T2) * ((size_t)2 * B * (L + 1) + L / 2);
  const int chunks = (n_inner + B - 1) / B;
  const dim3 grid((unsigned)((size_t)n_outer * chunks), 1, ncomp);
  const T2* tw = reinterpret_cast<const T2*>(sizeof(R) == 8 ? op.tw64.p : op.tw32.p) +
                 op.tw_off[ax];
  if (io.valid < 0) io.valid = L;
  if (inverse)
    fft_lines<R, true><<<grid, kFftThreads, smem, st>>>(data, op.mtot, L, B, elem, n_outer,
                                                        outer, n_inner, inner, tw, skip, io);
  else
    fft_lines<R, false><<<grid, kFftThreads, smem, st>>>(data, op.mtot, L, B, elem, n_outer,
                                                         outer, n_inner, inner, tw, skip, io);
  LUM_CHECK_LAUNCH();
  return LUM_OK;
}

lum_status FftOperator::build(const double* pos_host, int n_, double spacing_, double cell_,
                              int use_fcd_, cudaStream_t st) {
  n = n_;
  spacing = spacing_ > 0.0 ? spacing_ : cell_;
  cell = cell_;
  use_fcd = use_fcd_;
  if (n <= 0) {
    set_error("No dipoles provided");
    return LUM_ERR_INVALID;
  }
  if (!(spacing > 0.0) || !std::isfinite(spacing)) {
    set_error("the FFT operator needs a positive lattice spacing (got %g)", spacing);
    return LUM_ERR_INVALID;
  }
  if (use_fcd && !(cell > 0.0)) {
    set_error("FCD needs a positive cell size (got %g)", cell);
    return LUM_ERR_INVALID;
  }
  // lattice nodes (fft_matvec.rs:19-59): offsets from the bounding-box corner
  // in units of the spacing, each within 1e-6 of an integer
  double lo[3] = {1e300, 1e300, 1e300};
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      const double v = pos_host[3 * (size_t)i + c];
      if (!std::isfinite(v)) {
        set_error("non-finite dipole position at index %d", i);
        return LUM_ERR_INVALID;
      }
      lo[c] = std::min(lo[c], v);
    }
  std::vector<int> node(3 * (size_t)n);
  int hi[3] = {0, 0, 0};
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      const double f = (pos_host[3 * (size_t)i + c] - lo[c]) / spacing;
      const double r = std::round(f);
      if (std::fabs(f - r) >= 1e-6 || r > 1e6) {
        set_error("dipole %d is not on a cubic lattice of spacing %g", i, spacing);
        return LUM_ERR_INVALID;
      }
      node[3 * (size_t)i + c] = (int)r;
      hi[c] = std::max(hi[c], (int)r);
    }
  lo_z = lo[2];
  for (int c = 0; c < 3; ++c) {
    gn[c] = hi[c] + 1;
    M[c] = 1;
    while (M[c] < 2 * gn[c] - 1) M[c] <<= 1;
    if (M[c] > 1024) {
      set_error("FFT grid too large along axis %d (%d nodes; at most 512)", c, gn[c]);
      return LUM_ERR_INVALID;
    }
  }
  mtot = (size_t)M[0] * M[1] * M[2];
  std::vector<int> node_dip(mtot, -1), grid_of(n);
  for (int i = 0; i < n; ++i) {
    const size_t g = ((size_t)node[3 * (size_t)i] * M[1] + node[3 * (size_t)i + 1]) * M[2] +
                     node[3 * (size_t)i + 2];
    if (node_dip[g] >= 0) {
      set_error("dipoles %d and %d occupy the same lattice node", node_dip[g], i);
      return LUM_ERR_INVALID;
    }
    node_dip[g] = i;
    grid_of[i] = (int)g;
  }
  LUM_TRY(d_node_dip.alloc(sizeof(int) * mtot));
  LUM_TRY(d_grid_of.alloc(sizeof(int) * n));
  LUM_TRY_CUDA(cudaMemcpyAsync(d_node_dip.p, node_dip.data(), sizeof(int) * mtot,
                               cudaMemcpyHostToDevice, st));
  LUM_TRY_CUDA(cudaMemcpyAsync(d_grid_of.p, grid_of.data(), sizeof(int) * n,
                               cudaMemcpyHostToDevice, st));
  // twiddle tables, one per axis length
  size_t off = 0;
  for (int c = 0; c < 3; ++c) {
    tw_off[c] = off;
    off += std::max(1, M[c] / 2);
  }
  LUM_TRY(tw64.alloc(sizeof(double2) * off));
  LUM_TRY(tw32.alloc(sizeof(float2) * off));
  for (int c = 0; c < 3; ++c)
    if (M[c] > 1) {
      fft_twiddles<<<(M[c] / 2 + 255) / 256, 256, 0, st>>>(
          M[c], tw64.as<double2>() + tw_off[c], tw32.as<float2>() + tw_off[c]);
      LUM_CHECK_LAUNCH();
    }
  LUM_TRY(kern64.alloc(sizeof(double2) * 6 * mtot));
  LUM_TRY(kern32.alloc(sizeof(float2) * 6 * mtot));
  LUM_TRY(buf64.alloc(sizeof(double2) * 3 * mtot));
  LUM_TRY(buf32.alloc(sizeof(float2) * 3 * mtot));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));  // host tables are freed on return
  return LUM_OK;
}

lum_status FftOperator::set_physics(double k_, const double* inv_alpha_host, cudaStream_t st) {
  if (!(k_ > 0.0) || !std::isfinite(k_)) {
    set_error("wavenumber must be positive and finite (got %g)", k_);
    return LUM_ERR_INVALID;
  }
  k = k_;
  // alpha^-1 element-major [9][n]
  std::vector<double2> ia(9 * (size_t)n);
  for (int i = 0; i < n; ++i)
    for (int e = 0; e < 9; ++e)
      ia[(size_t)e * n + i] = make_double2(inv_alpha_host[18 * (size_t)i + 2 * e],
                                           inv_alpha_host[18 * (size_t)i + 2 * e + 1]);
  LUM_TRY(inv_alpha.alloc(sizeof(double2) * ia.size()));
  LUM_TRY_CUDA(cudaMemcpyAsync(inv_alpha.p, ia.data(), sizeof(double2) * ia.size(),
                               cudaMemcpyHostToDevice, st));
  fft_kernel_table<<<grid_for(mtot), 256, 0, st>>>(M[0], M[1], M[2], gn[0], gn[1], gn[2],
                                                   spacing, k, use_fcd, cell,
                                                   kern64.as<double2>());
  LUM_CHECK_LAUNCH();
  // forward transform of the six components over the whole circulant
  double2* K = kern64.as<double2>();
  LUM_TRY(fft_pass<double>(*this, K, 6, 2, false, M[0], M[1], nullptr, st));
  LUM_TRY(fft_pass<double>(*this, K, 6, 1, false, M[0], M[2], nullptr, st));
  LUM_TRY(fft_pass<double>(*this, K, 6, 0, false, M[1], M[2], nullptr, st));
  narrow_spectra<<<grid_for(6 * mtot), 256, 0, st>>>(6 * mtot, K, kern32.as<float2>());
  LUM_CHECK_LAUNCH();
  LUM_TRY_CUDA(cudaStreamSynchronize(st));  // ia is freed on return
  return LUM_OK;
}

lum_status FftOperator::set_reflection(int mode, const lum_substrate* fresnel,
                                      const SommDev* somm, cudaStream_t st) {
  refl_mode = mode;
  refl_stale = 0;
  if (mode == 0) {
    refl64.release();
    refl32.release();
    return LUM_OK;
  }
  SommDev S{};
  double z0 = 0.0;
  if (mode == 1) {
    z0 = fresnel->z_interface;
    const double2 r = make_double2(fresnel->refl_re, fresnel->refl_im);
    refl_m[0] = make_double2(-r.x, -r.y);
    refl_m[1] = make_double2(-r.x, -r.y);
    refl_m[2] = r;
  } else {
    S = *somm;
    z0 = S.z0;
    for (int c = 0; c < 3; ++c) refl_m[c] = make_double2(1.0, 0.0);
  }
  if (!refl64.p) {
    LUM_TRY(refl64.alloc(sizeof(double2) * 6 * mtot));
    LUM_TRY(refl32.alloc(sizeof(float2) * 6 * mtot));
  }
  double2* K = refl64.as<double2>();
  fft_refl_table<<<grid_for(mtot), 256, 0, st>>>(M[0], M[1], M[2], gn[0], gn[1], gn[2], spacing,
                                                 lo_z, z0, mode, k, S, K);
  LUM_CHECK_LAUNCH();
  LUM_TRY(fft_pass<double>(*this, K, 6, 2, false, M[0], M[1], nullptr, st));
  LUM_TRY(fft_pass<double>(*this, K, 6, 1, false, M[0], M[2], nullptr, st));
  LUM_TRY(fft_pass<double>(*this, K, 6, 0, false, M[1], M[2], nullptr, st));
  narrow_spectra<<<grid_for(6 * mtot), 256, 0, st>>>(6 * mtot, K, refl32.as<float2>());
  LUM_CHECK_LAUNCH();
  return LUM_OK;
}

template <typename R>
static lum_status fft_apply_t(FftOperator& op, typename Cx<R>::T* buf,
                              const typename Cx<R>::T* kern, const typename Cx<R>::T* refl,
                              const double2* x, double2* y, cudaStream_t st, const int* skip) {
  // With more than one layer the first z pass reads x through the node map
  // and the last one writes y (no scatter / gather kernels, no zero fill);
  // a single layer (M_z = 1, no z pass) scatters and gathers.
  const bool fused = op.M[2] > 1;
  const FftIO plain{0, -1, nullptr, nullptr, nullptr, nullptr, 0, 0.0};
  const FftIO load_x{1, op.gn[2], op.d_node_dip.as<int>(), x, nullptr, nullptr, op.n, 0.0};
  const FftIO store_y{2, -1, op.d_node_dip.as<int>(), x, op.inv_alpha.as<double2>(), y, op.n,
                      1.0 / (double)op.mtot};
  if (!fused) {
    fft_scatter<R><<<grid_for(op.mtot), 256, 0, st>>>(op.mtot, op.d_node_dip.as<int>(), x, buf,
                                                      skip);
    LUM_CHECK_LAUNCH();
  }
  // forward: z lines of the occupied (x, y) box, y lines of the occupied x
  // range (y beyond the box masked), then every x line (x beyond it masked)
  LUM_TRY(fft_pass<R>(op, buf, 3, 2, false, op.gn[0], op.gn[1], skip, st, load_x));
  FftIO yv = plain, xv = plain;
  if (fused) {
    yv.valid = op.gn[1];
    xv.valid = op.gn[0];
  }
  LUM_TRY(fft_pass<R>(op, buf, 3, 1, false, op.gn[0], op.M[2], skip, st, yv));
  LUM_TRY(fft_pass<R>(op, buf, 3, 0, false, op.M[1], op.M[2], skip, st, xv));
  if (refl) {
    using T2 = typename Cx<R>::T;
    T2 m[3];
    for (int c = 0; c < 3; ++c) {
      m[c].x = (R)op.refl_m[c].x;
      m[c].y = (R)op.refl_m[c].y;
    }
    const int lines = op.M[0] * op.M[1];
    fft_spectral_product_refl<R><<<grid_for((size_t)lines * (op.M[2] / 2 + 1)), 256, 0, st>>>(
        lines, op.M[2], op.mtot, kern, refl, m[0], m[1], m[2], buf, skip);
  } else {
    fft_spectral_product<R><<<grid_for(op.mtot), 256, 0, st>>>(op.mtot, kern, buf, skip);
  }
  LUM_CHECK_LAUNCH();
  // inverse: every x line, then only the lines that hold dipole nodes
  LUM_TRY(fft_pass<R>(op, buf, 3, 0, true, op.M[1], op.M[2], skip, st));
  LUM_TRY(fft_pass<R>(op, buf, 3, 1, true, op.gn[0], op.M[2], skip, st));
  LUM_TRY(fft_pass<R>(op, buf, 3, 2, true, op.gn[0], op.gn[1], skip, st,
                      fused ? store_y : plain));
  if (!fused) {
    fft_gather<R><<<(op.n + 255) / 256, 256, 0, st>>>(op.n, op.mtot, op.d_grid_of.as<int>(),
                                                      op.inv_alpha.as<double2>(), x, buf, y,
                                                      skip);
    LUM_CHECK_LAUNCH();
  }
  return LUM_OK;
}

lum_status FftOperator::apply(int precision, const double2* x, double2* y, cudaStream_t st,
                              cudaEvent_t ev0, cudaEvent_t ev1, const int* skip) {
  if (refl_stale) {
    set_error("the Sommerfeld spectra belong to another wavelength: call "
              "lum_session_set_sommerfeld after lum_session_set_wavelength");
    return LUM_ERR_INVALID;
  }
  if (ev0) cudaEventRecord(ev0, st);
  lum_status s;
  const bool r = refl_mode != 0;
  if (precision == LUM_FP32)
    s = fft_apply_t<float>(*this, buf32.as<float2>(), kern32.as<float2>(),
                           r ? refl32.as<float2>() : nullptr, x, y, st, skip);
  else
    s = fft_apply_t<double>(*this, buf64.as<double2>(), kern64.as<double2>(),
                            r ? refl64.as<double2>() : nullptr, x, y, st, skip);
  if (ev1) cudaEventRecord(ev1, st);
  return s;
}

}  // namespace lum
