// cached.cu -- the dense 3N x 3N interaction matrix on the device.
//
// Assembly (assemble_interaction_matrix, assembly.rs:45-175): one thread per
// dipole pair (i, j) evaluates the 3x3 block once (the reference's WGSL
// shader re-evaluated G for each of the 9 entries, matrix_assemble.wgsl:59)
// and writes row segments 3j..3j+2 of rows 3i..3i+2; consecutive threads
// take consecutive j, so each warp store is a contiguous run of a row.  The
// alpha^-1 diagonal is written on the device (no host patch,
// cf. gpu.rs:585-603), the FCD near pairs are corrected by a second pass
// over the ELL near list, and a substrate image term and the Ewald sum are
// included as in the reference.
//
// Matvec (MatvecSession::matvec): y = A x is bound by reading A from HBM
// (8 or 16 bytes per complex entry).  One warp per row streams the row with
// coalesced 8/16-byte loads, x is read through L1/L2 (3N complex is a few
// MB at most), products accumulate in FP64 and the warp reduces by shuffle.
#include "lumina_internal.cuh"
#include "device_physics.cuh"

namespace lum {


template <typename T2> __device__ __forceinline__ T2 mk(double re, double im);
template <> __device__ __forceinline__ float2 mk<float2>(double re, double im) {
  return make_float2((float)re, (float)im);
}
template <> __device__ __forceinline__ double2 mk<double2>(double re, double im) {
  return make_double2(re, im);
}

template <typename T2>
__global__ void __launch_bounds__(128)
assemble_pairs(int n, const double4* __restrict__ pos, const double2* __restrict__ inv_alpha,
               double k, int has_lat, LatticeDev L, const double4* __restrict__ lreal,
               const double4* __restrict__ lrecip, double kb0, double kb1, double kb2,
               int has_sub, SubstrateDev sub, size_t ld, T2* __restrict__ A) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long npairs = (long long)n * n;
  if (idx >= npairs) return;
  const int i = (int)(idx / n), j = (int)(idx % n);
  const double4 ri = pos[i], rj = pos[j];
  const double kb[3] = {kb0, kb1, kb2};
  double2 blk[9];
  for (int e = 0; e < 9; ++e) blk[e] = make_double2(0.0, 0.0);
  if (i == j)
    for (int e = 0; e < 9; ++e) blk[e] = inv_alpha[(size_t)e * n + i];
  double2 g[9];
  if (has_lat) {
    ewald_tensor(L, lreal, lrecip, ri.x - rj.x, ri.y - rj.y, ri.z - rj.z, kb, k, g);
    for (int e = 0; e < 9; ++e) {
      blk[e].x -= g[e].x;
      blk[e].y -= g[e].y;
    }
  } else if (i != j) {
    greens_point_d(ri.x - rj.x, ri.y - rj.y, ri.z - rj.z, k, g);
    for (int e = 0; e < 9; ++e) {
      blk[e].x -= g[e].x;
      blk[e].y -= g[e].y;
    }
  }
  if (has_sub) {  // assembly.rs:129-156, all (i, j) including i == j
    double dx = ri.x - rj.x, dy = ri.y - rj.y, dz = ri.z - (2.0 * sub.z_interface - rj.z);
    if (dx * dx + dy * dy + dz * dz >= 1e-20) {
      if (has_lat)
        ewald_tensor(L, lreal, lrecip, dx, dy, dz, kb, k, g);
      else
        greens_point_d(dx, dy, dz, k, g);
      const double2 r = make_double2(sub.refl_re, sub.refl_im);
      const double2 m[3] = {make_double2(-r.x, -r.y), make_double2(-r.x, -r.y), r};
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          double2 gg = g[3 * a + b];
          double tr = m[b].x * gg.x - m[b].y * gg.y, ti = m[b].x * gg.y + m[b].y * gg.x;
          blk[3 * a + b].x -= tr;
          blk[3 * a + b].y -= ti;
        }
    }
  }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      A[(3 * (size_t)i + a) * ld + 3 * (size_t)j + b] = mk<T2>(blk[3 * a + b].x, blk[3 * a + b].y);
}

// FCD: A[i][j] -= (G_fcd - G_point) for every near pair.
template <typename T2>
__global__ void assemble_fcd(int n, int ell_w, const int* __restrict__ near_j,
                             const double2* __restrict__ fcd, size_t ld, T2* __restrict__ A) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * ell_w) return;
  const int w = idx / n, i = idx % n;
  const int j = near_j[(size_t)w * n + i];
  if (j < 0) return;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      const double2 c = fcd[((size_t)w * 9 + 3 * a + b) * n + i];
      T2& e = A[(3 * (size_t)i + a) * ld + 3 * (size_t)j + b];
      e = mk<T2>((double)e.x - c.x, (double)e.y - c.y);
    }
}

// y = A x in two launches.  gemv_part: one warp per (row, column chunk), the
// chunk streamed with 16-byte loads (two FP32 complex or one FP64 complex per
// load, four in flight per lane), FP64 accumulation, shuffle reduction, one
// partial per chunk.  Many small blocks let the block scheduler balance the
// SMs to the last wave.  gemv_reduce sums the chunks of a row in chunk order
// (deterministic).
constexpr int kGemvRows = 8;  // rows (warps) per block

__device__ __forceinline__ void cmac(double& sr, double& si, float ar, float ai, double2 x) {
  sr += (double)ar * x.x - (double)ai * x.y;
  si += (double)ar * x.y + (double)ai * x.x;
}

template <typename T2>
__global__ void __launch_bounds__(256)
gemv_part(int dim, size_t ld, int chunk, const T2* __restrict__ A,
          const double2* __restrict__ x, double2* __restrict__ part,
          const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int row = blockIdx.x * kGemvRows + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= dim) return;
  const int c0 = blockIdx.y * chunk, c1 = min(dim, c0 + chunk);
  const T2* a = A + (size_t)row * ld;
  double sr = 0.0, si = 0.0;
  if constexpr (sizeof(T2) == sizeof(float2)) {
    // float4 p holds complex 2p and 2p+1 (rows start 128-byte aligned, c0 even)
    const float4* a4 = reinterpret_cast<const float4*>(a);
    const int p1 = c1 >> 1;
    int p = (c0 >> 1) + lane;
    for (; p + 96 < p1; p += 128) {
      const float4 v0 = __ldcs(&a4[p]), v1 = __ldcs(&a4[p + 32]), v2 = __ldcs(&a4[p + 64]),
                   v3 = __ldcs(&a4[p + 96]);
      cmac(sr, si, v0.x, v0.y, __ldg(&x[2 * p]));
      cmac(sr, si, v0.z, v0.w, __ldg(&x[2 * p + 1]));
      cmac(sr, si, v1.x, v1.y, __ldg(&x[2 * p + 64]));
      cmac(sr, si, v1.z, v1.w, __ldg(&x[2 * p + 65]));
      cmac(sr, si, v2.x, v2.y, __ldg(&x[2 * p + 128]));
      cmac(sr, si, v2.z, v2.w, __ldg(&x[2 * p + 129]));
      cmac(sr, si, v3.x, v3.y, __ldg(&x[2 * p + 192]));
      cmac(sr, si, v3.z, v3.w, __ldg(&x[2 * p + 193]));
    }
    for (; p < p1; p += 32) {
      const float4 v = __ldcs(&a4[p]);
      cmac(sr, si, v.x, v.y, __ldg(&x[2 * p]));
      cmac(sr, si, v.z, v.w, __ldg(&x[2 * p + 1]));
    }
    if ((c1 & 1) && lane == 0) {  // odd last column of the row
      const float2 v = a[c1 - 1];
      cmac(sr, si, v.x, v.y, __ldg(&x[c1 - 1]));
    }
  } else {
    int c = c0 + lane;
    for (; c + 96 < c1; c += 128) {
      const double2 a0 = __ldcs(&a[c]), a1 = __ldcs(&a[c + 32]), a2 = __ldcs(&a[c + 64]),
                    a3 = __ldcs(&a[c + 96]);
      const double2 x0 = __ldg(&x[c]), x1 = __ldg(&x[c + 32]), x2 = __ldg(&x[c + 64]),
                    x3 = __ldg(&x[c + 96]);
      sr += a0.x * x0.x - a0.y * x0.y;
      si += a0.x * x0.y + a0.y * x0.x;
      sr += a1.x * x1.x - a1.y * x1.y;
      si += a1.x * x1.y + a1.y * x1.x;
      sr += a2.x * x2.x - a2.y * x2.y;
      si += a2.x * x2.y + a2.y * x2.x;
      sr += a3.x * x3.x - a3.y * x3.y;
      si += a3.x * x3.y + a3.y * x3.x;
    }
    for (; c < c1; c += 32) {
      const double2 a0 = __ldcs(&a[c]), x0 = __ldg(&x[c]);
      sr += a0.x * x0.x - a0.y * x0.y;
      si += a0.x * x0.y + a0.y * x0.x;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    sr += __shfl_down_sync(0xffffffffu, sr, o);
    si += __shfl_down_sync(0xffffffffu, si, o);
  }
  if (lane == 0) part[(size_t)blockIdx.y * dim + row] = make_double2(sr, si);
}

__global__ void gemv_reduce(int dim, int nchunks, const double2* __restrict__ part,
                            double2* __restrict__ y, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= dim) return;
  double sr = 0.0, si = 0.0;
  for (int c = 0; c < nchunks; ++c) {
    const double2 v = part[(size_t)c * dim + row];
    sr += v.x;
    si += v.y;
  }
  y[row] = make_double2(sr, si);
}

// Y = A X for nrhs right-hand sides on the CUDA cores: one warp per row, A
// read once per NR vectors held in registers.  Element (c, r) of X is at
// X[c * sc + r * sr] (row-major dim x nrhs: sc = nrhs, sr = 1; vectors back to
// back: sc = 1, sr = dim), and the same strides address Y.
template <typename T2, int NR>
__global__ void __launch_bounds__(256)
gemm_rows(int dim, size_t ld, const T2* __restrict__ A, const double2* __restrict__ X,
          long long sc, long long sr_, int c0, double2* __restrict__ Y) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= dim) return;
  const T2* row = A + (size_t)warp * ld;
  double sr[NR], si[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) sr[r] = si[r] = 0.0;
  for (int c = lane; c < dim; c += 32) {
    T2 a = row[c];
    const double2* xr = X + (long long)c * sc + (long long)c0 * sr_;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      double2 xv = __ldg(&xr[r * sr_]);
      sr[r] += (double)a.x * xv.x - (double)a.y * xv.y;
      si[r] += (double)a.x * xv.y + (double)a.y * xv.x;
    }
  }
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    for (int o = 16; o > 0; o >>= 1) {
      sr[r] += __shfl_down_sync(0xffffffffu, sr[r], o);
      si[r] += __shfl_down_sync(0xffffffffu, si[r], o);
    }
    if (lane == 0) Y[(long long)warp * sc + (long long)(c0 + r) * sr_] = make_double2(sr[r], si[r]);
  }
}

// FP64 rows (dense, dim entries each) -> FP32 rows of pitch ld.
__global__ void narrow_rows(size_t rows, int dim, const double2* __restrict__ src, size_t ld,
                            float2* __restrict__ dst) {
  const size_t count = rows * dim;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < count;
       q += (size_t)gridDim.x * blockDim.x) {
    const size_t r = q / dim, c = q % dim;
    const double2 v = src[q];
    dst[r * ld + c] = make_float2((float)v.x, (float)v.y);
  }
}

lum_status CachedOperator::allocate(int dim_, int precision_) {
  dim = dim_;
  precision = precision_;
  // Rows are padded to a multiple of 16 complex entries (128 B in FP32):
  // every row starts 128-byte aligned, and the tensor-core GEMM reads the
  // matrix through a TMA map whose row pitch must be a multiple of 16 bytes.
  // The padding is zero so that it contributes nothing to a product.
  ld = ((size_t)dim + 15) / 16 * 16;
  const size_t es = (precision == LUM_FP32) ? sizeof(float2) : sizeof(double2);
  LUM_TRY(A.alloc(es * ld * dim));
  LUM_TRY_CUDA(cudaMemset(A.p, 0, es * ld * dim));
  tc.release();
  gemv_chunks = 0;
  return LUM_OK;
}

lum_status CachedOperator::upload(const double* host, cudaStream_t st) {
  if (precision == LUM_FP64) {
    LUM_TRY_CUDA(cudaMemcpy2DAsync(A.p, sizeof(double2) * ld, host, sizeof(double2) * dim,
                                   sizeof(double2) * dim, dim, cudaMemcpyHostToDevice, st));
    LUM_TRY_CUDA(cudaStreamSynchronize(st));
    return LUM_OK;
  }
  // FP32 storage: stream the FP64 host matrix through a staging buffer and
  // narrow on the device, a bounded number of rows at a time.
  const size_t rows_per = std::max<size_t>(1, (size_t)(64u << 20) / (sizeof(double2) * dim));
  DevBuf stage;
  LUM_TRY(stage.alloc(sizeof(double2) * rows_per * dim));
  for (size_t r0 = 0; r0 < (size_t)dim; r0 += rows_per) {
    const size_t nr = std::min(rows_per, (size_t)dim - r0);
    LUM_TRY_CUDA(cudaMemcpyAsync(stage.p, host + 2 * r0 * dim, sizeof(double2) * nr * dim,
                                 cudaMemcpyHostToDevice, st));
    narrow_rows<<<1024, 256, 0, st>>>(nr, dim, stage.as<double2>(), ld,
                                      A.as<float2>() + r0 * ld);
    LUM_CHECK_LAUNCH();
  }
  LUM_TRY_CUDA(cudaStreamSynchronize(st));
  return LUM_OK;
}

lum_status CachedOperator::assemble(const OtfOperator& g, cudaStream_t st) {
  const int n = g.n;
  const long long npairs = (long long)n * n;
  const int threads = 128;
  const long long blocks = (npairs + threads - 1) / threads;
  if (blocks > 0x7fffffffLL) {
    set_error("matrix too large for device assembly");
    return LUM_ERR_INVALID;
  }
  if (g.has_lattice && g.table_ok) {
    LUM_TRY(assemble_from_table(g, precision, A.p, ld, st));
    return somm_assemble(g, precision, A.p, ld, st);
  }
  if (precision == LUM_FP32)
    assemble_pairs<float2><<<(unsigned)blocks, threads, 0, st>>>(
        n, g.pos64.as<double4>(), g.inv_alpha.as<double2>(), g.k, g.has_lattice, g.latdev,
        g.lat_real.as<double4>(), g.lat_recip.as<double4>(), g.kbloch[0], g.kbloch[1],
        g.kbloch[2], g.has_substrate, g.substrate, ld, A.as<float2>());
  else
    assemble_pairs<double2><<<(unsigned)blocks, threads, 0, st>>>(
        n, g.pos64.as<double4>(), g.inv_alpha.as<double2>(), g.k, g.has_lattice, g.latdev,
        g.lat_real.as<double4>(), g.lat_recip.as<double4>(), g.kbloch[0], g.kbloch[1],
        g.kbloch[2], g.has_substrate, g.substrate, ld, A.as<double2>());
  LUM_CHECK_LAUNCH();
  if (g.ell_w > 0 && !g.has_lattice) {
    const int total = n * g.ell_w;
    if (precision == LUM_FP32)
      assemble_fcd<float2><<<(total + 255) / 256, 256, 0, st>>>(
          n, g.ell_w, g.near_j.as<int>(), g.fcd64.as<double2>(), ld, A.as<float2>());
    else
      assemble_fcd<double2><<<(total + 255) / 256, 256, 0, st>>>(
          n, g.ell_w, g.near_j.as<int>(), g.fcd64.as<double2>(), ld, A.as<double2>());
    LUM_CHECK_LAUNCH();
  }
  return somm_assemble(g, precision, A.p, ld, st);
}

lum_status CachedOperator::apply(const double2* x, double2* y, cudaStream_t st,
                                 const int* skip) {
  if (gemv_chunks == 0) {
    // about 8 waves of 8-warp blocks (8 resident per SM), chunks of >= 512
    // complex entries, an even chunk length (16-byte loads of FP32 pairs)
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int row_blocks = (dim + kGemvRows - 1) / kGemvRows;
    const int want = std::max(1, (8 * 8 * sms + row_blocks - 1) / row_blocks);
    gemv_chunks = std::max(1, std::min(want, (dim + 511) / 512));
    gemv_chunk = ((dim + gemv_chunks - 1) / gemv_chunks + 63) / 64 * 64;
    gemv_chunks = (dim + gemv_chunk - 1) / gemv_chunk;
    LUM_TRY(gemv_part_buf.alloc(sizeof(double2) * (size_t)gemv_chunks * dim));
  }
  const dim3 grid((dim + kGemvRows - 1) / kGemvRows, gemv_chunks);
  if (precision == LUM_FP32)
    gemv_part<float2><<<grid, 32 * kGemvRows, 0, st>>>(dim, ld, gemv_chunk, A.as<float2>(), x,
                                                       gemv_part_buf.as<double2>(), skip);
  else
    gemv_part<double2><<<grid, 32 * kGemvRows, 0, st>>>(dim, ld, gemv_chunk, A.as<double2>(), x,
                                                        gemv_part_buf.as<double2>(), skip);
  LUM_CHECK_LAUNCH();
  gemv_reduce<<<(dim + 255) / 256, 256, 0, st>>>(dim, gemv_chunks, gemv_part_buf.as<double2>(),
                                                 y, skip);
  LUM_CHECK_LAUNCH();
  return LUM_OK;
}

lum_status CachedOperator::apply_multi_cuda_cores(const double2* X, double2* Y, int nrhs,
                                                  long long sc, long long sr, cudaStream_t st) {
  const int blocks = (int)(((size_t)dim * 32 + 255) / 256);
  int c0 = 0;
  while (c0 < nrhs) {
    int left = nrhs - c0;
    int nr = left >= 8 ? 8 : (left >= 4 ? 4 : (left >= 2 ? 2 : 1));
#define LUM_GEMM_CASE(NRV)                                                                     \
  case NRV:                                                                                    \
    if (precision == LUM_FP32)                                                                 \
      gemm_rows<float2, NRV><<<blocks, 256, 0, st>>>(dim, ld, A.as<float2>(), X, sc, sr, c0,   \
                                                     Y);                                       \
    else                                                                                       \
      gemm_rows<double2, NRV><<<blocks, 256, 0, st>>>(dim, ld, A.as<double2>(), X, sc, sr, c0, \
                                                      Y);                                      \
    break;
    switch (nr) {
      LUM_GEMM_CASE(8)
      LUM_GEMM_CASE(4)
      LUM_GEMM_CASE(2)
      LUM_GEMM_CASE(1)
    }
#undef LUM_GEMM_CASE
    LUM_CHECK_LAUNCH();
    c0 += nr;
  }
  return LUM_OK;
}

lum_status CachedOperator::apply_multi(const double2* X, double2* Y, int nrhs, long long sc,
                                       long long sr, int method, cudaStream_t st) {
  const bool tensor = precision == LUM_FP32 &&
                      (method == LUM_MATMUL_TENSOR || (method == LUM_MATMUL_AUTO && nrhs >= kTcMinRhs));
  if (method == LUM_MATMUL_TENSOR && precision != LUM_FP32) {
    set_error("the tensor-core product needs FP32 matrix storage");
    return LUM_ERR_INVALID;
  }
  if (tensor) return cgemm_tf32x3(*this, X, sc, sr, Y, sc, sr, nrhs, st);
  return apply_multi_cuda_cores(X, Y, nrhs, sc, sr, st);
}

}  // namespace lum
