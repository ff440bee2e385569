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
// (8 or 16 bytes per complex entry).  The product runs over blocks of
// 192 x 192 entries (gemv_sym_tiles): one CTA reads a block once with
// 16-byte streaming loads, holds the block's 192 entries of x in registers
// and shared memory, and writes the block's partial row sums to a slot that
// gemv_reduce adds in order.  The same kernel serves the symmetric tile
// storage, where each stored tile is also applied transposed.  The older
// row-chunk GEMV (gemv_part: one warp per row chunk, FP64 accumulation) is
// kept behind LUMINA_DENSE_GEMV=rows.
#include "lumina_internal.cuh"
#include "device_physics.cuh"

#include <cstdlib>

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

// ---------------------------------------------------------------------------
// Symmetric tile storage.  Without a lattice sum or a substrate term the
// matrix is complex symmetric: G(d) = G(d)^T = G(-d) (greens.rs:34-71), the
// FCD cell average is symmetric in its two dipoles (greens.rs:94-167: the
// 27 nodes are symmetric about the cell centre), and the diagonal blocks
// sit in diagonal tiles, which are stored whole.  So A is kept as its tiles
// (I, J), I <= J, of kSymTile x kSymTile entries -- half the bytes of the
// dense rows -- and a product reads each stored tile once and applies it
// twice: y_I += A_IJ x_J (row side) and, for I < J, y_J += A_IJ^T x_I
// (column side).
// ---------------------------------------------------------------------------
constexpr int kSymTileDip = kSymTile / 3;         // 64 dipoles a side
constexpr int kSymWarps = 8;
constexpr int kSymRowsPerWarp = kSymTile / kSymWarps;  // 24

// Offset (in tiles) of tile (I, J), I <= J, among nt tiles a side: the
// tile rows before I hold sum_{r < I} (nt - r) = I (2 nt - I + 1) / 2 tiles.
__host__ __device__ __forceinline__ size_t sym_tile_offset(int I, int J, int nt) {
  return (size_t)I * (size_t)(2 * nt - I + 1) / 2 + (size_t)(J - I);
}

// One block per tile (I, J) of the grid (nt, nt); blocks below the diagonal
// return.  Each thread evaluates whole 3x3 dipole blocks (i, j) as
// assemble_pairs does for a free-space system: alpha^-1 on i == j, -G_ij
// otherwise.  Entries past dim keep the zero of the allocation.
template <typename T2>
__global__ void __launch_bounds__(256)
assemble_sym_tiles(int n, int nt, const double4* __restrict__ pos,
                   const double2* __restrict__ inv_alpha, double k, T2* __restrict__ A) {
  const int I = blockIdx.y, J = blockIdx.x;
  if (I > J) return;
  T2* tile = A + sym_tile_offset(I, J, nt) * (size_t)(kSymTile * kSymTile);
  for (int q = threadIdx.x; q < kSymTileDip * kSymTileDip; q += blockDim.x) {
    const int li = q / kSymTileDip, lj = q % kSymTileDip;
    const int i = I * kSymTileDip + li, j = J * kSymTileDip + lj;
    if (i >= n || j >= n) continue;
    double2 blk[9];
    if (i == j) {
      for (int e = 0; e < 9; ++e) blk[e] = inv_alpha[(size_t)e * n + i];
    } else {
      const double4 ri = pos[i], rj = pos[j];
      double2 g[9];
      greens_point_d(ri.x - rj.x, ri.y - rj.y, ri.z - rj.z, k, g);
      for (int e = 0; e < 9; ++e) blk[e] = make_double2(-g[e].x, -g[e].y);
    }
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        tile[(size_t)(3 * li + a) * kSymTile + 3 * lj + b] =
            mk<T2>(blk[3 * a + b].x, blk[3 * a + b].y);
  }
}

// FCD: A[i][j] -= (G_fcd - G_point) for the near pairs whose block is
// stored (tile of i <= tile of j); the pair (j, i) of the other tiles is the
// transpose and is read through the column side of the product.
template <typename T2>
__global__ void assemble_sym_fcd(int n, int nt, int ell_w, const int* __restrict__ near_j,
                                 const double2* __restrict__ fcd, T2* __restrict__ A) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * ell_w) return;
  const int w = idx / n, i = idx % n;
  const int j = near_j[(size_t)w * n + i];
  if (j < 0) return;
  const int I = i / kSymTileDip, J = j / kSymTileDip;
  if (I > J) return;
  T2* tile = A + sym_tile_offset(I, J, nt) * (size_t)(kSymTile * kSymTile);
  const int li = i - I * kSymTileDip, lj = j - J * kSymTileDip;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      const double2 c = fcd[((size_t)w * 9 + 3 * a + b) * n + i];
      T2& e = tile[(size_t)(3 * li + a) * kSymTile + 3 * lj + b];
      e = mk<T2>((double)e.x - c.x, (double)e.y - c.y);
    }
}

// Element types of the tile product: FP32 storage computes in FP32 (as the
// FP32 operator does), FP64 storage in FP64; a 16-byte load carries CPV
// complex entries.
template <typename T2> struct SymGemvT;
template <> struct SymGemvT<float2> {
  using R = float;
  using V = float4;
  static constexpr int CPV = 2;
  static constexpr int RG = 4;  // rows whose loads are in flight together
  __device__ static float2 get(const float4& v, int h) {
    return h == 0 ? make_float2(v.x, v.y) : make_float2(v.z, v.w);
  }
};
template <> struct SymGemvT<double2> {
  using R = double;
  using V = double2;
  static constexpr int CPV = 1;
  static constexpr int RG = 2;
  __device__ static double2 get(const double2& v, int) { return v; }
};

// Sum over the 32 lanes of 16 values per lane, transposed: afterwards lane l
// holds in v[0] the total of value 8 b4 + 4 b3 + 2 b2 + b1 (b = bits of l);
// lanes l and l ^ 1 hold the same total.
template <typename R>
__device__ __forceinline__ void sym_transpose_reduce16(R (&v)[16], int lane) {
#pragma unroll
  for (int h = 8, m = 16; h >= 1; h >>= 1, m >>= 1) {
    const bool up = (lane & m) != 0;
#pragma unroll
    for (int i = 0; i < h; ++i) {
      const R send = up ? v[i] : v[i + h];
      const R keep = up ? v[i + h] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, m);
    }
  }
  v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
}

// One block per stored tile (items[blockIdx.x] = (I, J)).  Warp w owns tile
// rows 24 w .. 24 w + 23; lane l owns the complex columns CPV (l + 32 e) + h
// (e < 6 / CPV, h < CPV), so every load instruction of a warp reads one
// contiguous run of a tile row.  Row side: each row's 6 products per lane
// are summed over the warp by a transposed shuffle reduction, 8 rows at a
// time.  Column side: each lane sums A[r][c] x_I[r] over its warp's rows,
// and the 8 warps' sums are added in warp order through shared memory.
// Output (no atomics, every entry written once per product):
//   part[J][I*T + r] = sum_c A_IJ[r][c] x_J[c]       (row side)
//   part[I][J*T + c] = sum_r A_IJ[r][c] x_I[r]       (column side, I < J)
// so for the rows of tile row R, slot S >= R comes from tile (R, S) and slot
// S < R from tile (S, R); gemv_reduce adds the nt slots in order.
//
// DENSE: the same row side over dense rows [dim][ld] (every block (I, J) of
// the nt x nt grid, no column side): the block of rows I*T.. and columns
// J*T.. is read with the row pitch ld, rows past dim and vectors past ld
// are not read.  Against gemv_part (a warp streaming one row chunk, FP64
// accumulation) it keeps x_J in registers for all 192 rows of the block and
// computes FP32 storage in FP32, so no x is re-read per row and no FP32
// entry is converted to FP64.
template <typename T2, bool DENSE>
__global__ void __launch_bounds__(kSymWarps * 32, 2)
gemv_sym_tiles(int dim, int nt, size_t ld, const T2* __restrict__ A,
               const int2* __restrict__ items, const double2* __restrict__ x,
               double2* __restrict__ part, const int* __restrict__ skip) {
  if (skip && *skip) return;
  using G = SymGemvT<T2>;
  using R = typename G::R;
  using V = typename G::V;
  constexpr int CPV = G::CPV, RG = G::RG;
  constexpr int EV = kSymTile / (32 * CPV);  // 16-byte loads per lane per row
  __shared__ R sXI[2 * kSymTile];            // x_I (re, im), zero past dim
  __shared__ R sCol[DENSE ? 1 : kSymWarps][2 * kSymTile];
  const int2 it = items[blockIdx.x];
  const int I = it.x, J = it.y;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int rowI0 = I * kSymTile, colJ0 = J * kSymTile;
  if (tid < kSymTile) {
    const int r = rowI0 + tid;
    const double2 v = r < dim ? x[r] : make_double2(0.0, 0.0);
    sXI[2 * tid] = (R)v.x;
    sXI[2 * tid + 1] = (R)v.y;
  }
  // x_J at this lane's columns
  R xr[EV * CPV], xi[EV * CPV];
#pragma unroll
  for (int e = 0; e < EV; ++e)
#pragma unroll
    for (int h = 0; h < CPV; ++h) {
      const int c = colJ0 + CPV * (lane + 32 * e) + h;
      const double2 v = c < dim ? x[c] : make_double2(0.0, 0.0);
      xr[e * CPV + h] = (R)v.x;
      xi[e * CPV + h] = (R)v.y;
    }
  __syncthreads();
  R cr[EV * CPV], ci[EV * CPV];
#pragma unroll
  for (int q = 0; q < EV * CPV; ++q) cr[q] = ci[q] = (R)0;
  const bool offdiag = !DENSE && I != J;
  // the block's first vector and the row pitch in 16-byte vectors
  const V* tile = DENSE ? reinterpret_cast<const V*>(A + (size_t)rowI0 * ld + colJ0)
                        : reinterpret_cast<const V*>(A + sym_tile_offset(I, J, nt) *
                                                             (size_t)(kSymTile * kSymTile));
  const size_t pitch = DENSE ? ld / CPV : (size_t)(kSymTile / CPV);
  // DENSE: this lane's vectors that lie inside the row pitch (ld is a
  // multiple of 16 complex entries, so a vector is inside or past it whole)
  bool vec_ok[EV];
#pragma unroll
  for (int e = 0; e < EV; ++e)
    vec_ok[e] = !DENSE || (size_t)colJ0 + (size_t)(CPV * (lane + 32 * e)) < ld;
  const int r_begin = warp * kSymRowsPerWarp;
  double2* slotJ = part + (size_t)J * dim;  // row side of this tile
#pragma unroll 1
  for (int g8 = 0; g8 < kSymRowsPerWarp; g8 += 8) {
    R red[16];
#pragma unroll
    for (int k0 = 0; k0 < 8; k0 += RG) {
      V v[RG][EV];
#pragma unroll
      for (int k = 0; k < RG; ++k) {
        const int lr = r_begin + g8 + k0 + k;
        const bool row_ok = !DENSE || rowI0 + lr < dim;
#pragma unroll
        for (int e = 0; e < EV; ++e)
          v[k][e] = (row_ok && vec_ok[e]) ? __ldcs(&tile[(size_t)lr * pitch + lane + 32 * e])
                                          : V{};
      }
#pragma unroll
      for (int k = 0; k < RG; ++k) {
        const int lr = r_begin + g8 + k0 + k;
        const R ar = sXI[2 * lr], ai = sXI[2 * lr + 1];
        R sr = (R)0, si = (R)0;
#pragma unroll
        for (int e = 0; e < EV; ++e)
#pragma unroll
          for (int h = 0; h < CPV; ++h) {
            const T2 a = G::get(v[k][e], h);
            const int q = e * CPV + h;
            sr += (R)a.x * xr[q] - (R)a.y * xi[q];
            si += (R)a.x * xi[q] + (R)a.y * xr[q];
            cr[q] += (R)a.x * ar - (R)a.y * ai;
            ci[q] += (R)a.x * ai + (R)a.y * ar;
          }
        red[2 * (k0 + k)] = sr;
        red[2 * (k0 + k) + 1] = si;
      }
    }
    sym_transpose_reduce16(red, lane);
    if ((lane & 1) == 0) {
      const int vidx = 8 * ((lane >> 4) & 1) + 4 * ((lane >> 3) & 1) + 2 * ((lane >> 2) & 1) +
                       ((lane >> 1) & 1);
      const int row = rowI0 + r_begin + g8 + (vidx >> 1);
      if (row < dim) reinterpret_cast<double*>(slotJ + row)[vidx & 1] = (double)red[0];
    }
  }
  // a diagonal tile is stored whole, and dense rows have no column side
  if constexpr (!DENSE) {
    if (!offdiag) return;
#pragma unroll
    for (int e = 0; e < EV; ++e)
#pragma unroll
      for (int h = 0; h < CPV; ++h) {
        const int c = CPV * (lane + 32 * e) + h, q = e * CPV + h;
        sCol[warp][2 * c] = cr[q];
        sCol[warp][2 * c + 1] = ci[q];
      }
    __syncthreads();
    if (tid < kSymTile) {
      const int row = colJ0 + tid;
      if (row < dim) {
        double sr = 0.0, si = 0.0;
#pragma unroll
        for (int w = 0; w < kSymWarps; ++w) {
          sr += (double)sCol[w][2 * tid];
          si += (double)sCol[w][2 * tid + 1];
        }
        part[(size_t)I * dim + row] = make_double2(sr, si);
      }
    }
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

// The work list of a tile product and its per-block partial sums: the
// stored tiles I <= J (symmetric storage) or every block (I, J) of the
// nt x nt grid (dense rows).
lum_status CachedOperator::tile_blocks(bool upper) {
  std::vector<int2> it;
  for (int I = 0; I < nt; ++I)
    for (int J = upper ? I : 0; J < nt; ++J) it.push_back(make_int2(I, J));
  LUM_TRY(tile_items.alloc(sizeof(int2) * it.size()));
  LUM_TRY_CUDA(cudaMemcpy(tile_items.p, it.data(), sizeof(int2) * it.size(),
                          cudaMemcpyHostToDevice));
  LUM_TRY(tile_part.alloc(sizeof(double2) * (size_t)nt * dim));
  return LUM_OK;
}

lum_status CachedOperator::allocate(int dim_, int precision_, bool packed_) {
  dim = dim_;
  precision = precision_;
  packed = packed_;
  if (packed) {
    if (dim % 3 != 0) {
      set_error("symmetric tile storage needs whole 3x3 dipole blocks (dim %d)", dim);
      return LUM_ERR_INVALID;
    }
    nt = (dim + kSymTile - 1) / kSymTile;
    const size_t tiles = (size_t)nt * (nt + 1) / 2;
    const size_t es = (precision == LUM_FP32) ? sizeof(float2) : sizeof(double2);
    ld = 0;
    LUM_TRY(A.alloc(es * tiles * kSymTile * kSymTile));
    LUM_TRY_CUDA(cudaMemset(A.p, 0, A.bytes));
    LUM_TRY(tile_blocks(true));
    tc.release();
    gemv_chunks = 0;
    return LUM_OK;
  }
  nt = (dim + kSymTile - 1) / kSymTile;
  tile_items.release();
  tile_part.release();
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
  if (packed) {
    if (g.has_lattice || g.has_substrate || g.has_somm) {
      set_error("symmetric tile storage needs a free-space system (no lattice sum, no "
                "substrate)");
      return LUM_ERR_INVALID;
    }
    if (3 * n != dim) {
      set_error("symmetric tile storage of dimension %d for %d dipoles", dim, n);
      return LUM_ERR_INVALID;
    }
    const dim3 grid(nt, nt);
    if (precision == LUM_FP32)
      assemble_sym_tiles<float2><<<grid, 256, 0, st>>>(n, nt, g.pos64.as<double4>(),
                                                       g.inv_alpha.as<double2>(), g.k,
                                                       A.as<float2>());
    else
      assemble_sym_tiles<double2><<<grid, 256, 0, st>>>(n, nt, g.pos64.as<double4>(),
                                                        g.inv_alpha.as<double2>(), g.k,
                                                        A.as<double2>());
    LUM_CHECK_LAUNCH();
    if (g.ell_w > 0) {
      const int total = n * g.ell_w;
      if (precision == LUM_FP32)
        assemble_sym_fcd<float2><<<(total + 255) / 256, 256, 0, st>>>(
            n, nt, g.ell_w, g.near_j.as<int>(), g.fcd64.as<double2>(), A.as<float2>());
      else
        assemble_sym_fcd<double2><<<(total + 255) / 256, 256, 0, st>>>(
            n, nt, g.ell_w, g.near_j.as<int>(), g.fcd64.as<double2>(), A.as<double2>());
      LUM_CHECK_LAUNCH();
    }
    return LUM_OK;
  }
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
  if (packed) {
    const unsigned tiles = (unsigned)((size_t)nt * (nt + 1) / 2);
    if (precision == LUM_FP32)
      gemv_sym_tiles<float2, false><<<tiles, kSymWarps * 32, 0, st>>>(
          dim, nt, ld, A.as<float2>(), tile_items.as<int2>(), x, tile_part.as<double2>(), skip);
    else
      gemv_sym_tiles<double2, false><<<tiles, kSymWarps * 32, 0, st>>>(
          dim, nt, ld, A.as<double2>(), tile_items.as<int2>(), x, tile_part.as<double2>(), skip);
    LUM_CHECK_LAUNCH();
    gemv_reduce<<<(dim + 255) / 256, 256, 0, st>>>(dim, nt, tile_part.as<double2>(), y, skip);
    LUM_CHECK_LAUNCH();
    return LUM_OK;
  }
  // Dense rows: the block product (x_J held in registers per block, FP32
  // arithmetic for FP32 storage) unless LUMINA_DENSE_GEMV=rows selects the
  // row-chunk GEMV below.
  static const bool rows_gemv = [] {
    const char* e = std::getenv("LUMINA_DENSE_GEMV");
    return e && std::string(e) == "rows";
  }();
  if (!rows_gemv) {
    if (!tile_items.p) LUM_TRY(tile_blocks(false));
    const unsigned blocks = (unsigned)((size_t)nt * nt);
    if (precision == LUM_FP32)
      gemv_sym_tiles<float2, true><<<blocks, kSymWarps * 32, 0, st>>>(
          dim, nt, ld, A.as<float2>(), tile_items.as<int2>(), x, tile_part.as<double2>(), skip);
    else
      gemv_sym_tiles<double2, true><<<blocks, kSymWarps * 32, 0, st>>>(
          dim, nt, ld, A.as<double2>(), tile_items.as<int2>(), x, tile_part.as<double2>(), skip);
    LUM_CHECK_LAUNCH();
    gemv_reduce<<<(dim + 255) / 256, 256, 0, st>>>(dim, nt, tile_part.as<double2>(), y, skip);
    LUM_CHECK_LAUNCH();
    return LUM_OK;
  }
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
  if (packed) {
    // one tile product per vector; the tensor-core product reads dense rows
    if (method == LUM_MATMUL_TENSOR) {
      set_error("the tensor-core product needs dense matrix storage, not symmetric tiles");
      return LUM_ERR_INVALID;
    }
    if (sc != 1) {
      set_error("a symmetric-tile matrix takes its vectors back to back (one vector, or "
                "lum_session_matmul_vectors)");
      return LUM_ERR_INVALID;
    }
    for (int r = 0; r < nrhs; ++r) LUM_TRY(apply(X + r * sr, Y + r * sr, st));
    return LUM_OK;
  }
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
