// pairs_f64_sym.cuh -- FP64 dense pair kernels that evaluate each unordered
// pair once (the FP64 counterpart of pairs_f32_sym.cuh).
//
// G(r_i - r_j) = G(r_j - r_i) = G^T (greens.rs:34-71), so the pair scalars
// (A, B', d) -- one rsqrt and one sincos in FP64 (the table-driven sincos of
// device_sincos.cuh) -- serve
// both y_i += G x_j and y_j += G x_i.  The FP64 pipe is the bound; halving
// the transcendental sequences per ordered pair is the point.
//
// Work: the superblock pairs (I, J), I <= J, of kSymRows rows, as in the
// FP32 scheme.  A CTA has kSymRows threads, one row of I each, with its
// position, moments x_i and row sums in registers.  The sources of J are
// staged 32 at a time in shared memory; in step s lane l pairs its row with
// source (l + s) mod 32 and passes its source-side sums to lane l - 1 after
// the step, so after 32 steps lane l holds source l's sums over the warp's
// 32 rows.  The warps' sums are folded in pairs and added in a fixed order.
// NV = 2 contracts the same tensor scalars with two vectors (forward +
// adjoint, two polarisations).
//
// Output (deterministic, no atomics): slot[S][3i + c] as in the FP32 scheme.
// The diagonal item (I, I) takes only pairs j > i; the source-side sum of
// source j there belongs to row j of the same item, so it is handed to the
// thread that owns row j through shared memory and added to its row sum
// before the single store of slot I.
#pragma once

#include "device_sincos.cuh"

namespace lum {

constexpr int kSym64Threads = kSymRows;  // one row per thread

template <int NV, bool DIAG>
__device__ __forceinline__ void sym64_superblock_pair_t(
    int n, const double4* __restrict__ pos, const double2* __restrict__ xa_v,
    const double2* __restrict__ xb_v, double k, double inv_k, double s0, int I, int J,
    double2* __restrict__ slots_a, double2* __restrict__ slots_b, double4* sP,
    double2 (*sX)[3 * NV], double2 (*sAcc)[32][3 * NV], double2 (*sRed)[3 * NV],
    const double2* sTab) {
  constexpr int kWarps = kSym64Threads / 32;
  constexpr int kHalf = kWarps / 2;
  const double2* xv[2] = {xa_v, xb_v};
  double2* sl_v[2] = {slots_a, slots_b};
  constexpr bool diag = DIAG;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t n3 = 3 * (size_t)n;

  // this thread's row; a row past n sits far away with x = 0 and is never written
  const int i = I * kSymRows + tid;
  const bool vi = i < n;
  const double4 ri = vi ? pos[i] : make_double4(2e8, 2e8, 2e8, 0.0);
  double2 X[NV][3];
  double acc[NV][6];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
#pragma unroll
    for (int c = 0; c < 3; ++c) X[v][c] = vi ? xv[v][3 * (size_t)i + c] : make_double2(0.0, 0.0);
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[v][c] = 0.0;
  }

  const int j_base = J * kSymRows;
  const int ngroups = kSymRows / 32;
  for (int g = 0; g < ngroups; ++g) {
    const int jg = j_base + 32 * g;
    if (jg >= n) break;  // CTA-uniform
    __syncthreads();     // the previous group's sources and sums are consumed
    if (tid < 32) {
      const int j = jg + tid;
      sP[tid] = j < n ? pos[j] : make_double4(1e8, 1e8, 1e8, 0.0);
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int c = 0; c < 3; ++c)
          sX[tid][3 * v + c] = j < n ? xv[v][3 * (size_t)j + c] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    double sacc[NV][6];  // source-side sums of source (lane + s) mod 32
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int c = 0; c < 6; ++c) sacc[v][c] = 0.0;
#pragma unroll 1
    for (int s = 0; s < 32; ++s) {
      const int src = (lane + s) & 31;
      const double4 pj = sP[src];
      const double dx = ri.x - pj.x, dy = ri.y - pj.y, dz = ri.z - pj.z;
      double r2 = dx * dx + dy * dy + dz * dz;
      const bool drop = diag && !(jg + src > i);  // each unordered pair once: j > i
      if (drop) r2 = 1.0;
      const double ir = rsqrt(r2);
      const double Rr = r2 * ir;
      const double u = ir * inv_k;
      const double u2 = u * u;
      double sn, cs;
      sincos_tab(k * Rr, sTab, &sn, &cs);
      const double su = drop ? 0.0 : s0 * u;
      const double pr = su * cs, pi = su * sn;
      const double ar = 1.0 - u2;
      const double Ar = pr * ar - pi * u, Ai = pr * u + pi * ar;
      const double br = 3.0 * u2 - 1.0, bi = -3.0 * u;
      const double ir2 = ir * ir;
      const double Br = (pr * br - pi * bi) * ir2, Bi = (pr * bi + pi * br) * ir2;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        {  // row side: y_i += A x_j + B' d (d . x_j)
          const double2 xa = sX[src][3 * v], xb = sX[src][3 * v + 1], xc = sX[src][3 * v + 2];
          const double dxr = dx * xa.x + dy * xb.x + dz * xc.x;
          const double dxi = dx * xa.y + dy * xb.y + dz * xc.y;
          const double tr = Br * dxr - Bi * dxi, ti = Br * dxi + Bi * dxr;
          acc[v][0] += Ar * xa.x - Ai * xa.y + tr * dx;
          acc[v][1] += Ar * xa.y + Ai * xa.x + ti * dx;
          acc[v][2] += Ar * xb.x - Ai * xb.y + tr * dy;
          acc[v][3] += Ar * xb.y + Ai * xb.x + ti * dy;
          acc[v][4] += Ar * xc.x - Ai * xc.y + tr * dz;
          acc[v][5] += Ar * xc.y + Ai * xc.x + ti * dz;
        }
        {  // source side: y_j += A x_i + B' d (d . x_i), the same A, B', d
          const double dxr = dx * X[v][0].x + dy * X[v][1].x + dz * X[v][2].x;
          const double dxi = dx * X[v][0].y + dy * X[v][1].y + dz * X[v][2].y;
          const double tr = Br * dxr - Bi * dxi, ti = Br * dxi + Bi * dxr;
          sacc[v][0] += Ar * X[v][0].x - Ai * X[v][0].y + tr * dx;
          sacc[v][1] += Ar * X[v][0].y + Ai * X[v][0].x + ti * dx;
          sacc[v][2] += Ar * X[v][1].x - Ai * X[v][1].y + tr * dy;
          sacc[v][3] += Ar * X[v][1].y + Ai * X[v][1].x + ti * dy;
          sacc[v][4] += Ar * X[v][2].x - Ai * X[v][2].y + tr * dz;
          sacc[v][5] += Ar * X[v][2].y + Ai * X[v][2].x + ti * dz;
        }
      }
      // pass each source's sums on: lane l takes those of source (l + s + 1)
      const int from = (lane + 1) & 31;
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int c = 0; c < 6; ++c) sacc[v][c] = __shfl_sync(0xffffffffu, sacc[v][c], from);
    }
    // lane l now holds source l's sums over the warp's 32 rows; fold warps
    // w and w + kHalf into slot w (fixed order), then add the slots
    if (warp >= kHalf) {
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int c = 0; c < 3; ++c)
          sAcc[warp - kHalf][lane][3 * v + c] = make_double2(sacc[v][2 * c], sacc[v][2 * c + 1]);
    }
    __syncthreads();
    if (warp < kHalf) {
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double2 o = sAcc[warp][lane][3 * v + c];
          sAcc[warp][lane][3 * v + c] = make_double2(sacc[v][2 * c] + o.x, sacc[v][2 * c + 1] + o.y);
        }
    }
    __syncthreads();
    if (tid < 32 * 3 * NV) {
      const int sl = tid / (3 * NV), cv = tid % (3 * NV);
      double re = 0.0, im = 0.0;
#pragma unroll
      for (int w = 0; w < kHalf; ++w) {
        re += sAcc[w][sl][cv].x;
        im += sAcc[w][sl][cv].y;
      }
      const int j = jg + sl;
      if (diag)
        sRed[sl][cv] = make_double2(re, im);
      else if (j < n)
        sl_v[cv / 3][(size_t)I * n3 + 3 * (size_t)j + cv % 3] = make_double2(re, im);
    }
    if (diag) {  // rows 32 g .. 32 g + 31 of this item take their source-side sums
      __syncthreads();
      if (warp == g) {
#pragma unroll
        for (int v = 0; v < NV; ++v)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            acc[v][2 * c] += sRed[lane][3 * v + c].x;
            acc[v][2 * c + 1] += sRed[lane][3 * v + c].y;
          }
      }
    }
  }
  // row side: slot J for the row of I (diagonal: both sides)
  if (vi) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double2* dst = sl_v[v] + (size_t)J * n3 + 3 * (size_t)i;
#pragma unroll
      for (int c = 0; c < 3; ++c) dst[c] = make_double2(acc[v][2 * c], acc[v][2 * c + 1]);
    }
  }
}

// Diagonal and off-diagonal items as separate instantiations: the masking
// of the diagonal stays out of the off-diagonal step loop.
template <int NV>
__device__ __forceinline__ void sym64_superblock_pair(
    int n, const double4* __restrict__ pos, const double2* __restrict__ xa_v,
    const double2* __restrict__ xb_v, double k, double inv_k, double s0, int I, int J,
    double2* __restrict__ slots_a, double2* __restrict__ slots_b, double4* sP,
    double2 (*sX)[3 * NV], double2 (*sAcc)[32][3 * NV], double2 (*sRed)[3 * NV],
    const double2* sTab) {
  if (I == J)
    sym64_superblock_pair_t<NV, true>(n, pos, xa_v, xb_v, k, inv_k, s0, I, J, slots_a, slots_b,
                                      sP, sX, sAcc, sRed, sTab);
  else
    sym64_superblock_pair_t<NV, false>(n, pos, xa_v, xb_v, k, inv_k, s0, I, J, slots_a, slots_b,
                                       sP, sX, sAcc, sRed, sTab);
}

__global__ void __launch_bounds__(kSym64Threads, 1)
otf_pairs_f64_sym(int n, const double4* __restrict__ pos, const double2* __restrict__ x,
                  double k, double inv_k, double s0, const int2* __restrict__ items,
                  double2* __restrict__ slots, const int* __restrict__ skip) {
  if (skip && *skip) return;
  __shared__ double4 sP[32];
  __shared__ double2 sX[32][3];
  __shared__ double2 sAcc[kSym64Threads / 64][32][3];
  __shared__ double2 sRed[32][3];
  __shared__ double2 sTab[kScTab];
  sincos_table_stage(sTab);  // the first group's barrier precedes its use
  const int2 it = items[blockIdx.x];
  sym64_superblock_pair<1>(n, pos, x, nullptr, k, inv_k, s0, it.x, it.y, slots, nullptr, sP, sX,
                           sAcc, sRed, sTab);
}

// Two vectors; a vector whose skip flag is set is left out, with both set
// the kernel returns at once.
__global__ void __launch_bounds__(kSym64Threads, 1)
otf_pairs_f64_sym2(int n, const double4* __restrict__ pos, const double2* __restrict__ x,
                   const double2* __restrict__ x2, double k, double inv_k, double s0,
                   const int2* __restrict__ items, double2* __restrict__ slots,
                   double2* __restrict__ slots2, const int* __restrict__ skip,
                   const int* __restrict__ skip2) {
  const bool live = !(skip && *skip), live2 = !(skip2 && *skip2);
  if (!live && !live2) return;
  __shared__ double4 sP[32];
  __shared__ double2 sX[32][6];
  __shared__ double2 sAcc[kSym64Threads / 64][32][6];
  __shared__ double2 sRed[32][6];
  __shared__ double2 sTab[kScTab];
  sincos_table_stage(sTab);  // the first group's barrier precedes its use
  const int2 it = items[blockIdx.x];
  if (live && live2) {
    sym64_superblock_pair<2>(n, pos, x, x2, k, inv_k, s0, it.x, it.y, slots, slots2, sP, sX,
                             sAcc, sRed, sTab);
  } else {
    // the single-vector layout inside the same shared arrays
    sym64_superblock_pair<1>(n, pos, live ? x : x2, nullptr, k, inv_k, s0, it.x, it.y,
                             live ? slots : slots2, nullptr, sP,
                             reinterpret_cast<double2(*)[3]>(sX),
                             reinterpret_cast<double2(*)[32][3]>(sAcc),
                             reinterpret_cast<double2(*)[3]>(sRed), sTab);
  }
}

}  // namespace lum
