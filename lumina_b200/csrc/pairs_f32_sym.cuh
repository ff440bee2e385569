// pairs_f32_sym.cuh -- FP32 dense pair kernels that evaluate each unordered
// pair once.
//
// The point-dipole tensor is symmetric and even in the displacement
// (G(r_i - r_j) = G(r_j - r_i) = G^T, greens.rs:34-71), so one evaluation of
// the pair scalars (A, B', d) serves both y_i += G x_j and y_j += G x_i.  The
// shared part of a pair (~27 FP32 operations, rsqrt, sin, cos) is done once
// per unordered pair instead of once per ordered pair; each direction keeps
// its own 28-operation contraction per vector.
//
// Work: superblocks of kSymRows rows.  A CTA takes one superblock pair
// (I, J), I <= J.  A thread holds 2*RP rows of I, packed in pairs into the
// two halves of a float2 as in pairs_f32x2.cuh (warp w, row pair p: rows
// I*kSymRows + 64*RP*w + 64*p + {lane, lane + 32}), with their positions,
// moments x_i and row sums in registers; the CTA has kSymRows / (2*RP)
// threads (RP = 4: 64).  The sources of J are staged 32 at a time in shared
// memory; in step s of a group, lane l pairs its rows with source (l + s) mod 32
// (conflict-free: consecutive lanes read consecutive entries).  The
// source-side sums travel with the sources: after each step every lane
// passes its source accumulator (summed over its 2*RP rows) to lane l - 1,
// so after 32 steps lane l holds the sum for source l over the warp's rows.
// The warps' sums are then added in warp order.  RP = 2 halves the shared
// loads and shuffles per pair and gives each step two independent tensor
// evaluations to interleave, at the cost of registers; UNR = 2 unrolls the
// step loop so that one step's shuffles overlap the next step's tensor.
//
// NV = 2 applies the operator to two vectors at once (forward + adjoint,
// two polarisations): the tensor scalars are evaluated once per unordered
// pair and contracted with both vectors on both sides.
//
// Output, deterministic and free of atomics: slot[S][3i + c] is the sum over
// sources of superblock S for row i.  Item (I, J), I < J, writes slot J for
// the rows of I (row side) and slot I for the rows of J (source side).  The
// diagonal item (I, I) takes only pairs j > i; there the source-side sum of
// a source belongs to a row of the same item, so after each source group it
// is handed through shared memory to the thread that owns that row and added
// to its row sum before the single store of slot I.  Every (slot, row) is
// written exactly once; the epilogue sums the slots in order.
#pragma once

namespace lum {

constexpr int kSymRows = 512;   // rows (and sources) per superblock

template <int RP>
struct SymShape {
  static constexpr int kThreads = kSymRows / (2 * RP);
  static constexpr int kWarps = kThreads / 32;
};

// Scalars of the packed row pair (OX, OY, OZ [+ lo]) against one staged
// source: displacement d and the tensor coefficients A, B' (with -Ai, -Bi).
template <bool FAST, bool LOFREE>
__device__ __forceinline__ void sym_pair_tensor(
    float2 OX, float2 OY, float2 OZ, float2 LX, float2 LY, float2 LZ, const float4& S0,
    const float4& S1, const float4& S4, const float4& S5, bool diag, int j, int ia, int ib,
    float2 kk2, float2 s02, float2& dx, float2& dy, float2& dz, float2& Ar, float2& Ai,
    float2& nAi, float2& Br, float2& Bi, float2& nBi) {
  const float2 m3 = make_float2(-3.0f, -3.0f), m1 = make_float2(-1.0f, -1.0f),
               one = make_float2(1.0f, 1.0f);
  dx = sub2(OX, lo2(S0));
  dy = sub2(OY, hi2(S0));
  dz = sub2(OZ, lo2(S1));
  if (!LOFREE) {
    dx = add2(dx, sub2(LX, hi2(S4)));
    dy = add2(dy, sub2(LY, lo2(S5)));
    dz = add2(dz, sub2(LZ, hi2(S5)));
  }
  float2 r2 = fma2(dx, dx, fma2(dy, dy, mul2(dz, dz)));
  float2 keep = one;
  if (diag) {  // each unordered pair once: j > i; the self pair is masked
    if (!(j > ia)) { keep.x = 0.f; if (r2.x < 1e-30f) r2.x = 1.f; }
    if (!(j > ib)) { keep.y = 0.f; if (r2.y < 1e-30f) r2.y = 1.f; }
  }
  const float2 kr2 = mul2(r2, kk2);
  const float2 u = make_float2(rsqrtf(kr2.x), rsqrtf(kr2.y));
  const float2 kR = mul2(kr2, u);
  float2 sn, cs;
  if (FAST) {
    __sincosf(kR.x, &sn.x, &cs.x);
    __sincosf(kR.y, &sn.y, &cs.y);
  } else {
    sincosf(kR.x, &sn.x, &cs.x);
    sincosf(kR.y, &sn.y, &cs.y);
  }
  const float2 u2 = mul2(u, u);
  float2 q = mul2(s02, u);
  if (diag) q = mul2(q, keep);
  const float2 pr = mul2(q, cs), pi = mul2(q, sn);
  const float2 ar = sub2(one, u2);
  Ar = sub2(mul2(pr, ar), mul2(pi, u));
  Ai = fma2(pr, u, mul2(pi, ar));
  const float2 ir2 = mul2(u2, kk2);
  Br = mul2(fma2(Ar, m3, add2(pr, pr)), ir2);
  Bi = mul2(fma2(Ai, m3, add2(pi, pi)), ir2);
  nAi = mul2(Ai, m1);
  nBi = mul2(Bi, m1);
}

// acc += A v + B' d (d . v) for the packed vector v = (v0r, v0i, v1r, v1i, v2r, v2i).
__device__ __forceinline__ void sym_contract(float2 dx, float2 dy, float2 dz, float2 Ar,
                                             float2 Ai, float2 nAi, float2 Br, float2 Bi,
                                             float2 nBi, float2 v0r, float2 v0i, float2 v1r,
                                             float2 v1i, float2 v2r, float2 v2i,
                                             float2 (&acc)[6]) {
  const float2 dvr = fma2(dx, v0r, fma2(dy, v1r, mul2(dz, v2r)));
  const float2 dvi = fma2(dx, v0i, fma2(dy, v1i, mul2(dz, v2i)));
  const float2 tr = fma2(Br, dvr, mul2(nBi, dvi));
  const float2 ti = fma2(Br, dvi, mul2(Bi, dvr));
  acc[0] = fma2(tr, dx, fma2(Ar, v0r, fma2(nAi, v0i, acc[0])));
  acc[1] = fma2(ti, dx, fma2(Ar, v0i, fma2(Ai, v0r, acc[1])));
  acc[2] = fma2(tr, dy, fma2(Ar, v1r, fma2(nAi, v1i, acc[2])));
  acc[3] = fma2(ti, dy, fma2(Ar, v1i, fma2(Ai, v1r, acc[3])));
  acc[4] = fma2(tr, dz, fma2(Ar, v2r, fma2(nAi, v2i, acc[4])));
  acc[5] = fma2(ti, dz, fma2(Ar, v2i, fma2(Ai, v2r, acc[5])));
}

// The work of one superblock pair for NV vectors (DIAG: the item I == J).
// Slot S of a vector starts at slots + S * slot_stride (3n for one system; 3N
// for a batch, whose systems share the slot layout of the global dipole
// range).  Shared memory comes from the caller: sS [6 + 3 (NV - 1)][32]
// staged sources, sAcc [warps][32][6 NV] per-warp source sums, sRed
// [32][6 NV] the diagonal hand-off.
template <bool FAST, bool LOFREE, int RP, int NV, int UNR, bool DIAG>
__device__ __forceinline__ void sym_superblock_pair_t(
    int n, const float4* __restrict__ obs_hi, const float4* __restrict__ obs_lo,
    const double2* __restrict__ xa_v, const double2* __restrict__ xb_v, float k, float s0,
    int I, int J, float2* __restrict__ slots_a, float2* __restrict__ slots_b, size_t slot_stride,
    float4 (*sS)[32], float2* sAcc, float* sRed) {
  constexpr int kThreads = SymShape<RP>::kThreads, kWarps = SymShape<RP>::kWarps;
  constexpr int W = 6 * NV;  // floats of source-side sum per source
  const double2* xv[2] = {xa_v, xb_v};
  float2* sl_v[2] = {slots_a, slots_b};
  constexpr bool diag = DIAG;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // rows of this thread: pair p holds a = lane, b = lane + 32 of its 64;
  // rows past n sit far away with x = 0 and are never written
  const float4 far4 = make_float4(2e8f, 2e8f, 2e8f, 0.f), zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
  int ia[RP], ib[RP];
  float2 OX[RP], OY[RP], OZ[RP], LX[RP], LY[RP], LZ[RP];
  float2 X[RP][NV][6];  // (x0r, x0i, x1r, x1i, x2r, x2i) of rows a / b
  float2 acc[RP][NV][6];
#pragma unroll
  for (int p = 0; p < RP; ++p) {
    ia[p] = I * kSymRows + 64 * (RP * warp + p) + lane;
    ib[p] = ia[p] + 32;
    const bool va = ia[p] < n, vb = ib[p] < n;
    const float4 ha = va ? obs_hi[ia[p]] : far4, hb = vb ? obs_hi[ib[p]] : far4;
    OX[p] = make_float2(ha.x, hb.x);
    OY[p] = make_float2(ha.y, hb.y);
    OZ[p] = make_float2(ha.z, hb.z);
    LX[p] = LY[p] = LZ[p] = make_float2(0.f, 0.f);
    if (!LOFREE) {
      const float4 la = va ? obs_lo[ia[p]] : zero4, lb = vb ? obs_lo[ib[p]] : zero4;
      LX[p] = make_float2(la.x, lb.x);
      LY[p] = make_float2(la.y, lb.y);
      LZ[p] = make_float2(la.z, lb.z);
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double2 xa = va ? xv[v][3 * (size_t)ia[p] + c] : make_double2(0.0, 0.0);
        const double2 xb = vb ? xv[v][3 * (size_t)ib[p] + c] : make_double2(0.0, 0.0);
        X[p][v][2 * c] = make_float2((float)xa.x, (float)xb.x);
        X[p][v][2 * c + 1] = make_float2((float)xa.y, (float)xb.y);
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) acc[p][v][c] = make_float2(0.f, 0.f);
    }
  }

  const float2 kk2 = make_float2(k * k, k * k), s02 = make_float2(s0, s0);
  const int j_base = J * kSymRows;
  const int ngroups = kSymRows / 32;
  for (int g = 0; g < ngroups; ++g) {
    const int jg = j_base + 32 * g;
    if (jg >= n) break;  // CTA-uniform
    __syncthreads();     // the previous group's sources and sums are consumed
    if (tid < 32) {
      const int j = jg + tid;
      float4 h = make_float4(1e8f, 1e8f, 1e8f, 0.f), l = zero4;
      float2 xa = make_float2(0.f, 0.f), xb = xa, xc = xa;
      if (j < n) {
        h = obs_hi[j];
        if (!LOFREE) l = obs_lo[j];
        const double2 a = xv[0][3 * (size_t)j], b = xv[0][3 * (size_t)j + 1],
                      c = xv[0][3 * (size_t)j + 2];
        xa = make_float2((float)a.x, (float)a.y);
        xb = make_float2((float)b.x, (float)b.y);
        xc = make_float2((float)c.x, (float)c.y);
      }
      sS[0][tid] = make_float4(h.x, h.x, h.y, h.y);
      sS[1][tid] = make_float4(h.z, h.z, xa.x, xa.x);
      sS[2][tid] = make_float4(xa.y, xa.y, xb.x, xb.x);
      sS[3][tid] = make_float4(xb.y, xb.y, xc.x, xc.x);
      sS[4][tid] = make_float4(xc.y, xc.y, l.x, l.x);
      sS[5][tid] = make_float4(l.y, l.y, l.z, l.z);
      if constexpr (NV == 2) {
        double2 a = make_double2(0.0, 0.0), b = a, c = a;
        if (j < n) {
          a = xv[1][3 * (size_t)j];
          b = xv[1][3 * (size_t)j + 1];
          c = xv[1][3 * (size_t)j + 2];
        }
        sS[6][tid] = make_float4((float)a.x, (float)a.x, (float)a.y, (float)a.y);
        sS[7][tid] = make_float4((float)b.x, (float)b.x, (float)b.y, (float)b.y);
        sS[8][tid] = make_float4((float)c.x, (float)c.x, (float)c.y, (float)c.y);
      }
    }
    __syncthreads();
    float2 sacc[NV][6];  // source-side sums of source (lane + s) mod 32, halves a / b
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int c = 0; c < 6; ++c) sacc[v][c] = make_float2(0.f, 0.f);
#pragma unroll UNR
    for (int s = 0; s < 32; ++s) {
      const int src = (lane + s) & 31;
      const float4 S0 = sS[0][src], S1 = sS[1][src], S2 = sS[2][src], S3 = sS[3][src],
                   S4 = sS[4][src];
      float4 S5 = zero4;
      if (!LOFREE) S5 = sS[5][src];
      const int j = jg + src;
      const float2 x0r = hi2(S1), x0i = lo2(S2), x1r = hi2(S2), x1i = lo2(S3), x2r = hi2(S3),
                   x2i = lo2(S4);
      float4 S6 = zero4, S7 = zero4, S8 = zero4;
      if constexpr (NV == 2) {
        S6 = sS[6][src];
        S7 = sS[7][src];
        S8 = sS[8][src];
      }
#pragma unroll
      for (int p = 0; p < RP; ++p) {
        float2 dx, dy, dz, Ar, Ai, nAi, Br, Bi, nBi;
        sym_pair_tensor<FAST, LOFREE>(OX[p], OY[p], OZ[p], LX[p], LY[p], LZ[p], S0, S1, S4, S5,
                                      diag, j, ia[p], ib[p], kk2, s02, dx, dy, dz, Ar, Ai, nAi,
                                      Br, Bi, nBi);
        // row side: y_i += A x_j + B' d (d . x_j)
        sym_contract(dx, dy, dz, Ar, Ai, nAi, Br, Bi, nBi, x0r, x0i, x1r, x1i, x2r, x2i,
                     acc[p][0]);
        if constexpr (NV == 2)
          sym_contract(dx, dy, dz, Ar, Ai, nAi, Br, Bi, nBi, lo2(S6), hi2(S6), lo2(S7), hi2(S7),
                       lo2(S8), hi2(S8), acc[p][1]);
        // source side: y_j += A x_i + B' d (d . x_i), the same A, B', d
#pragma unroll
        for (int v = 0; v < NV; ++v)
          sym_contract(dx, dy, dz, Ar, Ai, nAi, Br, Bi, nBi, X[p][v][0], X[p][v][1],
                       X[p][v][2], X[p][v][3], X[p][v][4], X[p][v][5], sacc[v]);
      }
      // pass each source's sums on: lane l takes those of source (l + s + 1)
      const int from = (lane + 1) & 31;
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          sacc[v][c].x = __shfl_sync(0xffffffffu, sacc[v][c].x, from);
          sacc[v][c].y = __shfl_sync(0xffffffffu, sacc[v][c].y, from);
        }
    }
    // lane l now holds source l's sums over the warp's rows (halves a / b)
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int c = 0; c < 6; ++c) sAcc[(warp * 32 + lane) * W + 6 * v + c] = sacc[v][c];
    __syncthreads();
    for (int q = tid; q < 32 * W; q += kThreads) {
      const int sl = q / W, cv = q % W;
      float val = 0.f;
#pragma unroll
      for (int w = 0; w < kWarps; ++w) {
        const float2 t = sAcc[(w * 32 + sl) * W + cv];
        val += t.x + t.y;
      }
      const int j = jg + sl;
      if (diag) {
        sRed[sl * W + cv] = val;
      } else if (j < n) {
        float* dst =
            reinterpret_cast<float*>(sl_v[cv / 6] + (size_t)I * slot_stride + 3 * (size_t)j);
        dst[cv % 6] = val;  // 2 * component + (0 re | 1 im)
      }
    }
    if (diag) {  // rows 32 g .. 32 g + 31 of this item take their source-side sums
      __syncthreads();
      const int lr0 = 32 * g;
      if (warp == lr0 / (64 * RP)) {
        const int pw = (lr0 % (64 * RP)) / 64, half = (lr0 % 64) / 32;
#pragma unroll
        for (int p = 0; p < RP; ++p)
          if (p == pw) {
#pragma unroll
            for (int v = 0; v < NV; ++v)
#pragma unroll
              for (int c = 0; c < 6; ++c) {
                const float t = sRed[lane * W + 6 * v + c];
                if (half == 0)
                  acc[p][v][c].x += t;
                else
                  acc[p][v][c].y += t;
              }
          }
      }
    }
  }
  // row side: slot J for the rows of I (diagonal: both sides)
#pragma unroll
  for (int p = 0; p < RP; ++p)
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      if (ia[p] < n) {
        float2* dst = sl_v[v] + (size_t)J * slot_stride + 3 * (size_t)ia[p];
#pragma unroll
        for (int c = 0; c < 3; ++c) dst[c] = make_float2(acc[p][v][2 * c].x, acc[p][v][2 * c + 1].x);
      }
      if (ib[p] < n) {
        float2* dst = sl_v[v] + (size_t)J * slot_stride + 3 * (size_t)ib[p];
#pragma unroll
        for (int c = 0; c < 3; ++c) dst[c] = make_float2(acc[p][v][2 * c].y, acc[p][v][2 * c + 1].y);
      }
    }
}

// The diagonal items (one per superblock) and the off-diagonal ones are
// separate instantiations, so the masking of the diagonal stays out of the
// off-diagonal step loop.
template <bool FAST, bool LOFREE, int RP, int NV, int UNR = 1>
__device__ __forceinline__ void sym_superblock_pair(
    int n, const float4* __restrict__ obs_hi, const float4* __restrict__ obs_lo,
    const double2* __restrict__ xa_v, const double2* __restrict__ xb_v, float k, float s0,
    int I, int J, float2* __restrict__ slots_a, float2* __restrict__ slots_b, size_t slot_stride,
    float4 (*sS)[32], float2* sAcc, float* sRed) {
  if (I == J)
    sym_superblock_pair_t<FAST, LOFREE, RP, NV, UNR, true>(n, obs_hi, obs_lo, xa_v, xb_v, k, s0,
                                                           I, J, slots_a, slots_b, slot_stride,
                                                           sS, sAcc, sRed);
  else
    sym_superblock_pair_t<FAST, LOFREE, RP, NV, UNR, false>(n, obs_hi, obs_lo, xa_v, xb_v, k, s0,
                                                            I, J, slots_a, slots_b, slot_stride,
                                                            sS, sAcc, sRed);
}

template <bool FAST, bool LOFREE, int MINB, int RP, int UNR = 1>
__global__ void __launch_bounds__(SymShape<RP>::kThreads, MINB)
otf_pairs_f32_sym(int n, const float4* __restrict__ obs_hi, const float4* __restrict__ obs_lo,
                  const double2* __restrict__ x, float k, float s0,
                  const int2* __restrict__ items, float2* __restrict__ slots,
                  const int* __restrict__ skip) {
  if (skip && *skip) return;
  __shared__ float4 sS[6][32];
  __shared__ float2 sAcc[SymShape<RP>::kWarps * 32 * 6];
  __shared__ float sRed[32 * 6];
  const int2 it = items[blockIdx.x];
  sym_superblock_pair<FAST, LOFREE, RP, 1, UNR>(n, obs_hi, obs_lo, x, nullptr, k, s0, it.x,
                                                it.y, slots, nullptr, 3 * (size_t)n, sS, sAcc,
                                                sRed);
}

// Two vectors (see NV above).  A vector whose skip flag is set is left out;
// with both set the kernel returns at once.
template <bool FAST, bool LOFREE, int MINB, int RP, int UNR = 1>
__global__ void __launch_bounds__(SymShape<RP>::kThreads, MINB)
otf_pairs_f32_sym2(int n, const float4* __restrict__ obs_hi, const float4* __restrict__ obs_lo,
                   const double2* __restrict__ x, const double2* __restrict__ x2, float k,
                   float s0, const int2* __restrict__ items, float2* __restrict__ slots,
                   float2* __restrict__ slots2, const int* __restrict__ skip,
                   const int* __restrict__ skip2) {
  const bool live = !(skip && *skip), live2 = !(skip2 && *skip2);
  if (!live && !live2) return;
  __shared__ float4 sS[9][32];
  __shared__ float2 sAcc[SymShape<RP>::kWarps * 32 * 12];
  __shared__ float sRed[32 * 12];
  const int2 it = items[blockIdx.x];
  if (live && live2)
    sym_superblock_pair<FAST, LOFREE, RP, 2, UNR>(n, obs_hi, obs_lo, x, x2, k, s0, it.x, it.y,
                                                  slots, slots2, 3 * (size_t)n, sS, sAcc, sRed);
  else
    sym_superblock_pair<FAST, LOFREE, RP, 1, UNR>(n, obs_hi, obs_lo, live ? x : x2, nullptr, k,
                                                  s0, it.x, it.y, live ? slots : slots2, nullptr,
                                                  3 * (size_t)n, sS, sAcc, sRed);
}

}  // namespace lum
