// pairs_f32x2.cuh -- FP32 dense pair kernel with packed f32x2 arithmetic.
//
// Each thread owns 2*RP observer dipoles.  Rows are packed in pairs into the
// two halves of a float2, and every scalar step of the pair interaction runs
// as one sm_100 f32x2 instruction (__ffma2_rn / __fmul2_rn / __fadd2_rn) for
// both rows.  The kernel was issue-bound (~78 instructions per pair at 87 %
// issue utilisation); packing halves the issue count, so the FP32 pipe
// becomes the limit.  Only the rsqrt and sin/cos (MUFU) stay per row.
//
// Shared source tile, 6 x float4 per source, each value duplicated so that
// one broadcast LDS.128 yields two (v, v) pairs:
//   S0 = (hx,hx,hy,hy)  S1 = (hz,hz,x0r,x0r)  S2 = (x0i,x0i,x1r,x1r)
//   S3 = (x1i,x1i,x2r,x2r)  S4 = (x2i,x2i,lx,lx)  S5 = (ly,ly,lz,lz)
// LOFREE skips S5 and the lo terms when every centred position is exact in
// FP32 (lo == 0), e.g. a lattice whose coordinates are multiples of 2^-k.
//
// NR = 2 applies the operator to two right-hand sides at once (e.g. the
// forward and adjoint solves, or two polarisations): the tensor scalars A
// and B' are evaluated once per pair and contracted with both source
// vectors; the second vector adds three shared rows per source,
//   S6 = (y0r,y0r,y0i,y0i)  S7 = (y1r,y1r,y1i,y1i)  S8 = (y2r,y2r,y2i,y2i).
//
// The self pair (j == i) only occurs in the two tiles that hold the CTA's
// own rows; only those tiles run the masked loop.  The substrate image pass
// (IMAGE) masks pairs whose image distance is below 1e-10 nm (r^2 < 1e-20).
#pragma once

namespace lum {

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 lo2(const float4& v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4& v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b as one FMA: b * (-1) + a is exact-rounded like the subtraction
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}

template <bool FAST, bool IMAGE, bool LOFREE, bool CHECKED, int RP, int NR>
__device__ __forceinline__ void pair_tile_f32x2(
    const float4 (*__restrict__ sS)[kOtfBlock], int cnt, int jt, const int* irow,
    const float2* OX, const float2* OY, const float2* OZ, const float2* LX, const float2* LY,
    const float2* LZ, float2 (*acc)[6], float2 (*acc2)[6], float2 kk2, float2 s02) {
#pragma unroll 2
  for (int jj = 0; jj < cnt; ++jj) {
    const float4 S0 = sS[0][jj], S1 = sS[1][jj], S2 = sS[2][jj], S3 = sS[3][jj], S4 = sS[4][jj];
    float4 S5 = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!LOFREE) S5 = sS[5][jj];
    const float2 x0r = hi2(S1), x0i = lo2(S2), x1r = hi2(S2), x1i = lo2(S3), x2r = hi2(S3),
                 x2i = lo2(S4);
    float4 S6 = make_float4(0.f, 0.f, 0.f, 0.f), S7 = S6, S8 = S6;
    if constexpr (NR == 2) {
      S6 = sS[6][jj];
      S7 = sS[7][jj];
      S8 = sS[8][jj];
    }
    const float2 y0r = lo2(S6), y0i = hi2(S6), y1r = lo2(S7), y1i = hi2(S7), y2r = lo2(S8),
                 y2i = hi2(S8);
    const int j = jt + jj;
#pragma unroll
    for (int p = 0; p < RP; ++p) {
      float2 dx = sub2(OX[p], lo2(S0));
      float2 dy = sub2(OY[p], hi2(S0));
      float2 dz = sub2(OZ[p], lo2(S1));
      if (!LOFREE) {
        dx = add2(dx, sub2(LX[p], hi2(S4)));
        dy = add2(dy, sub2(LY[p], lo2(S5)));
        dz = add2(dz, sub2(LZ[p], hi2(S5)));
      }
      float2 r2 = fma2(dx, dx, fma2(dy, dy, mul2(dz, dz)));
      float2 keep = make_float2(1.0f, 1.0f);
      if (CHECKED) {
        const bool sx = IMAGE ? (r2.x < 1e-20f) : (j == irow[2 * p]);
        const bool sy = IMAGE ? (r2.y < 1e-20f) : (j == irow[2 * p + 1]);
        if (sx) { r2.x = 1.0f; keep.x = 0.0f; }
        if (sy) { r2.y = 1.0f; keep.y = 0.0f; }
      }
      const float2 kr2 = mul2(r2, kk2);                   // (k R)^2
      const float2 u = make_float2(rsqrtf(kr2.x), rsqrtf(kr2.y));  // 1/(kR)
      const float2 kR = mul2(kr2, u);                     // k R
      float2 sn, cs;
      if (FAST) {
        __sincosf(kR.x, &sn.x, &cs.x);
        __sincosf(kR.y, &sn.y, &cs.y);
      } else {
        sincosf(kR.x, &sn.x, &cs.x);
        sincosf(kR.y, &sn.y, &cs.y);
      }
      const float2 u2 = mul2(u, u);
      float2 q = mul2(s02, u);                           // k^3/(4 pi) u
      if (CHECKED) q = mul2(q, keep);
      const float2 pr = mul2(q, cs), pi = mul2(q, sn);   // pf = pr + i pi
      const float2 ar = sub2(make_float2(1.0f, 1.0f), u2);
      // A = pf a,  a = 1 - u^2 + i u
      const float2 Ar = sub2(mul2(pr, ar), mul2(pi, u));
      const float2 Ai = fma2(pr, u, mul2(pi, ar));
      // B' = pf b / R^2 with b = 3u^2 - 1 - 3iu = 2 - 3a, so B' = (2 pf - 3 A) ir^2,
      // ir^2 = u^2 k^2
      const float2 m3 = make_float2(-3.0f, -3.0f), m1 = make_float2(-1.0f, -1.0f);
      const float2 ir2 = mul2(u2, kk2);
      const float2 Br = mul2(fma2(Ar, m3, add2(pr, pr)), ir2);
      const float2 Bi = mul2(fma2(Ai, m3, add2(pi, pi)), ir2);
      // -Ai and -Bi turn the real parts of the complex products into one FMA
      // each (shared by every right-hand side)
      const float2 nAi = mul2(Ai, m1), nBi = mul2(Bi, m1);
      // d . x_j
      const float2 dxr = fma2(dx, x0r, fma2(dy, x1r, mul2(dz, x2r)));
      const float2 dxi = fma2(dx, x0i, fma2(dy, x1i, mul2(dz, x2i)));
      const float2 tr = fma2(Br, dxr, mul2(nBi, dxi));
      const float2 ti = fma2(Br, dxi, mul2(Bi, dxr));
      acc[p][0] = fma2(tr, dx, fma2(Ar, x0r, fma2(nAi, x0i, acc[p][0])));
      acc[p][1] = fma2(ti, dx, fma2(Ar, x0i, fma2(Ai, x0r, acc[p][1])));
      acc[p][2] = fma2(tr, dy, fma2(Ar, x1r, fma2(nAi, x1i, acc[p][2])));
      acc[p][3] = fma2(ti, dy, fma2(Ar, x1i, fma2(Ai, x1r, acc[p][3])));
      acc[p][4] = fma2(tr, dz, fma2(Ar, x2r, fma2(nAi, x2i, acc[p][4])));
      acc[p][5] = fma2(ti, dz, fma2(Ar, x2i, fma2(Ai, x2r, acc[p][5])));
      if constexpr (NR == 2) {
        const float2 dyr = fma2(dx, y0r, fma2(dy, y1r, mul2(dz, y2r)));
        const float2 dyi = fma2(dx, y0i, fma2(dy, y1i, mul2(dz, y2i)));
        const float2 ur = fma2(Br, dyr, mul2(nBi, dyi));
        const float2 ui = fma2(Br, dyi, mul2(Bi, dyr));
        acc2[p][0] = fma2(ur, dx, fma2(Ar, y0r, fma2(nAi, y0i, acc2[p][0])));
        acc2[p][1] = fma2(ui, dx, fma2(Ar, y0i, fma2(Ai, y0r, acc2[p][1])));
        acc2[p][2] = fma2(ur, dy, fma2(Ar, y1r, fma2(nAi, y1i, acc2[p][2])));
        acc2[p][3] = fma2(ui, dy, fma2(Ar, y1i, fma2(Ai, y1r, acc2[p][3])));
        acc2[p][4] = fma2(ur, dz, fma2(Ar, y2r, fma2(nAi, y2i, acc2[p][4])));
        acc2[p][5] = fma2(ui, dz, fma2(Ar, y2i, fma2(Ai, y2r, acc2[p][5])));
      }
    }
  }
}

// One CTA's work: rows [row0, row0 + 256*RP) of a system of n dipoles against
// sources [j_begin, j_end); out[3i + c] = sum_j G(r_i - r_j) x'_j for the
// CTA's rows (out is this split's slice of the partial buffer), and the same
// for x2 into out2 when NR == 2.  Shared by the single-system kernel below
// and the batched kernel.
template <bool FAST, bool IMAGE, bool LOFREE, int RP, int NR>
__device__ __forceinline__ void pairs_f32_cta(
    int n, const float4* __restrict__ obs_hi, const float4* __restrict__ obs_lo,
    const float4* __restrict__ src_hi, const float4* __restrict__ src_lo,
    const double2* __restrict__ x, const double2* __restrict__ x2, float2 m0, float2 m1,
    float2 m2, float k, float inv_k, float s0, int row0, int j_begin, int j_end,
    float2* __restrict__ out, float2* __restrict__ out2) {
  constexpr int ROWS = 2 * RP;
  __shared__ float4 sS[NR == 2 ? 9 : 6][kOtfBlock];
  const int tid = threadIdx.x;
  int irow[ROWS];
  float2 OX[RP], OY[RP], OZ[RP], LX[RP], LY[RP], LZ[RP];
  float2 acc[RP][6], acc2[NR == 2 ? RP : 1][6];
#pragma unroll
  for (int p = 0; p < RP; ++p) {
    const int ia = row0 + (2 * p) * kOtfBlock + tid, ib = ia + kOtfBlock;
    irow[2 * p] = ia;
    irow[2 * p + 1] = ib;
    const float4 ha = obs_hi[min(ia, n - 1)], hb = obs_hi[min(ib, n - 1)];
    OX[p] = f2(ha.x, hb.x);
    OY[p] = f2(ha.y, hb.y);
    OZ[p] = f2(ha.z, hb.z);
    if (!LOFREE) {
      const float4 la = obs_lo[min(ia, n - 1)], lb = obs_lo[min(ib, n - 1)];
      LX[p] = f2(la.x, lb.x);
      LY[p] = f2(la.y, lb.y);
      LZ[p] = f2(la.z, lb.z);
    } else {
      LX[p] = LY[p] = LZ[p] = f2(0.f, 0.f);
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[p][c] = f2(0.f, 0.f);
    if constexpr (NR == 2) {
#pragma unroll
      for (int c = 0; c < 6; ++c) acc2[p][c] = f2(0.f, 0.f);
    }
  }
  const float2 kk2 = f2(k * k, k * k), s02 = f2(s0, s0);
  const int row_end = row0 + kOtfBlock * ROWS;
  // Software pipeline: the source of the next tile is loaded into registers
  // before the current tile is computed, hiding its global-load latency.
  float4 nh = make_float4(0.f, 0.f, 0.f, 0.f), nl = nh;
  double2 na = make_double2(0.0, 0.0), nb = na, nc = na, nd = na, ne = na, nf = na;
  if (j_begin < j_end && tid < min(kOtfBlock, j_end - j_begin)) {
    const int j = j_begin + tid;
    nh = src_hi[j];
    if (!LOFREE) nl = src_lo[j];
    na = x[3 * j];
    nb = x[3 * j + 1];
    nc = x[3 * j + 2];
    if constexpr (NR == 2) {
      nd = x2[3 * j];
      ne = x2[3 * j + 1];
      nf = x2[3 * j + 2];
    }
  }
  for (int jt = j_begin; jt < j_end; jt += kOtfBlock) {
    const int cnt = min(kOtfBlock, j_end - jt);
    __syncthreads();
    if (tid < cnt) {
      float2 xa = f2((float)na.x, (float)na.y), xb = f2((float)nb.x, (float)nb.y),
             xc = f2((float)nc.x, (float)nc.y);
      if (IMAGE) {  // x'_b = m_b x_b, m = (-r, -r, +r)  (assembly.rs:288-292)
        xa = f2(m0.x * xa.x - m0.y * xa.y, m0.x * xa.y + m0.y * xa.x);
        xb = f2(m1.x * xb.x - m1.y * xb.y, m1.x * xb.y + m1.y * xb.x);
        xc = f2(m2.x * xc.x - m2.y * xc.y, m2.x * xc.y + m2.y * xc.x);
      }
      sS[0][tid] = make_float4(nh.x, nh.x, nh.y, nh.y);
      sS[1][tid] = make_float4(nh.z, nh.z, xa.x, xa.x);
      sS[2][tid] = make_float4(xa.y, xa.y, xb.x, xb.x);
      sS[3][tid] = make_float4(xb.y, xb.y, xc.x, xc.x);
      sS[4][tid] = make_float4(xc.y, xc.y, nl.x, nl.x);
      sS[5][tid] = make_float4(nl.y, nl.y, nl.z, nl.z);
      if constexpr (NR == 2) {
        float2 ya = f2((float)nd.x, (float)nd.y), yb = f2((float)ne.x, (float)ne.y),
               yc = f2((float)nf.x, (float)nf.y);
        if (IMAGE) {
          ya = f2(m0.x * ya.x - m0.y * ya.y, m0.x * ya.y + m0.y * ya.x);
          yb = f2(m1.x * yb.x - m1.y * yb.y, m1.x * yb.y + m1.y * yb.x);
          yc = f2(m2.x * yc.x - m2.y * yc.y, m2.x * yc.y + m2.y * yc.x);
        }
        sS[6][tid] = make_float4(ya.x, ya.x, ya.y, ya.y);
        sS[7][tid] = make_float4(yb.x, yb.x, yb.y, yb.y);
        sS[8][tid] = make_float4(yc.x, yc.x, yc.y, yc.y);
      }
    }
    __syncthreads();
    {
      const int jn = jt + kOtfBlock;
      if (jn < j_end && tid < min(kOtfBlock, j_end - jn)) {
        const int j = jn + tid;
        nh = src_hi[j];
        if (!LOFREE) nl = src_lo[j];
        na = x[3 * j];
        nb = x[3 * j + 1];
        nc = x[3 * j + 2];
        if constexpr (NR == 2) {
          nd = x2[3 * j];
          ne = x2[3 * j + 1];
          nf = x2[3 * j + 2];
        }
      }
    }
    const bool diag = IMAGE || (jt < row_end && jt + kOtfBlock > row0);  // CTA-uniform
    if (diag)
      pair_tile_f32x2<FAST, IMAGE, LOFREE, true, RP, NR>(sS, cnt, jt, irow, OX, OY, OZ, LX, LY,
                                                         LZ, acc, acc2, kk2, s02);
    else
      pair_tile_f32x2<FAST, IMAGE, LOFREE, false, RP, NR>(sS, cnt, jt, irow, OX, OY, OZ, LX, LY,
                                                          LZ, acc, acc2, kk2, s02);
  }
#pragma unroll
  for (int p = 0; p < RP; ++p) {
    if (irow[2 * p] < n) {
      const int i = irow[2 * p];
      out[3 * i + 0] = f2(acc[p][0].x, acc[p][1].x);
      out[3 * i + 1] = f2(acc[p][2].x, acc[p][3].x);
      out[3 * i + 2] = f2(acc[p][4].x, acc[p][5].x);
      if constexpr (NR == 2) {
        out2[3 * i + 0] = f2(acc2[p][0].x, acc2[p][1].x);
        out2[3 * i + 1] = f2(acc2[p][2].x, acc2[p][3].x);
        out2[3 * i + 2] = f2(acc2[p][4].x, acc2[p][5].x);
      }
    }
    if (irow[2 * p + 1] < n) {
      const int i = irow[2 * p + 1];
      out[3 * i + 0] = f2(acc[p][0].y, acc[p][1].y);
      out[3 * i + 1] = f2(acc[p][2].y, acc[p][3].y);
      out[3 * i + 2] = f2(acc[p][4].y, acc[p][5].y);
      if constexpr (NR == 2) {
        out2[3 * i + 0] = f2(acc2[p][0].y, acc2[p][1].y);
        out2[3 * i + 1] = f2(acc2[p][2].y, acc2[p][3].y);
        out2[3 * i + 2] = f2(acc2[p][4].y, acc2[p][5].y);
      }
    }
  }
}

// partial[blockIdx.y][3i + c] = sum over split blockIdx.y of G(r_i - r_j) x'_j
template <bool FAST, bool IMAGE, bool LOFREE, int RP, int MINB>
__global__ void __launch_bounds__(kOtfBlock, MINB)
otf_pairs_f32(int n, const float4* __restrict__ obs_hi, const float4* __restrict__ obs_lo,
              const float4* __restrict__ src_hi, const float4* __restrict__ src_lo,
              const double2* __restrict__ x, float2 m0, float2 m1, float2 m2, float k,
              float inv_k, float s0, int chunk, float2* __restrict__ partial,
              const int* __restrict__ skip) {
  if (skip && *skip) return;  // CTA-uniform: the solve no longer needs this product
  const int j_begin = blockIdx.y * chunk;
  pairs_f32_cta<FAST, IMAGE, LOFREE, RP, 1>(
      n, obs_hi, obs_lo, src_hi, src_lo, x, nullptr, m0, m1, m2, k, inv_k, s0,
      blockIdx.x * (kOtfBlock * 2 * RP), j_begin, min(n, j_begin + chunk),
      partial + (size_t)blockIdx.y * (3 * (size_t)n), nullptr);
}

// Two right-hand sides with their own skip flags: both live -> one pass that
// shares the tensor evaluation; one live -> the single-vector pass on it.
// partial / partial2 receive the splits of x / x2.
template <bool FAST, bool IMAGE, bool LOFREE, int RP, int MINB>
__global__ void __launch_bounds__(kOtfBlock, MINB)
otf_pairs_f32_x2(int n, const float4* __restrict__ obs_hi, const float4* __restrict__ obs_lo,
                 const float4* __restrict__ src_hi, const float4* __restrict__ src_lo,
                 const double2* __restrict__ x, const double2* __restrict__ x2, float2 m0,
                 float2 m1, float2 m2, float k, float inv_k, float s0, int chunk,
                 float2* __restrict__ partial, float2* __restrict__ partial2,
                 const int* __restrict__ skip, const int* __restrict__ skip2) {
  const bool live = !(skip && *skip), live2 = !(skip2 && *skip2);  // CTA-uniform
  if (!live && !live2) return;
  const int j_begin = blockIdx.y * chunk, j_end = min(n, j_begin + chunk);
  const int row0 = blockIdx.x * (kOtfBlock * 2 * RP);
  const size_t off = (size_t)blockIdx.y * (3 * (size_t)n);
  if (live && live2)
    pairs_f32_cta<FAST, IMAGE, LOFREE, RP, 2>(n, obs_hi, obs_lo, src_hi, src_lo, x, x2, m0, m1,
                                              m2, k, inv_k, s0, row0, j_begin, j_end,
                                              partial + off, partial2 + off);
  else
    pairs_f32_cta<FAST, IMAGE, LOFREE, RP, 1>(n, obs_hi, obs_lo, src_hi, src_lo,
                                              live ? x : x2, nullptr, m0, m1, m2, k, inv_k, s0,
                                              row0, j_begin, j_end,
                                              (live ? partial : partial2) + off, nullptr);
}

}  // namespace lum
