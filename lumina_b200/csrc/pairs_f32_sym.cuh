// pairs_f32_sym.cuh -- FP32 dense pair kernel that evaluates each unordered
// pair once.
//
// The point-dipole tensor is symmetric and even in the displacement
// (G(r_i - r_j) = G(r_j - r_i) = G^T, greens.rs:34-71), so one evaluation of
// the pair scalars (A, B', d) serves both y_i += G x_j and y_j += G x_i.  The
// shared part of a pair (~27 FP32 operations, rsqrt, sin, cos) is done once
// per unordered pair instead of once per ordered pair; each direction keeps
// its own 28-operation contraction.
//
// Work: superblocks of kSymRows rows.  A CTA (8 warps) takes one superblock
// pair (I, J), I <= J.  Warp w holds rows I*kSymRows + 64 w + {lane,
// lane + 32}, packed into the two halves of a float2 as in pairs_f32x2.cuh,
// with their positions, moments x_i and row sums in registers.  The sources
// of J are staged 32 at a time in shared memory; in step s of a group, lane
// l pairs its rows with source (l + s) mod 32 (conflict-free: consecutive
// lanes read consecutive entries).  The source-side sums travel with the
// sources: after each step every lane passes its source accumulator to lane
// l - 1, so after 32 steps lane l holds the sum for source l over the warp's
// 64 rows.  The eight warps' sums are then added in warp order.
//
// Output, deterministic and free of atomics: slot[S][3i + c] is the sum over
// sources of superblock S for row i.  Item (I, J), I < J, writes slot J for
// the rows of I (row side) and slot I for the rows of J (source side); the
// diagonal item (I, I) takes only pairs j > i and writes slot I for the rows
// of I, both sides added together.  Every (slot, row) is written exactly
// once; the epilogue sums the slots in order.
#pragma once

namespace lum {

constexpr int kSymRows = 512;   // rows (and sources) per superblock
constexpr int kSymThreads = 256;

template <bool FAST, bool LOFREE, int MINB>
__global__ void __launch_bounds__(kSymThreads, MINB)
otf_pairs_f32_sym(int n, const float4* __restrict__ obs_hi, const float4* __restrict__ obs_lo,
                  const double2* __restrict__ x, float k, float s0,
                  const int2* __restrict__ items, float2* __restrict__ slots,
                  const int* __restrict__ skip) {
  if (skip && *skip) return;
  __shared__ float4 sS[6][32];
  __shared__ float2 sAcc[kSymThreads / 32][32][6];
  __shared__ float sDiag[kSymRows][6];
  const int2 it = items[blockIdx.x];
  const int I = it.x, J = it.y;
  const bool diag = (I == J);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t n3 = 3 * (size_t)n;

  // rows of this thread (a = lane, b = lane + 32 of the warp's 64); rows past
  // n sit far away with x = 0 and are never written
  const int ia = I * kSymRows + 64 * warp + lane, ib = ia + 32;
  const bool va = ia < n, vb = ib < n;
  const float4 far4 = make_float4(2e8f, 2e8f, 2e8f, 0.f), zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
  const float4 ha = va ? obs_hi[ia] : far4, hb = vb ? obs_hi[ib] : far4;
  const float2 OX = make_float2(ha.x, hb.x), OY = make_float2(ha.y, hb.y),
               OZ = make_float2(ha.z, hb.z);
  float2 LX = make_float2(0.f, 0.f), LY = LX, LZ = LX;
  if (!LOFREE) {
    const float4 la = va ? obs_lo[ia] : zero4, lb = vb ? obs_lo[ib] : zero4;
    LX = make_float2(la.x, lb.x);
    LY = make_float2(la.y, lb.y);
    LZ = make_float2(la.z, lb.z);
  }
  float2 X[6];  // (x0r, x0i, x1r, x1i, x2r, x2i) of rows a / b
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double2 xa = va ? x[3 * (size_t)ia + c] : make_double2(0.0, 0.0);
    const double2 xb = vb ? x[3 * (size_t)ib + c] : make_double2(0.0, 0.0);
    X[2 * c] = make_float2((float)xa.x, (float)xb.x);
    X[2 * c + 1] = make_float2((float)xa.y, (float)xb.y);
  }
  float2 acc[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) acc[c] = make_float2(0.f, 0.f);
  if (diag)
    for (int q = tid; q < kSymRows * 6; q += kSymThreads) (&sDiag[0][0])[q] = 0.f;

  const float2 kk2 = make_float2(k * k, k * k), s02 = make_float2(s0, s0);
  const float2 m3 = make_float2(-3.0f, -3.0f), m1 = make_float2(-1.0f, -1.0f),
               one = make_float2(1.0f, 1.0f);
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
        const double2 a = x[3 * (size_t)j], b = x[3 * (size_t)j + 1], c = x[3 * (size_t)j + 2];
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
    }
    __syncthreads();
    float2 sacc[6];  // source-side sum of source (lane + s) mod 32, halves a / b
#pragma unroll
    for (int c = 0; c < 6; ++c) sacc[c] = make_float2(0.f, 0.f);
#pragma unroll 1
    for (int s = 0; s < 32; ++s) {
      const int src = (lane + s) & 31;
      const float4 S0 = sS[0][src], S1 = sS[1][src], S2 = sS[2][src], S3 = sS[3][src],
                   S4 = sS[4][src];
      float2 dx = sub2(OX, lo2(S0));
      float2 dy = sub2(OY, hi2(S0));
      float2 dz = sub2(OZ, lo2(S1));
      if (!LOFREE) {
        const float4 S5 = sS[5][src];
        dx = add2(dx, sub2(LX, hi2(S4)));
        dy = add2(dy, sub2(LY, lo2(S5)));
        dz = add2(dz, sub2(LZ, hi2(S5)));
      }
      float2 r2 = fma2(dx, dx, fma2(dy, dy, mul2(dz, dz)));
      float2 keep = one;
      if (diag) {  // each unordered pair once: j > i; the self pair is masked
        const int j = jg + src;
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
      const float2 Ar = sub2(mul2(pr, ar), mul2(pi, u));
      const float2 Ai = fma2(pr, u, mul2(pi, ar));
      const float2 ir2 = mul2(u2, kk2);
      const float2 Br = mul2(fma2(Ar, m3, add2(pr, pr)), ir2);
      const float2 Bi = mul2(fma2(Ai, m3, add2(pi, pi)), ir2);
      const float2 nAi = mul2(Ai, m1), nBi = mul2(Bi, m1);
      // row side: y_i += A x_j + B' d (d . x_j)
      const float2 x0r = hi2(S1), x0i = lo2(S2), x1r = hi2(S2), x1i = lo2(S3), x2r = hi2(S3),
                   x2i = lo2(S4);
      {
        const float2 dxr = fma2(dx, x0r, fma2(dy, x1r, mul2(dz, x2r)));
        const float2 dxi = fma2(dx, x0i, fma2(dy, x1i, mul2(dz, x2i)));
        const float2 tr = fma2(Br, dxr, mul2(nBi, dxi));
        const float2 ti = fma2(Br, dxi, mul2(Bi, dxr));
        acc[0] = fma2(tr, dx, fma2(Ar, x0r, fma2(nAi, x0i, acc[0])));
        acc[1] = fma2(ti, dx, fma2(Ar, x0i, fma2(Ai, x0r, acc[1])));
        acc[2] = fma2(tr, dy, fma2(Ar, x1r, fma2(nAi, x1i, acc[2])));
        acc[3] = fma2(ti, dy, fma2(Ar, x1i, fma2(Ai, x1r, acc[3])));
        acc[4] = fma2(tr, dz, fma2(Ar, x2r, fma2(nAi, x2i, acc[4])));
        acc[5] = fma2(ti, dz, fma2(Ar, x2i, fma2(Ai, x2r, acc[5])));
      }
      // source side: y_j += A x_i + B' d (d . x_i), the same A, B', d
      {
        const float2 dxr = fma2(dx, X[0], fma2(dy, X[2], mul2(dz, X[4])));
        const float2 dxi = fma2(dx, X[1], fma2(dy, X[3], mul2(dz, X[5])));
        const float2 tr = fma2(Br, dxr, mul2(nBi, dxi));
        const float2 ti = fma2(Br, dxi, mul2(Bi, dxr));
        sacc[0] = fma2(tr, dx, fma2(Ar, X[0], fma2(nAi, X[1], sacc[0])));
        sacc[1] = fma2(ti, dx, fma2(Ar, X[1], fma2(Ai, X[0], sacc[1])));
        sacc[2] = fma2(tr, dy, fma2(Ar, X[2], fma2(nAi, X[3], sacc[2])));
        sacc[3] = fma2(ti, dy, fma2(Ar, X[3], fma2(Ai, X[2], sacc[3])));
        sacc[4] = fma2(tr, dz, fma2(Ar, X[4], fma2(nAi, X[5], sacc[4])));
        sacc[5] = fma2(ti, dz, fma2(Ar, X[5], fma2(Ai, X[4], sacc[5])));
      }
      // pass each source's sum on: lane l takes the one of source (l + s + 1)
      const int from = (lane + 1) & 31;
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        sacc[c].x = __shfl_sync(0xffffffffu, sacc[c].x, from);
        sacc[c].y = __shfl_sync(0xffffffffu, sacc[c].y, from);
      }
    }
    // lane l now holds source l's sum over the warp's rows (halves a / b)
#pragma unroll
    for (int c = 0; c < 6; ++c) sAcc[warp][lane][c] = sacc[c];
    __syncthreads();
    if (tid < 32 * 6) {
      const int sl = tid / 6, c = tid % 6;
      float v = 0.f;
#pragma unroll
      for (int w = 0; w < kSymThreads / 32; ++w) v += sAcc[w][sl][c].x + sAcc[w][sl][c].y;
      const int j = jg + sl;
      if (diag) {
        sDiag[32 * g + sl][c] = v;
      } else if (j < n) {
        float* dst = reinterpret_cast<float*>(slots + (size_t)I * n3 + 3 * (size_t)j);
        dst[c] = v;  // c = 2 * component + (0 re | 1 im)
      }
    }
  }
  __syncthreads();
  // row side: slot J for the rows of I (diagonal: plus the source-side sums)
  const int lr = 64 * warp + lane;
  if (va) {
    float2* dst = slots + (size_t)J * n3 + 3 * (size_t)ia;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float re = acc[2 * c].x, im = acc[2 * c + 1].x;
      if (diag) {
        re += sDiag[lr][2 * c];
        im += sDiag[lr][2 * c + 1];
      }
      dst[c] = make_float2(re, im);
    }
  }
  if (vb) {
    float2* dst = slots + (size_t)J * n3 + 3 * (size_t)ib;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float re = acc[2 * c].y, im = acc[2 * c + 1].y;
      if (diag) {
        re += sDiag[lr + 32][2 * c];
        im += sDiag[lr + 32][2 * c + 1];
      }
      dst[c] = make_float2(re, im);
    }
  }
}

}  // namespace lum
