// gmres.cu -- device-resident restarted GMRES (iterative.rs:33-206).
//
// The Krylov basis V ((m+1) x 3N complex FP64), the Hessenberg matrix, the
// Givens rotations and the least-squares right-hand side live in device
// memory.  Every Arnoldi step is: one operator application (FP64, or FP32
// in the refinement mode), j+1 modified Gram-Schmidt kernels, one kernel that
// normalises and runs the Givens update on a single thread, and an 8-byte
// read of |g_{j+1}| for the host's convergence test.
//
// Each MGS kernel fuses the previous projection's subtraction
// (w -= h_{i-1,j} v_{i-1}) with the next inner product <v_i, w>, which is
// the reference's MGS order (iterative.rs:92-96) with one pass over w per
// projection.  Reductions write one partial per block and the last block to
// finish sums the partials in block order, so results are deterministic.
#include "lumina_internal.cuh"

#include <cooperative_groups.h>

#include <chrono>
#include <cstdlib>
#include <cmath>
#include <cstddef>

namespace lum {

constexpr int kVecThreads = 256;
constexpr int kM = kMaxRestart;

__device__ __forceinline__ double2 dmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 dconjmul(double2 a, double2 b) {  // conj(a) * b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 ddiv(double2 a, double2 b) {
  double n = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / n, (a.y * b.x - a.x * b.y) / n);
}
__device__ __forceinline__ double dabs(double2 a) { return hypot(a.x, a.y); }

// Block reduction of a complex pair; result valid in thread 0.
__device__ double2 block_sum2(double2 v) {
  __shared__ double2 sh[kVecThreads / 32];
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = (lane < kVecThreads / 32) ? sh[lane] : make_double2(0.0, 0.0);
    for (int o = 16; o > 0; o >>= 1) {
      v.x += __shfl_down_sync(0xffffffffu, v.x, o);
      v.y += __shfl_down_sync(0xffffffffu, v.y, o);
    }
  }
  return v;
}

// Publishes this block's partial; returns true (in every thread) in the last
// block to finish, whose thread 0 then holds the total in *total.  The last
// block sums the partials with all its threads and a fixed-shape tree, so
// the result does not depend on which block finished last.
__device__ bool last_block_total(double2 part, double2* partials, unsigned* counter,
                                 double2* total) {
  __shared__ bool am_last;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = part;
    __threadfence();
    unsigned t = atomicAdd(counter, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  double2 v = make_double2(0.0, 0.0);
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    const double2 p = __ldcg(&partials[b]);  // L2: written by other blocks
    v.x += p.x;
    v.y += p.y;
  }
  v = block_sum2(v);
  if (threadIdx.x == 0) {
    *total = v;
    *counter = 0u;
  }
  return true;
}

__global__ void __launch_bounds__(kVecThreads)
k_norm(int len, const double2* __restrict__ v, double2* partials, unsigned* counter,
       GmresState* S, int slot) {
  double2 acc = make_double2(0.0, 0.0);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < len; q += gridDim.x * blockDim.x) {
    double2 a = v[q];
    acc.x += a.x * a.x + a.y * a.y;
  }
  acc = block_sum2(acc);
  double2 tot;
  if (last_block_total(acc, partials, counter, &tot) && threadIdx.x == 0)
    S->scal[slot] = sqrt(tot.x);
}

// r = b - Ax, ||r||  -> S->scal[3]
__global__ void __launch_bounds__(kVecThreads)
k_residual(int len, const double2* __restrict__ b, const double2* __restrict__ ax,
           double2* __restrict__ r, double2* partials, unsigned* counter, GmresState* S) {
  double2 acc = make_double2(0.0, 0.0);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < len; q += gridDim.x * blockDim.x) {
    double2 bb = b[q], aa = ax[q];
    double2 d = make_double2(bb.x - aa.x, bb.y - aa.y);
    r[q] = d;
    acc.x += d.x * d.x + d.y * d.y;
  }
  acc = block_sum2(acc);
  double2 tot;
  if (last_block_total(acc, partials, counter, &tot) && threadIdx.x == 0)
    S->scal[3] = sqrt(tot.x);
}

// v0 = r / beta (beta = S->scal[3]); g = beta e1
__global__ void __launch_bounds__(kVecThreads)
k_start_cycle(int len, const double2* __restrict__ r, double2* __restrict__ v0, GmresState* S,
              int m) {
  const double beta = S->scal[3];
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < len; q += gridDim.x * blockDim.x) {
    double2 a = r[q];
    v0[q] = make_double2(a.x / beta, a.y / beta);
  }
  if (blockIdx.x == 0 && threadIdx.x <= m) {
    S->g[threadIdx.x] = make_double2(threadIdx.x == 0 ? beta : 0.0, 0.0);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    S->done = 0;
    S->jdone = 0;
    S->bad = 0;
  }
}

// Per-step arguments of one right-hand side.  The step kernels serve one or
// two right-hand sides per launch (blockIdx.y selects the set), each with its
// own reduction counter, so lockstep solves pay one launch per step kernel.
struct MgsArgs {
  double2* w;
  double2* V;
  double2* partials;
  unsigned* counter;
  GmresState* S;
  double abs_tol, inner_thr;
  int jmax;
};

// MGS projection i of column j: w -= h_{i-1,j} v_{i-1} (i>0); h_{i,j} = <v_i, w>.
__global__ void __launch_bounds__(kVecThreads)
k_mgs(int len, int i, int j, MgsArgs a0, MgsArgs a1) {
  const MgsArgs a = blockIdx.y ? a1 : a0;
  double2* __restrict__ w = a.w;
  const double2* __restrict__ V = a.V;
  GmresState* S = a.S;
  if (S->done) return;  // uniform over this right-hand side's blocks
  const double2* vi = V + (size_t)i * len;
  const double2* vp = V + (size_t)(i > 0 ? i - 1 : 0) * len;
  const double2 hp = (i > 0) ? S->H[(i - 1) * kM + j] : make_double2(0.0, 0.0);
  double2 acc = make_double2(0.0, 0.0);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < len; q += gridDim.x * blockDim.x) {
    double2 wq = w[q];
    if (i > 0) {
      double2 t = dmul(vp[q], hp);
      wq.x -= t.x;
      wq.y -= t.y;
      w[q] = wq;
    }
    double2 d = dconjmul(vi[q], wq);
    acc.x += d.x;
    acc.y += d.y;
  }
  acc = block_sum2(acc);
  double2 tot;
  if (last_block_total(acc, a.partials, a.counter, &tot) && threadIdx.x == 0)
    S->H[i * kM + j] = tot;
}

// Givens pair (iterative.rs:180-191): c real, s complex.
__device__ void givens(double2 a, double2 b, double* c, double2* s) {
  if (dabs(b) < 1e-30) {
    *c = 1.0;
    *s = make_double2(0.0, 0.0);
    return;
  }
  if (dabs(a) < 1e-30) {
    *c = 0.0;
    *s = ddiv(b, make_double2(dabs(b), 0.0));
    return;
  }
  double r = sqrt((a.x * a.x + a.y * a.y) + (b.x * b.x + b.y * b.y));
  *c = dabs(a) / r;
  double2 an = ddiv(a, make_double2(dabs(a), 0.0));
  double2 t = dmul(an, make_double2(b.x, -b.y));
  *s = make_double2(t.x / r, t.y / r);
}

// Last projection of column j, ||w||, then (single thread) the rotations of
// iterative.rs:98-127.  |g_{j+1}| -> S->scal[2], h_{j+1,j} -> S->scal[1].
// The step's convergence test runs here too: |g_{j+1}| < abs_tol (the
// reference's in-cycle test, iterative.rs:133) or, in the refinement mode,
// below inner_thr; either ends the cycle by setting S->done, which turns the
// kernels already queued for later steps of the cycle into no-ops.  The
// cycle's last step (j + 1 == jmax) sets it too, so a second right-hand side
// sharing the operator applications skips the steps this one does not take.
__global__ void __launch_bounds__(kVecThreads)
k_mgs_final(int len, int j, MgsArgs a0, MgsArgs a1) {
  const MgsArgs a = blockIdx.y ? a1 : a0;
  double2* __restrict__ w = a.w;
  const double2* __restrict__ V = a.V;
  GmresState* S = a.S;
  const double abs_tol = a.abs_tol, inner_thr = a.inner_thr;
  const int jmax = a.jmax;
  if (S->done) return;  // uniform over this right-hand side's blocks
  const double2* vj = V + (size_t)j * len;
  const double2 hp = S->H[j * kM + j];
  double2 acc = make_double2(0.0, 0.0);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < len; q += gridDim.x * blockDim.x) {
    double2 t = dmul(vj[q], hp);
    double2 wq = w[q];
    wq.x -= t.x;
    wq.y -= t.y;
    w[q] = wq;
    acc.x += wq.x * wq.x + wq.y * wq.y;
  }
  acc = block_sum2(acc);
  double2 tot;
  __shared__ double s_hn;
  __shared__ double2 sH[kM + 1], sS[kM], sG[2];
  __shared__ double sC[kM];
  if (!last_block_total(acc, a.partials, a.counter, &tot)) return;  // block-uniform
  // last block: stage column j, the rotations and g[j..j+1] in shared memory
  const int t = threadIdx.x;
  if (t == 0) s_hn = sqrt(tot.x);
  if (t <= j) sH[t] = S->H[t * kM + j];
  if (t < j) {
    sC[t] = S->cs[t];
    sS[t] = S->sn[t];
  }
  if (t < 2) sG[t] = S->g[j + t];
  __syncthreads();
  if (t == 0) {
    const double hn = s_hn;
    sH[j + 1] = make_double2(hn, 0.0);
    for (int i = 0; i < j; ++i) {
      const double c = sC[i];
      const double2 s = sS[i];
      const double2 hij = sH[i], hi1 = sH[i + 1];
      const double2 t1 = dmul(s, hi1);
      const double2 temp = make_double2(c * hij.x + t1.x, c * hij.y + t1.y);
      const double2 t2 = dmul(make_double2(-s.x, s.y), hij);  // -conj(s) * h_ij
      sH[i + 1] = make_double2(t2.x + c * hi1.x, t2.y + c * hi1.y);
      sH[i] = temp;
    }
    double c;
    double2 s;
    givens(sH[j], sH[j + 1], &c, &s);
    const double2 hjj = sH[j], hj1 = sH[j + 1];
    const double2 t1 = dmul(s, hj1);
    sH[j] = make_double2(c * hjj.x + t1.x, c * hjj.y + t1.y);
    sH[j + 1] = make_double2(0.0, 0.0);
    const double2 gj = sG[0], gj1 = sG[1];
    const double2 t3 = dmul(s, gj1);
    const double2 t4 = dmul(make_double2(-s.x, s.y), gj);
    const double2 g1 = make_double2(t4.x + c * gj1.x, t4.y + c * gj1.y);
    S->g[j] = make_double2(c * gj.x + t3.x, c * gj.y + t3.y);
    S->g[j + 1] = g1;
    S->cs[j] = c;
    S->sn[j] = s;
    S->scal[1] = hn;
    const double gabs = dabs(g1);
    S->scal[2] = gabs;
    S->jdone = j + 1;
    if (!isfinite(gabs)) {
      S->bad = 1;
      S->done = 1;
    } else if (gabs < abs_tol || gabs < inner_thr || j + 1 >= jmax) {
      S->done = 1;  // the last step of the cycle also ends it (later kernels skip)
    }
  }
  __syncthreads();
  if (t <= j + 1) S->H[t * kM + j] = sH[t];
}

// The whole Arnoldi step j in one cooperative launch: the j+1 projections of
// modified Gram-Schmidt in the order of iterative.rs:92-96, ||w||, the
// Givens update of k_mgs_final and v_{j+1} = w / h_{j+1,j}.  Each reduction
// crosses one grid barrier: every block writes its partial, and after the
// barrier every block sums all partials in the same fixed order, so every
// block holds the same h_{i,j} (deterministic, no atomics).  Partials are
// double-buffered by barrier parity: a buffer is rewritten two barriers after
// it was filled, when every block has read it.  All blocks pass the same
// j + 2 barriers; a right-hand side whose cycle is done does no work but
// still takes part, and the launch returns at once (before any barrier) only
// when every right-hand side is done.
__device__ double2 coop_total(const double2* part, int G) {
  double2 v = make_double2(0.0, 0.0);
  for (int b = threadIdx.x; b < G; b += blockDim.x) {
    const double2 p = __ldcg(&part[b]);
    v.x += p.x;
    v.y += p.y;
  }
  v = block_sum2(v);
  __shared__ double2 s_tot;
  if (threadIdx.x == 0) s_tot = v;
  __syncthreads();
  const double2 t = s_tot;
  __syncthreads();
  return t;
}

__global__ void __launch_bounds__(kVecThreads)
k_arnoldi_coop(int len, int j, int nrhs, MgsArgs a0, MgsArgs a1, double2* part0,
               double2* part1) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  const int r = blockIdx.y;
  const MgsArgs a = r ? a1 : a0;
  double2* part = r ? part1 : part0;
  const int G = gridDim.x;
  const bool done0 = a0.S->done != 0, done1 = (nrhs > 1) ? (a1.S->done != 0) : true;
  if (done0 && done1) return;  // grid-uniform: no barrier is taken
  const bool active = !(r ? done1 : done0);
  double2* __restrict__ w = a.w;
  const double2* __restrict__ V = a.V;
  GmresState* S = a.S;
  const int stride = G * blockDim.x;
  double2 hprev = make_double2(0.0, 0.0);
  double hn = 0.0;
  for (int i = 0; i <= j + 1; ++i) {
    double2 acc = make_double2(0.0, 0.0);
    if (active) {
      const double2* vp = V + (size_t)(i > 0 ? i - 1 : 0) * len;
      if (i <= j) {  // w -= h_{i-1,j} v_{i-1};  <v_i, w>
        const double2* vi = V + (size_t)i * len;
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < len; q += stride) {
          double2 wq = w[q];
          if (i > 0) {
            const double2 t = dmul(vp[q], hprev);
            wq.x -= t.x;
            wq.y -= t.y;
            w[q] = wq;
          }
          const double2 d = dconjmul(vi[q], wq);
          acc.x += d.x;
          acc.y += d.y;
        }
      } else {  // w -= h_{j,j} v_j;  ||w||^2
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < len; q += stride) {
          const double2 t = dmul(vp[q], hprev);
          double2 wq = w[q];
          wq.x -= t.x;
          wq.y -= t.y;
          w[q] = wq;
          acc.x += wq.x * wq.x + wq.y * wq.y;
        }
      }
    }
    acc = block_sum2(acc);
    double2* buf = part + (size_t)(i & 1) * G;
    if (threadIdx.x == 0) buf[blockIdx.x] = acc;
    grid.sync();
    const double2 tot = coop_total(buf, G);
    if (i <= j) {
      hprev = tot;
      if (active && blockIdx.x == 0 && threadIdx.x == 0) S->H[i * kM + j] = tot;
    } else {
      hn = sqrt(tot.x);
    }
  }
  if (!active) return;
  // v_{j+1} = w / h_{j+1,j} (iterative.rs:101-106); this block's own entries
  {
    double2* __restrict__ vnext = a.V + (size_t)(j + 1) * len;
    const bool ok = hn > 1e-30;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < len; q += stride) {
      const double2 wq = w[q];
      vnext[q] = ok ? make_double2(wq.x / hn, wq.y / hn) : make_double2(0.0, 0.0);
    }
  }
  if (blockIdx.x != 0) return;
  // Givens update of column j (iterative.rs:98-133) on block 0, as k_mgs_final
  __shared__ double2 sH[kM + 1], sSn[kM], sG[2];
  __shared__ double sC[kM];
  const int t = threadIdx.x;
  __syncthreads();  // S->H[i][j] written by thread 0 above
  if (t <= j) sH[t] = S->H[t * kM + j];
  if (t < j) {
    sC[t] = S->cs[t];
    sSn[t] = S->sn[t];
  }
  if (t < 2) sG[t] = S->g[j + t];
  __syncthreads();
  if (t == 0) {
    sH[j + 1] = make_double2(hn, 0.0);
    for (int i = 0; i < j; ++i) {
      const double c = sC[i];
      const double2 s = sSn[i];
      const double2 hij = sH[i], hi1 = sH[i + 1];
      const double2 t1 = dmul(s, hi1);
      const double2 temp = make_double2(c * hij.x + t1.x, c * hij.y + t1.y);
      const double2 t2 = dmul(make_double2(-s.x, s.y), hij);  // -conj(s) * h_ij
      sH[i + 1] = make_double2(t2.x + c * hi1.x, t2.y + c * hi1.y);
      sH[i] = temp;
    }
    double c;
    double2 s;
    givens(sH[j], sH[j + 1], &c, &s);
    const double2 hjj = sH[j], hj1 = sH[j + 1];
    const double2 t1 = dmul(s, hj1);
    sH[j] = make_double2(c * hjj.x + t1.x, c * hjj.y + t1.y);
    sH[j + 1] = make_double2(0.0, 0.0);
    const double2 gj = sG[0], gj1 = sG[1];
    const double2 t3 = dmul(s, gj1);
    const double2 t4 = dmul(make_double2(-s.x, s.y), gj);
    const double2 g1 = make_double2(t4.x + c * gj1.x, t4.y + c * gj1.y);
    S->g[j] = make_double2(c * gj.x + t3.x, c * gj.y + t3.y);
    S->g[j + 1] = g1;
    S->cs[j] = c;
    S->sn[j] = s;
    S->scal[1] = hn;
    const double gabs = dabs(g1);
    S->scal[2] = gabs;
    S->jdone = j + 1;
    if (!isfinite(gabs)) {
      S->bad = 1;
      S->done = 1;
    } else if (gabs < a.abs_tol || gabs < a.inner_thr || j + 1 >= a.jmax) {
      S->done = 1;
    }
  }
  __syncthreads();
  if (t <= j + 1) S->H[t * kM + j] = sH[t];
}

// v_{j+1} = w / h_{j+1,j}, or 0 on a lucky breakdown (iterative.rs:101-106)
__global__ void __launch_bounds__(kVecThreads)
k_next_basis(int len, int j, MgsArgs a0, MgsArgs a1) {
  const MgsArgs a = blockIdx.y ? a1 : a0;
  const double2* __restrict__ w = a.w;
  double2* __restrict__ vnext = a.V + (size_t)(j + 1) * len;
  const GmresState* S = a.S;
  if (S->done) return;  // the basis beyond a finished step is never used
  const double hn = S->scal[1];
  const bool ok = hn > 1e-30;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < len; q += gridDim.x * blockDim.x) {
    double2 a = w[q];
    vnext[q] = ok ? make_double2(a.x / hn, a.y / hn) : make_double2(0.0, 0.0);
  }
}

// Back substitution H[0..j,0..j] y = g[0..j] (iterative.rs:194-206).
// The leading j x j block of H and g[0..j) are staged in shared memory by
// the whole block, then one thread substitutes.
// Upper triangle packed row by row: row r holds columns r..j-1 at
// tri_off(r) = r*j - r*(r-1)/2 (at most 64*65/2 entries, 33 KB).
__device__ __forceinline__ int tri_off(int r, int j) { return r * j - (r * (r - 1)) / 2; }

__global__ void __launch_bounds__(kVecThreads) k_backsub(GmresState* S) {
  const int j = S->jdone;
  __shared__ double2 sH[kM * (kM + 1) / 2];
  __shared__ double2 sg[kM], sy[kM];
  for (int e = threadIdx.x; e < j * j; e += blockDim.x) {
    const int r = e / j, c = e % j;
    if (c >= r) sH[tri_off(r, j) + (c - r)] = S->H[r * kM + c];
  }
  if (threadIdx.x < j) sg[threadIdx.x] = S->g[threadIdx.x];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = j - 1; i >= 0; --i) {
      double2 sum = sg[i];
      const double2* row = sH + tri_off(i, j) - i;  // row[q] = H[i][q] for q >= i
      for (int q = i + 1; q < j; ++q) {
        const double2 t = dmul(row[q], sy[q]);
        sum.x -= t.x;
        sum.y -= t.y;
      }
      const double2 hii = row[i];
      sy[i] = (dabs(hii) > 1e-30) ? ddiv(sum, hii) : make_double2(0.0, 0.0);
    }
  }
  __syncthreads();
  if (threadIdx.x < j) S->y[threadIdx.x] = sy[threadIdx.x];
}

// x += sum_i y_i v_i (iterative.rs:142-144)
__global__ void __launch_bounds__(kVecThreads)
k_update_x(int len, double2* __restrict__ x, const double2* __restrict__ V,
           const GmresState* S) {
  const int j = S->jdone;
  __shared__ double2 ys[kM];
  if (threadIdx.x < j) ys[threadIdx.x] = S->y[threadIdx.x];
  __syncthreads();
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < len; q += gridDim.x * blockDim.x) {
    double2 acc = x[q];
    for (int i = 0; i < j; ++i) {
      double2 t = dmul(V[(size_t)i * len + q], ys[i]);
      acc.x += t.x;
      acc.y += t.y;
    }
    x[q] = acc;
  }
}

// ---------------------------------------------------------------------------
GmresWork::~GmresWork() {
  if (h_state) cudaFreeHost(h_state);
}

lum_status GmresWork::ensure(int len_, int m_, cudaStream_t st) {
  if (len_ == len && m_ <= m && V.p) return LUM_OK;
  len = len_;
  m = m_;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  nblk = std::max(1, std::min((len + kVecThreads - 1) / kVecThreads, 2 * sms));
  LUM_TRY(V.alloc(sizeof(double2) * (size_t)(m + 1) * len));
  LUM_TRY(w.alloc(sizeof(double2) * (size_t)len));
  LUM_TRY(r.alloc(sizeof(double2) * (size_t)len));
  LUM_TRY(tmp.alloc(sizeof(double2) * (size_t)len));
  LUM_TRY(partials.alloc(sizeof(double2) * (size_t)nblk));
  LUM_TRY(coop_part.alloc(sizeof(double2) * 2 * (size_t)nblk));
  LUM_TRY(counter.alloc(sizeof(unsigned)));
  LUM_TRY(state.alloc(sizeof(GmresState)));
  LUM_TRY_CUDA(cudaMemsetAsync(counter.p, 0, sizeof(unsigned), st));
  LUM_TRY_CUDA(cudaMemsetAsync(state.p, 0, sizeof(GmresState), st));
  if (!h_state) LUM_TRY_CUDA(cudaMallocHost((void**)&h_state, sizeof(GmresState)));
  return LUM_OK;
}

lum_status vec_norm(const double2* v, int len, GmresWork& W, int slot, cudaStream_t st) {
  k_norm<<<W.nblk, kVecThreads, 0, st>>>(len, v, W.partials.as<double2>(),
                                         W.counter.as<unsigned>(), W.state.as<GmresState>(),
                                         slot);
  LUM_CHECK_LAUNCH();
  return LUM_OK;
}

lum_status read_scalars(GmresWork& W, cudaStream_t st) {
  // scal[8] and the done/jdone/bad flags are contiguous at the end of the state
  const size_t bytes = sizeof(GmresState) - offsetof(GmresState, scal);
  LUM_TRY_CUDA(cudaMemcpyAsync(W.h_state->scal, W.state.as<GmresState>()->scal, bytes,
                               cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));
  return LUM_OK;
}

}  // namespace lum

using namespace lum;

// Host driver; called from the C ABI with device vectors.  One or two
// right-hand sides: with two, both GMRES runs advance in lockstep and every
// operator application serves both (lum_session::apply2), each run with its
// own Krylov basis, Hessenberg matrix, convergence flag and restart count.
// A run that has converged (or run out of iterations) drops out, and the
// other continues with single-vector applications.
namespace {
struct RhsRun {
  GmresWork* W = nullptr;
  const double2* b = nullptr;
  double2* x = nullptr;
  double rhs_norm = 0.0, abs_tol = 0.0, beta = 0.0;
  int total = 0, jmax = 0;
  bool active = false;
  lum_status result = LUM_OK;
  lum_solve_info loc{};
};
}  // namespace

lum_status lum_gmres_device_multi(lum_session* s, int nrhs, const double2* const* b,
                                  double2* const* x, double tol, int max_iter, int restart,
                                  int mode, lum_solve_info* info, cudaStream_t st) {
  if (nrhs < 1 || nrhs > 2) {
    set_error("lum_gmres_device_multi takes one or two right-hand sides");
    return LUM_ERR_INVALID;
  }
  auto t0 = std::chrono::steady_clock::now();
  const int len = s->dim;
  if (restart <= 0) restart = 30;
  const int m = std::min(std::min(restart, len), kMaxRestart);
  const int arnoldi_prec = (mode == LUM_SOLVE_FP32_REFINE) ? LUM_FP32 : LUM_FP64;
  const double inner_rel = 1e-5;
  RhsRun run[2];
  for (int r = 0; r < nrhs; ++r) {
    RhsRun& R = run[r];
    R.W = (r == 0) ? &s->gw : &s->gw2;
    R.b = b[r];
    R.x = x[r];
    LUM_TRY(R.W->ensure(len, m, st));
    LUM_TRY_CUDA(cudaMemsetAsync(R.x, 0, sizeof(double2) * (size_t)len, st));
    LUM_TRY(vec_norm(R.b, len, *R.W, 3, st));
  }
  for (int r = 0; r < nrhs; ++r) LUM_TRY(read_scalars(*run[r].W, st));
  for (int r = 0; r < nrhs; ++r) {
    RhsRun& R = run[r];
    R.rhs_norm = R.W->h_state->scal[3];
    if (!std::isfinite(R.rhs_norm)) {
      set_error("right-hand side is not finite");
      return LUM_ERR_INVALID;
    }
    if (R.rhs_norm < 1e-30) {
      R.loc.converged = 1;
      continue;
    }
    R.abs_tol = tol * R.rhs_norm;
    R.beta = R.rhs_norm;
    // r = b - A*0 = b; beta = ||b|| (already in scal[3])
    LUM_TRY_CUDA(cudaMemcpyAsync(R.W->r.p, R.b, sizeof(double2) * (size_t)len,
                                 cudaMemcpyDeviceToDevice, st));
    R.active = true;
  }
  // Blocks per right-hand side of the fused step kernel: the step kernels'
  // grid, bounded so that both right-hand sides' blocks are co-resident (a
  // cooperative launch needs that); 0 selects the per-projection kernels
  // (LUMINA_COOP=0, or no cooperative launch on the device).
  int coop_blocks = 0;
  {
    int dev = 0, coop = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_arnoldi_coop, kVecThreads, 0);
    const char* env = std::getenv("LUMINA_COOP");
    if (coop && per_sm > 0 && !(env && env[0] == '0'))
      coop_blocks = std::max(1, std::min(run[0].W->nblk, (per_sm * sms) / nrhs));
  }
  for (;;) {
    // the reference's loop head (iterative.rs:60-90): converged / out of steps
    int act[2], na = 0;
    for (int r = 0; r < nrhs; ++r) {
      RhsRun& R = run[r];
      if (!R.active) continue;
      if (R.beta < R.abs_tol) {
        R.loc.converged = 1;
        R.active = false;
      } else if (R.total >= max_iter) {
        R.result = LUM_ERR_NOT_CONVERGED;
        R.active = false;
      } else {
        act[na++] = r;
      }
    }
    if (na == 0) break;
    // One restart cycle is enqueued whole: the device ends it early (S->done)
    // when a step meets the test, and the host reads the outcome once, after
    // the cycle's FP64 residual.  No host round trip per Arnoldi step.
    int jcyc = 0;
    for (int q = 0; q < na; ++q) {
      RhsRun& R = run[act[q]];
      R.jmax = std::min(m, max_iter - R.total);
      jcyc = std::max(jcyc, R.jmax);
      GmresWork& W = *R.W;
      k_start_cycle<<<W.nblk, kVecThreads, 0, st>>>(len, W.r.as<double2>(), W.V.as<double2>(),
                                                    W.state.as<GmresState>(), m);
      LUM_CHECK_LAUNCH();
    }
    for (int j = 0; j < jcyc; ++j) {
      if (na == 2) {
        GmresWork &A = *run[act[0]].W, &B = *run[act[1]].W;
        LUM_TRY(s->apply2(arnoldi_prec, A.V.as<double2>() + (size_t)j * len,
                          B.V.as<double2>() + (size_t)j * len, A.w.as<double2>(),
                          B.w.as<double2>(), &A.state.as<GmresState>()->done,
                          &B.state.as<GmresState>()->done));
      } else {
        GmresWork& A = *run[act[0]].W;
        LUM_TRY(s->apply(arnoldi_prec, A.V.as<double2>() + (size_t)j * len, A.w.as<double2>(),
                         &A.state.as<GmresState>()->done));
      }
      // one launch per step kernel for all live right-hand sides (grid.y);
      // a run whose cycle has ended (its S->done) returns at once
      MgsArgs ma[2];
      for (int q = 0; q < na; ++q) {
        RhsRun& R = run[act[q]];
        GmresWork& W = *R.W;
        ma[q] = MgsArgs{W.w.as<double2>(), W.V.as<double2>(), W.partials.as<double2>(),
                        W.counter.as<unsigned>(), W.state.as<GmresState>(), R.abs_tol,
                        (mode == LUM_SOLVE_FP32_REFINE) ? inner_rel * R.beta : 0.0, R.jmax};
      }
      if (na == 1) ma[1] = ma[0];
      if (coop_blocks > 0) {
        // the whole step in one cooperative launch
        int nr = na;
        double2* p0 = run[act[0]].W->coop_part.as<double2>();
        double2* p1 = run[act[na - 1]].W->coop_part.as<double2>();
        int lenv = len, jv = j;
        void* args[] = {&lenv, &jv, &nr, &ma[0], &ma[1], &p0, &p1};
        LUM_TRY_CUDA(cudaLaunchCooperativeKernel((const void*)k_arnoldi_coop,
                                                 dim3(coop_blocks, na), dim3(kVecThreads),
                                                 args, 0, st));
        g_launches.fetch_add(1, std::memory_order_relaxed);
      } else {
        const dim3 grid(run[act[0]].W->nblk, na);
        for (int i = 0; i <= j; ++i) {
          k_mgs<<<grid, kVecThreads, 0, st>>>(len, i, j, ma[0], ma[1]);
          LUM_CHECK_LAUNCH();
        }
        k_mgs_final<<<grid, kVecThreads, 0, st>>>(len, j, ma[0], ma[1]);
        LUM_CHECK_LAUNCH();
        k_next_basis<<<grid, kVecThreads, 0, st>>>(len, j, ma[0], ma[1]);
        LUM_CHECK_LAUNCH();
      }
    }
    for (int q = 0; q < na; ++q) {
      RhsRun& R = run[act[q]];
      GmresWork& W = *R.W;
      k_backsub<<<1, kVecThreads, 0, st>>>(W.state.as<GmresState>());
      LUM_CHECK_LAUNCH();
      k_update_x<<<W.nblk, kVecThreads, 0, st>>>(len, R.x, W.V.as<double2>(),
                                                 W.state.as<GmresState>());
      LUM_CHECK_LAUNCH();
    }
    // true residual in FP64 (iterative.rs:147-151)
    if (na == 2) {
      RhsRun &A = run[act[0]], &B = run[act[1]];
      LUM_TRY(s->apply2(LUM_FP64, A.x, B.x, A.W->tmp.as<double2>(), B.W->tmp.as<double2>(),
                        nullptr, nullptr));
    } else {
      RhsRun& A = run[act[0]];
      LUM_TRY(s->apply(LUM_FP64, A.x, A.W->tmp.as<double2>()));
    }
    for (int q = 0; q < na; ++q) {
      RhsRun& R = run[act[q]];
      GmresWork& W = *R.W;
      R.loc.matvecs_fp64++;
      k_residual<<<W.nblk, kVecThreads, 0, st>>>(len, R.b, W.tmp.as<double2>(), W.r.as<double2>(),
                                                 W.partials.as<double2>(),
                                                 W.counter.as<unsigned>(),
                                                 W.state.as<GmresState>());
      LUM_CHECK_LAUNCH();
    }
    for (int q = 0; q < na; ++q) LUM_TRY(read_scalars(*run[act[q]].W, st));
    for (int q = 0; q < na; ++q) {
      RhsRun& R = run[act[q]];
      const GmresState* H = R.W->h_state;
      const int steps = H->jdone;
      R.total += steps;
      if (arnoldi_prec == LUM_FP32)
        R.loc.matvecs_fp32 += steps;
      else
        R.loc.matvecs_fp64 += steps;
      if (H->bad) {
        set_error("GMRES breakdown: non-finite residual estimate");
        return LUM_ERR_DEVICE;
      }
      R.beta = H->scal[3];
      R.loc.restarts++;
      if (!std::isfinite(R.beta)) {
        set_error("GMRES breakdown: non-finite residual");
        return LUM_ERR_DEVICE;
      }
    }
  }
  const double secs =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  lum_status result = LUM_OK;
  for (int r = 0; r < nrhs; ++r) {
    RhsRun& R = run[r];
    R.loc.iterations = R.total;
    R.loc.rel_residual = R.rhs_norm > 0.0 ? R.beta / R.rhs_norm : 0.0;
    R.loc.matvecs_reference = R.total + 2 * R.loc.restarts + (R.loc.restarts == 0 ? 1 : 0);
    R.loc.seconds = secs;
    if (R.result == LUM_ERR_NOT_CONVERGED) {
      set_error("Solver failed to converge after %d iterations (residual: %.2e)", max_iter,
                R.loc.rel_residual);
      result = LUM_ERR_NOT_CONVERGED;
    }
    if (info) info[r] = R.loc;
  }
  return result;
}

lum_status lum_gmres_device(lum_session* s, const double2* b, double2* x, double tol,
                            int max_iter, int restart, int mode, lum_solve_info* info,
                            cudaStream_t st) {
  return lum_gmres_device_multi(s, 1, &b, &x, tol, max_iter, restart, mode, info, st);
}
