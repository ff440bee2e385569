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

#include <chrono>
#include <cmath>

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

// Publishes this block's partial; returns true in the last block to finish,
// whose thread 0 then holds the ordered total in *total.
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
  if (threadIdx.x == 0) {
    __threadfence();
    double2 s = make_double2(0.0, 0.0);
    volatile double2* vp = partials;
    for (unsigned b = 0; b < gridDim.x; ++b) {
      s.x += vp[b].x;
      s.y += vp[b].y;
    }
    *total = s;
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
}

// MGS projection i of column j: w -= h_{i-1,j} v_{i-1} (i>0); h_{i,j} = <v_i, w>.
__global__ void __launch_bounds__(kVecThreads)
k_mgs(int len, double2* __restrict__ w, const double2* __restrict__ V, int i, int j,
      double2* partials, unsigned* counter, GmresState* S) {
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
  if (last_block_total(acc, partials, counter, &tot) && threadIdx.x == 0)
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
__global__ void __launch_bounds__(kVecThreads)
k_mgs_final(int len, double2* __restrict__ w, const double2* __restrict__ V, int j,
            double2* partials, unsigned* counter, GmresState* S) {
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
  if (last_block_total(acc, partials, counter, &tot) && threadIdx.x == 0) {
    const double hn = sqrt(tot.x);
    S->scal[1] = hn;
    double2* H = S->H;
    H[(j + 1) * kM + j] = make_double2(hn, 0.0);
    for (int i = 0; i < j; ++i) {
      double c = S->cs[i];
      double2 s = S->sn[i];
      double2 hij = H[i * kM + j], hi1 = H[(i + 1) * kM + j];
      double2 t1 = dmul(s, hi1);
      double2 temp = make_double2(c * hij.x + t1.x, c * hij.y + t1.y);
      double2 t2 = dmul(make_double2(-s.x, s.y), hij);  // -conj(s) * h_ij
      H[(i + 1) * kM + j] = make_double2(t2.x + c * hi1.x, t2.y + c * hi1.y);
      H[i * kM + j] = temp;
    }
    double c;
    double2 s;
    givens(H[j * kM + j], H[(j + 1) * kM + j], &c, &s);
    S->cs[j] = c;
    S->sn[j] = s;
    double2 hjj = H[j * kM + j], hj1 = H[(j + 1) * kM + j];
    double2 t1 = dmul(s, hj1);
    H[j * kM + j] = make_double2(c * hjj.x + t1.x, c * hjj.y + t1.y);
    H[(j + 1) * kM + j] = make_double2(0.0, 0.0);
    double2 gj = S->g[j], gj1 = S->g[j + 1];
    double2 t3 = dmul(s, gj1);
    double2 t4 = dmul(make_double2(-s.x, s.y), gj);
    S->g[j] = make_double2(c * gj.x + t3.x, c * gj.y + t3.y);
    S->g[j + 1] = make_double2(t4.x + c * gj1.x, t4.y + c * gj1.y);
    S->scal[2] = dabs(S->g[j + 1]);
  }
}

// v_{j+1} = w / h_{j+1,j}, or 0 on a lucky breakdown (iterative.rs:101-106)
__global__ void __launch_bounds__(kVecThreads)
k_next_basis(int len, const double2* __restrict__ w, double2* __restrict__ vnext,
             const GmresState* S) {
  const double hn = S->scal[1];
  const bool ok = hn > 1e-30;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < len; q += gridDim.x * blockDim.x) {
    double2 a = w[q];
    vnext[q] = ok ? make_double2(a.x / hn, a.y / hn) : make_double2(0.0, 0.0);
  }
}

// Back substitution H[0..j,0..j] y = g[0..j] (iterative.rs:194-206).
__global__ void k_backsub(int j, GmresState* S) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int i = j - 1; i >= 0; --i) {
    double2 sum = S->g[i];
    for (int q = i + 1; q < j; ++q) {
      double2 t = dmul(S->H[i * kM + q], S->y[q]);
      sum.x -= t.x;
      sum.y -= t.y;
    }
    double2 hii = S->H[i * kM + i];
    S->y[i] = (dabs(hii) > 1e-30) ? ddiv(sum, hii) : make_double2(0.0, 0.0);
  }
}

// x += sum_i y_i v_i (iterative.rs:142-144)
__global__ void __launch_bounds__(kVecThreads)
k_update_x(int len, double2* __restrict__ x, const double2* __restrict__ V, int j,
           const GmresState* S) {
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
  LUM_TRY_CUDA(cudaMemcpyAsync(W.h_state->scal, W.state.as<GmresState>()->scal,
                               sizeof(double) * 8, cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));
  return LUM_OK;
}

}  // namespace lum

using namespace lum;

// Host driver; called from the C ABI with device vectors.
lum_status lum_gmres_device(lum_session* s, const double2* b, double2* x, double tol,
                            int max_iter, int restart, int mode, lum_solve_info* info,
                            cudaStream_t st) {
  auto t0 = std::chrono::steady_clock::now();
  lum_solve_info loc{};
  const int len = s->dim;
  if (restart <= 0) restart = 30;
  const int m = std::min(std::min(restart, len), kMaxRestart);
  GmresWork& W = s->gw;
  LUM_TRY(W.ensure(len, m, st));
  GmresState* S = W.state.as<GmresState>();
  double2* V = W.V.as<double2>();
  double2* w = W.w.as<double2>();
  double2* r = W.r.as<double2>();
  double2* tmp = W.tmp.as<double2>();
  double2* parts = W.partials.as<double2>();
  unsigned* cnt = W.counter.as<unsigned>();
  const int nb = W.nblk;
  const int arnoldi_prec = (mode == LUM_SOLVE_FP32_REFINE) ? LUM_FP32 : LUM_FP64;
  const double inner_rel = 1e-5;

  LUM_TRY_CUDA(cudaMemsetAsync(x, 0, sizeof(double2) * (size_t)len, st));
  LUM_TRY(vec_norm(b, len, W, 3, st));
  LUM_TRY(read_scalars(W, st));
  const double rhs_norm = W.h_state->scal[3];
  lum_status result = LUM_OK;
  if (!std::isfinite(rhs_norm)) {
    set_error("right-hand side is not finite");
    return LUM_ERR_INVALID;
  }
  if (rhs_norm < 1e-30) {
    loc.converged = 1;
    if (info) *info = loc;
    return LUM_OK;
  }
  const double abs_tol = tol * rhs_norm;
  // r = b - A*0 = b; beta = ||b|| (already in scal[3])
  LUM_TRY_CUDA(cudaMemcpyAsync(r, b, sizeof(double2) * (size_t)len, cudaMemcpyDeviceToDevice, st));
  double beta = rhs_norm;
  int total = 0;
  for (;;) {
    if (beta < abs_tol) {
      loc.converged = 1;
      break;
    }
    if (total >= max_iter) {
      result = LUM_ERR_NOT_CONVERGED;
      break;
    }
    k_start_cycle<<<nb, kVecThreads, 0, st>>>(len, r, V, S, m);
    LUM_CHECK_LAUNCH();
    int j = 0;
    while (j < m && total < max_iter) {
      LUM_TRY(s->apply(arnoldi_prec, V + (size_t)j * len, w));
      if (arnoldi_prec == LUM_FP32)
        loc.matvecs_fp32++;
      else
        loc.matvecs_fp64++;
      for (int i = 0; i <= j; ++i) {
        k_mgs<<<nb, kVecThreads, 0, st>>>(len, w, V, i, j, parts, cnt, S);
        LUM_CHECK_LAUNCH();
      }
      k_mgs_final<<<nb, kVecThreads, 0, st>>>(len, w, V, j, parts, cnt, S);
      LUM_CHECK_LAUNCH();
      k_next_basis<<<nb, kVecThreads, 0, st>>>(len, w, V + (size_t)(j + 1) * len, S);
      LUM_CHECK_LAUNCH();
      LUM_TRY(read_scalars(W, st));
      const double gabs = W.h_state->scal[2];
      total++;
      j++;
      if (!std::isfinite(gabs)) {
        set_error("GMRES breakdown: non-finite residual estimate");
        return LUM_ERR_DEVICE;
      }
      if (gabs < abs_tol) break;
      if (mode == LUM_SOLVE_FP32_REFINE && gabs < inner_rel * beta) break;
    }
    k_backsub<<<1, 32, 0, st>>>(j, S);
    LUM_CHECK_LAUNCH();
    k_update_x<<<nb, kVecThreads, 0, st>>>(len, x, V, j, S);
    LUM_CHECK_LAUNCH();
    // true residual in FP64 (iterative.rs:147-151)
    LUM_TRY(s->apply(LUM_FP64, x, tmp));
    loc.matvecs_fp64++;
    k_residual<<<nb, kVecThreads, 0, st>>>(len, b, tmp, r, parts, cnt, S);
    LUM_CHECK_LAUNCH();
    LUM_TRY(read_scalars(W, st));
    beta = W.h_state->scal[3];
    loc.restarts++;
    if (!std::isfinite(beta)) {
      set_error("GMRES breakdown: non-finite residual");
      return LUM_ERR_DEVICE;
    }
    if (beta < abs_tol) {
      loc.converged = 1;
      break;
    }
    if (total >= max_iter) {
      result = LUM_ERR_NOT_CONVERGED;
      break;
    }
  }
  loc.iterations = total;
  loc.rel_residual = beta / rhs_norm;
  loc.matvecs_reference = total + 2 * loc.restarts + (loc.restarts == 0 ? 1 : 0);
  loc.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (result == LUM_ERR_NOT_CONVERGED)
    set_error("Solver failed to converge after %d iterations (residual: %.2e)", max_iter,
              loc.rel_residual);
  if (info) *info = loc;
  return result;
}
