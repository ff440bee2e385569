// batch.cu -- many independent CDA systems solved by one batched GMRES.
//
// K clusters of uneven size (each with its own positions, alpha^-1, wave
// number and FCD cell) are concatenated into one dipole range.  Every Krylov
// vector is one 3*N_total vector that holds all systems' segments, so a
// single persistent pair-kernel launch applies all K operators (otf.cu), and
// the per-system work of GMRES -- modified Gram-Schmidt, the Givens update,
// back substitution, the solution update and the FP64 residual -- runs as one
// thread-block cluster per system that reduces through distributed shared
// memory (fixed summation order: results do not depend on scheduling).
//
// The algorithm per system is the reference's restarted GMRES
// (iterative.rs:33-206): x0 = 0, MGS in the order of iterative.rs:92-96,
// Givens with real c and complex s (iterative.rs:180-191), the in-cycle test
// |g_{j+1}| < tol*||b|| and the FP64 true residual at the end of a cycle.
// In the FP32+refine mode the Arnoldi products run in FP32 and a cycle also
// ends once |g_{j+1}| < 1e-5 * beta, as in the single-system solver.
//
// One restart cycle (start, m Arnoldi steps, update, FP64 residual and a
// 4-byte read of the number of systems still active) is captured once as a
// CUDA graph and replayed.  Per-system flags decide on the device whether a
// system's cycle has ended (done) or whether it has converged or run out of
// iterations (frozen); the kernels of such systems return at once and their
// pair-kernel items are skipped when drawn.  The host synchronises once per
// cycle for the whole batch.
#include "lumina_internal.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <new>

namespace cg = cooperative_groups;

namespace lum {
namespace {

constexpr int kBT = 256;          // threads per CTA of the per-system kernels
constexpr int kBM = kMaxRestart;
constexpr int kMaxCluster = 8;    // portable cluster size

struct BatchSysState {
  double2 H[(kBM + 1) * kBM];
  double cs[kBM];
  double2 sn[kBM];
  double2 g[kBM + 1];
  double rhs_norm, abs_tol, beta, inner_thr;
  int total, restarts, converged, jmax;
  int mv_arnoldi, mv_fp64, pad0, pad1;
};

struct BatchCtl {
  double tol;
  double inner_rel;
  int max_iter;
  int m;
  int refine;
  int active;   // systems still active after the last cycle (host reads it)
  int live_items;  // symmetric work items of those systems (host reads it with active)
};

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 zconjmul(double2 a, double2 b) {  // conj(a) * b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 zdiv(double2 a, double2 b) {
  const double n = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / n, (a.y * b.x - a.x * b.y) / n);
}
__device__ __forceinline__ double zabs(double2 a) { return hypot(a.x, a.y); }

// Per-system segment of the cluster: CTA `rank` of `nb` owns elements
// q = rank*kBT + tid + e*nb*kBT (e < EPT) of the system's 3N entries.
struct Seg {
  int s, rank, nb;
  size_t base;
  int len;
  __device__ __forceinline__ int q(int e) const {
    return rank * kBT + (int)threadIdx.x + e * nb * kBT;
  }
};

__device__ __forceinline__ Seg make_seg(const int* __restrict__ sys_off) {
  cg::cluster_group cl = cg::this_cluster();
  Seg g;
  g.nb = (int)cl.num_blocks();
  g.rank = (int)cl.block_rank();
  g.s = blockIdx.x / g.nb;
  const int o0 = sys_off[g.s], o1 = sys_off[g.s + 1];
  g.base = 3 * (size_t)o0;
  g.len = 3 * (o1 - o0);
  return g;
}

// Scratch for cluster sums (double-buffered slot: one cluster barrier per sum).
struct ClusterSum {
  double2 warp[kBT / 32];
  double2 slot[2];
  int phase;
};

// Sum of v over every thread of the cluster, returned to all threads.  The
// block total is formed in a fixed order, then every thread adds the CTA
// totals of ranks 0..nb-1 read from distributed shared memory.  The slot
// written by sum t is rewritten by sum t+2 only after every CTA has passed
// the barrier of sum t+1, i.e. after all reads of sum t.
__device__ double2 cluster_sum(double2 v, ClusterSum& cs) {
  cg::cluster_group cl = cg::this_cluster();
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) cs.warp[wid] = v;
  __syncthreads();
  const int ph = cs.phase;
  if (threadIdx.x == 0) {
    double2 t = make_double2(0.0, 0.0);
    for (int w = 0; w < kBT / 32; ++w) {
      t.x += cs.warp[w].x;
      t.y += cs.warp[w].y;
    }
    cs.slot[ph] = t;
  }
  cl.sync();
  double2 t = make_double2(0.0, 0.0);
  const int nb = (int)cl.num_blocks();
  for (int r = 0; r < nb; ++r) {
    const double2 p = *cl.map_shared_rank(&cs.slot[ph], r);
    t.x += p.x;
    t.y += p.y;
  }
  __syncthreads();  // every thread has read the phase before thread 0 flips it
  if (threadIdx.x == 0) cs.phase = ph ^ 1;
  return t;
}

// x = 0, r = b, ||b||; per-system control state and flags.
template <int EPT>
__global__ void __launch_bounds__(kBT)
k_bat_init(const int* __restrict__ sys_off, const double2* __restrict__ b,
           double2* __restrict__ x, double2* __restrict__ r, BatchSysState* __restrict__ st,
           BatchFlags* __restrict__ flags, const BatchCtl* __restrict__ ctl) {
  __shared__ ClusterSum cs;
  if (threadIdx.x == 0) cs.phase = 0;
  const Seg sg = make_seg(sys_off);
  double2 acc = make_double2(0.0, 0.0);
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    const int q = sg.q(e);
    if (q < sg.len) {
      const double2 bb = b[sg.base + q];
      x[sg.base + q] = make_double2(0.0, 0.0);
      r[sg.base + q] = bb;
      acc.x += bb.x * bb.x + bb.y * bb.y;
    }
  }
  const double nb = sqrt(cluster_sum(acc, cs).x);
  if (sg.rank == 0 && threadIdx.x == 0) {
    BatchSysState& S = st[sg.s];
    S.rhs_norm = nb;
    S.abs_tol = ctl->tol * nb;
    S.beta = nb;
    S.inner_thr = 0.0;
    S.total = S.restarts = S.converged = S.jmax = 0;
    S.mv_arnoldi = S.mv_fp64 = 0;
    BatchFlags f{0, 0, 0, 0};
    if (!isfinite(nb)) {
      f.bad = 1;
      f.frozen = 1;
    } else if (nb < 1e-30 || nb < S.abs_tol) {
      S.converged = 1;
      f.frozen = 1;
    } else if (ctl->max_iter <= 0) {
      f.frozen = 1;
    }
    flags[sg.s] = f;
  }
  cg::this_cluster().sync();  // no CTA leaves while its slots may still be read
}

// v0 = r / beta, g = beta e1, cycle flags reset, jmax and the inner threshold.
template <int EPT>
__global__ void __launch_bounds__(kBT)
k_bat_start(const int* __restrict__ sys_off, const double2* __restrict__ r,
            double2* __restrict__ V, BatchSysState* __restrict__ st,
            BatchFlags* __restrict__ flags, BatchCtl* __restrict__ ctl) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->active = 0;
    ctl->live_items = 0;
  }
  const Seg sg = make_seg(sys_off);
  if (flags[sg.s].frozen) return;  // cluster-uniform
  BatchSysState& S = st[sg.s];
  const double beta = S.beta;
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    const int q = sg.q(e);
    if (q < sg.len) {
      const double2 a = r[sg.base + q];
      V[sg.base + q] = make_double2(a.x / beta, a.y / beta);
    }
  }
  if (sg.rank == 0) {
    const int m = ctl->m;
    if ((int)threadIdx.x <= m) S.g[threadIdx.x] = make_double2(threadIdx.x == 0 ? beta : 0.0, 0.0);
    if (threadIdx.x == 0) {
      S.jmax = min(min(m, sg.len), ctl->max_iter - S.total);  // restart min(m, 3N) per system
      S.inner_thr = ctl->refine ? ctl->inner_rel * beta : 0.0;
      flags[sg.s].done = 0;
      flags[sg.s].jdone = 0;
    }
  }
}

// Arnoldi step j of every active system: MGS against v_0..v_j with w and the
// basis vector held in registers, ||w||, the rotations and the step's
// convergence test, then v_{j+1} = w / h_{j+1,j}.
template <int EPT>
__global__ void __launch_bounds__(kBT)
k_bat_arnoldi(int j, size_t ldv, const int* __restrict__ sys_off, double2* __restrict__ V,
              const double2* __restrict__ w, BatchSysState* __restrict__ st,
              BatchFlags* __restrict__ flags) {
  __shared__ ClusterSum cs;
  __shared__ double2 sH[kBM + 2], sS[kBM], sG[2];
  __shared__ double sC[kBM];
  __shared__ double s_hn;
  __shared__ int s_done;
  const Seg sg = make_seg(sys_off);
  {
    const BatchFlags f = flags[sg.s];
    if (f.frozen || f.done) return;  // cluster-uniform, read before any cluster barrier
  }
  BatchSysState& S = st[sg.s];
  const int t = threadIdx.x;
  if (t == 0) cs.phase = 0;
  // rank 0 rewrites these after the last cluster barrier: read them first
  if (t < j) {
    sC[t] = S.cs[t];
    sS[t] = S.sn[t];
  }
  if (t < 2) sG[t] = S.g[j + t];
  double2 wr[EPT];
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    const int q = sg.q(e);
    wr[e] = q < sg.len ? w[sg.base + q] : make_double2(0.0, 0.0);
  }
  for (int i = 0; i <= j; ++i) {
    // v_i is read twice (dot, then subtract): the second read hits L1/L2 and
    // keeps the register footprint at w alone
    const double2* vi = V + (size_t)i * ldv + sg.base;
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      const int q = sg.q(e);
      const double2 v = q < sg.len ? vi[q] : make_double2(0.0, 0.0);
      const double2 d = zconjmul(v, wr[e]);
      acc.x += d.x;
      acc.y += d.y;
    }
    const double2 h = cluster_sum(acc, cs);
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      const int q = sg.q(e);
      const double2 v = q < sg.len ? vi[q] : make_double2(0.0, 0.0);
      const double2 p = zmul(v, h);
      wr[e].x -= p.x;
      wr[e].y -= p.y;
    }
    if (t == 0) sH[i] = h;
  }
  double2 acc = make_double2(0.0, 0.0);
#pragma unroll
  for (int e = 0; e < EPT; ++e) acc.x += wr[e].x * wr[e].x + wr[e].y * wr[e].y;
  const double hn = sqrt(cluster_sum(acc, cs).x);
  if (t == 0) {
    // rotations of iterative.rs:98-127 on column j (every CTA, same inputs)
    sH[j + 1] = make_double2(hn, 0.0);
    for (int i = 0; i < j; ++i) {
      const double c = sC[i];
      const double2 s = sS[i];
      const double2 hij = sH[i], hi1 = sH[i + 1];
      const double2 t1 = zmul(s, hi1);
      const double2 t2 = zmul(make_double2(-s.x, s.y), hij);  // -conj(s) * h_ij
      sH[i] = make_double2(c * hij.x + t1.x, c * hij.y + t1.y);
      sH[i + 1] = make_double2(t2.x + c * hi1.x, t2.y + c * hi1.y);
    }
    const double2 a = sH[j], bq = sH[j + 1];
    double c;
    double2 s;
    if (zabs(bq) < 1e-30) {
      c = 1.0;
      s = make_double2(0.0, 0.0);
    } else if (zabs(a) < 1e-30) {
      c = 0.0;
      s = zdiv(bq, make_double2(zabs(bq), 0.0));
    } else {
      const double rr = sqrt((a.x * a.x + a.y * a.y) + (bq.x * bq.x + bq.y * bq.y));
      c = zabs(a) / rr;
      const double2 an = zdiv(a, make_double2(zabs(a), 0.0));
      const double2 tt = zmul(an, make_double2(bq.x, -bq.y));
      s = make_double2(tt.x / rr, tt.y / rr);
    }
    const double2 t1 = zmul(s, bq);
    sH[j] = make_double2(c * a.x + t1.x, c * a.y + t1.y);
    sH[j + 1] = make_double2(0.0, 0.0);
    const double2 gj = sG[0], gj1 = sG[1];
    const double2 t3 = zmul(s, gj1);
    const double2 t4 = zmul(make_double2(-s.x, s.y), gj);
    const double2 g0 = make_double2(c * gj.x + t3.x, c * gj.y + t3.y);
    const double2 g1 = make_double2(t4.x + c * gj1.x, t4.y + c * gj1.y);
    const double gabs = zabs(g1);
    const int bad = !isfinite(gabs);
    const int done = bad || gabs < S.abs_tol || gabs < S.inner_thr || j + 1 >= S.jmax;
    s_done = done;
    s_hn = hn;
    if (sg.rank == 0) {
      S.g[j] = g0;
      S.g[j + 1] = g1;
      S.cs[j] = c;
      S.sn[j] = s;
      for (int i = 0; i <= j + 1; ++i) S.H[i * kBM + j] = sH[i];
      BatchFlags& f = flags[sg.s];
      f.jdone = j + 1;
      f.bad = bad;
      f.done = done;
    }
  }
  __syncthreads();
  if (!s_done) {
    // v_{j+1} = w / h_{j+1,j}, or 0 on a lucky breakdown (iterative.rs:101-106)
    const double h = s_hn;
    const bool ok = h > 1e-30;
    double2* vn = V + (size_t)(j + 1) * ldv + sg.base;
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      const int q = sg.q(e);
      if (q < sg.len) vn[q] = ok ? make_double2(wr[e].x / h, wr[e].y / h) : make_double2(0.0, 0.0);
    }
  }
  cg::this_cluster().sync();
}

// Back substitution H y = g over the jdone steps (iterative.rs:194-206),
// then x += V y on the system's segment.
__device__ __forceinline__ int tri_at(int r, int j) { return r * j - (r * (r - 1)) / 2; }

template <int EPT>
__global__ void __launch_bounds__(kBT)
k_bat_update(size_t ldv, const int* __restrict__ sys_off, const double2* __restrict__ V,
             double2* __restrict__ x, const BatchSysState* __restrict__ st,
             const BatchFlags* __restrict__ flags) {
  __shared__ double2 sT[kBM * (kBM + 1) / 2];
  __shared__ double2 sg_[kBM], sy[kBM];
  const Seg sg = make_seg(sys_off);
  const BatchFlags f = flags[sg.s];
  if (f.frozen) return;
  const int j = f.jdone;
  const BatchSysState& S = st[sg.s];
  for (int e = threadIdx.x; e < j * j; e += blockDim.x) {
    const int r = e / j, c = e % j;
    if (c >= r) sT[tri_at(r, j) + (c - r)] = S.H[r * kBM + c];
  }
  if ((int)threadIdx.x < j) sg_[threadIdx.x] = S.g[threadIdx.x];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = j - 1; i >= 0; --i) {
      double2 sum = sg_[i];
      const double2* row = sT + tri_at(i, j) - i;
      for (int q = i + 1; q < j; ++q) {
        const double2 tq = zmul(row[q], sy[q]);
        sum.x -= tq.x;
        sum.y -= tq.y;
      }
      const double2 hii = row[i];
      sy[i] = (zabs(hii) > 1e-30) ? zdiv(sum, hii) : make_double2(0.0, 0.0);
    }
  }
  __syncthreads();
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    const int q = sg.q(e);
    if (q < sg.len) {
      double2 acc = x[sg.base + q];
      for (int i = 0; i < j; ++i) {
        const double2 tq = zmul(V[(size_t)i * ldv + sg.base + q], sy[i]);
        acc.x += tq.x;
        acc.y += tq.y;
      }
      x[sg.base + q] = acc;
    }
  }
}

// r = b - A x (A x in ax), beta = ||r||, iteration bookkeeping and the
// end-of-cycle tests (iterative.rs:147-157).
template <int EPT>
__global__ void __launch_bounds__(kBT)
k_bat_residual(const int* __restrict__ sys_off, const double2* __restrict__ b,
               const double2* __restrict__ ax, double2* __restrict__ r,
               BatchSysState* __restrict__ st, BatchFlags* __restrict__ flags,
               BatchCtl* __restrict__ ctl, const int* __restrict__ sys_nb) {
  __shared__ ClusterSum cs;
  const Seg sg = make_seg(sys_off);
  const BatchFlags f = flags[sg.s];
  if (f.frozen) return;
  if (threadIdx.x == 0) cs.phase = 0;
  double2 acc = make_double2(0.0, 0.0);
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    const int q = sg.q(e);
    if (q < sg.len) {
      const double2 bb = b[sg.base + q], aa = ax[sg.base + q];
      const double2 d = make_double2(bb.x - aa.x, bb.y - aa.y);
      r[sg.base + q] = d;
      acc.x += d.x * d.x + d.y * d.y;
    }
  }
  const double beta = sqrt(cluster_sum(acc, cs).x);
  if (sg.rank == 0 && threadIdx.x == 0) {
    BatchSysState& S = st[sg.s];
    BatchFlags& F = flags[sg.s];
    S.total += f.jdone;
    S.mv_arnoldi += f.jdone;
    S.mv_fp64 += 1;
    S.restarts += 1;
    S.beta = beta;
    if (f.bad || !isfinite(beta)) {
      F.bad = 1;
      F.frozen = 1;
    } else if (beta < S.abs_tol) {
      S.converged = 1;
      F.frozen = 1;
    } else if (S.total >= ctl->max_iter) {
      F.frozen = 1;
    } else {
      atomicAdd(&ctl->active, 1);
      if (sys_nb) {
        const int nb = sys_nb[sg.s];
        atomicAdd(&ctl->live_items, nb * (nb + 1) / 2);
      }
    }
  }
  cg::this_cluster().sync();
}

template <typename... P, typename... A>
lum_status launch_cluster(void (*kern)(P...), int K, int cl, cudaStream_t st, A... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(K * cl));
  cfg.blockDim = dim3(kBT);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cl;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  g_launches.fetch_add(1, std::memory_order_relaxed);
  LUM_TRY_CUDA(cudaLaunchKernelEx(&cfg, kern, args...));
  return LUM_OK;
}

}  // namespace
}  // namespace lum

using namespace lum;

struct lum_batch {
  lum_ctx* ctx = nullptr;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  int K = 0, N = 0;
  int ept = 8, cl = 1;
  std::vector<int> off;
  BatchGeom g;
  DevBuf d_off, d_row_sys, d_ns32, d_ns64, d_ch32, d_ch64, d_k, d_cell;
  DevBuf pos64, hi, lo, inv_alpha, near_j, fcd64, fcd32;
  BatchQueue q32, q64, qsym;
  DevBuf d_nb;
  DevBuf part;
  DevBuf xin, yout;             // host-path staging of the matvec
  // solver workspace
  int m = 0;
  DevBuf V, w, r, tmp, xs, bs, state, flags, ctl;
  int* h_active = nullptr;  // [0] active systems, [1] their symmetric work items
  BatchSysState* h_state = nullptr;
  BatchFlags* h_flags = nullptr;
  // cycle graphs: FP64, FP32 on the split work list, FP32 on the symmetric one
  cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
  int graph_m[3] = {0, 0, 0};
  uint64_t graph_launches[3] = {0, 0, 0};
  int use_graph = 1;
  // A cycle of FP32 products takes the symmetric build g.sym32 while the
  // active systems hold at least sym_min_items symmetric items; below that
  // the split list, whose finer items keep the grid busy on a few systems.
  int sym_min_items = 0;
  // Right-hand-side batch (lum_batch_create_rhs): K vectors of one session's
  // operator, applied through that session instead of the pair work list.
  lum_session* src = nullptr;
  ~lum_batch() {
    for (auto& gx : graph)
      if (gx) cudaGraphExecDestroy(gx);
    if (h_active) cudaFreeHost(h_active);
    if (h_state) cudaFreeHost(h_state);
    if (h_flags) cudaFreeHost(h_flags);
  }
};

namespace {

bool bad_arg(const void* p, const char* what) {
  if (p) return false;
  set_error("null pointer: %s", what);
  return true;
}

// The per-system kernels are instantiated for EPT elements per thread.
template <template <int> class F, typename... A>
lum_status dispatch_ept(int ept, A... args) {
  switch (ept) {
    case 4: return F<4>::run(args...);
    case 8: return F<8>::run(args...);
    case 16: return F<16>::run(args...);
    default: return F<32>::run(args...);
  }
}

template <int E>
struct RunInit {
  static lum_status run(lum_batch* B, const double2* b) {
    return launch_cluster(k_bat_init<E>, B->K, B->cl, B->stream, B->d_off.as<const int>(), b,
                          B->xs.as<double2>(), B->r.as<double2>(), B->state.as<BatchSysState>(),
                          B->flags.as<BatchFlags>(), B->ctl.as<const BatchCtl>());
  }
};
template <int E>
struct RunStart {
  static lum_status run(lum_batch* B) {
    return launch_cluster(k_bat_start<E>, B->K, B->cl, B->stream, B->d_off.as<const int>(),
                          B->r.as<const double2>(), B->V.as<double2>(),
                          B->state.as<BatchSysState>(), B->flags.as<BatchFlags>(),
                          B->ctl.as<BatchCtl>());
  }
};
template <int E>
struct RunArnoldi {
  static lum_status run(lum_batch* B, int j) {
    return launch_cluster(k_bat_arnoldi<E>, B->K, B->cl, B->stream, j, (size_t)3 * B->N,
                          B->d_off.as<const int>(), B->V.as<double2>(), B->w.as<const double2>(),
                          B->state.as<BatchSysState>(), B->flags.as<BatchFlags>());
  }
};
template <int E>
struct RunUpdate {
  static lum_status run(lum_batch* B) {
    return launch_cluster(k_bat_update<E>, B->K, B->cl, B->stream, (size_t)3 * B->N,
                          B->d_off.as<const int>(), B->V.as<const double2>(), B->xs.as<double2>(),
                          B->state.as<const BatchSysState>(), B->flags.as<const BatchFlags>());
  }
};
template <int E>
struct RunResidual {
  static lum_status run(lum_batch* B) {
    return launch_cluster(k_bat_residual<E>, B->K, B->cl, B->stream, B->d_off.as<const int>(),
                          B->bs.as<const double2>(), B->tmp.as<const double2>(),
                          B->r.as<double2>(), B->state.as<BatchSysState>(),
                          B->flags.as<BatchFlags>(), B->ctl.as<BatchCtl>(),
                          B->d_nb.as<const int>());
  }
};

// Picks the FP32 pair scheme of a cluster batch (split work list or a
// symmetric build) by timing; see the creation code for the override.
lum_status batch_choose_scheme(lum_batch* B, cudaStream_t st) {
  BatchGeom& g = B->g;
  g.sym32 = 0;
  const char* e = std::getenv("LUMINA_BATCH_SYM");
  if (e && e[0] == '0') return LUM_OK;
  if (e && e[0] >= '1' && e[0] <= '9') {
    g.sym32 = std::min(e[0] - '0', batch_sym_variants());
    return LUM_OK;
  }
  const size_t len = 3 * (size_t)B->N;
  DevBuf xz, yz;
  LUM_TRY(xz.alloc(sizeof(double2) * len));
  LUM_TRY(yz.alloc(sizeof(double2) * len));
  LUM_TRY_CUDA(cudaMemsetAsync(xz.p, 0, xz.bytes, st));
  cudaEvent_t e0, e1;
  LUM_TRY_CUDA(cudaEventCreate(&e0));
  LUM_TRY_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int choice = 0;
  lum_status status = LUM_OK;
  for (int v = 0; v <= batch_sym_variants() && status == LUM_OK; ++v) {
    g.sym32 = v;
    float ms = 1e30f;
    for (int rep = 0; rep < 4 && status == LUM_OK; ++rep) {
      cudaEventRecord(e0, st);
      status = batch_apply(g, LUM_FP32, xz.as<double2>(), yz.as<double2>(), B->part.p, B->q32,
                           nullptr, 0, st);
      cudaEventRecord(e1, st);
      if (status != LUM_OK) break;
      const cudaError_t ce = cudaEventSynchronize(e1);
      if (ce != cudaSuccess) {
        status = cuda_status(ce, "batch scheme timing", __FILE__, __LINE__);
        break;
      }
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (rep > 0) ms = std::min(ms, t);  // the first launch warms
    }
    if (status == LUM_OK && ms < best) {
      best = ms;
      choice = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  g.sym32 = choice;
  return status;
}

lum_status batch_workspace(lum_batch* B, int m) {
  const size_t len = 3 * (size_t)B->N;
  if (B->m < m || !B->V.p) {
    LUM_TRY(B->V.alloc(sizeof(double2) * (size_t)(m + 1) * len));
    B->m = m;
    for (auto& gx : B->graph)
      if (gx) {
        cudaGraphExecDestroy(gx);
        gx = nullptr;
      }
  }
  if (!B->w.p) {
    LUM_TRY(B->w.alloc(sizeof(double2) * len));
    LUM_TRY(B->r.alloc(sizeof(double2) * len));
    LUM_TRY(B->tmp.alloc(sizeof(double2) * len));
    LUM_TRY(B->xs.alloc(sizeof(double2) * len));
    LUM_TRY(B->bs.alloc(sizeof(double2) * len));
    LUM_TRY(B->state.alloc(sizeof(BatchSysState) * (size_t)B->K));
    LUM_TRY(B->flags.alloc(sizeof(BatchFlags) * (size_t)B->K));
    LUM_TRY(B->ctl.alloc(sizeof(BatchCtl)));
    LUM_TRY_CUDA(cudaMemsetAsync(B->flags.p, 0, B->flags.bytes, B->stream));
    if (!B->h_active) LUM_TRY_CUDA(cudaMallocHost((void**)&B->h_active, 2 * sizeof(int)));
    if (!B->h_state)
      LUM_TRY_CUDA(cudaMallocHost((void**)&B->h_state, sizeof(BatchSysState) * (size_t)B->K));
    if (!B->h_flags)
      LUM_TRY_CUDA(cudaMallocHost((void**)&B->h_flags, sizeof(BatchFlags) * (size_t)B->K));
  }
  return LUM_OK;
}

// y = A x for the K vectors of a right-hand-side batch.  An FP32-storage
// cached matrix at FP32 takes the tensor-core product for all K vectors in
// one launch; otherwise (symmetric tile storage included) the session
// operator runs two vectors at a time (the two-vector pair kernels for an
// on-the-fly session).
lum_status rhs_apply(lum_batch* B, int prec, const double2* x, double2* y) {
  lum_session* s = B->src;
  const size_t n3 = (size_t)s->dim;
  if (s->otf.has_somm && s->otf.somm_stale) {
    set_error("the session's Sommerfeld term belongs to another wavelength: call "
              "lum_session_set_sommerfeld after lum_session_set_wavelength");
    return LUM_ERR_INVALID;
  }
  if (s->kind == 1 && !s->cached.packed && s->cached.precision == LUM_FP32 && prec == LUM_FP32)
    return s->cached.apply_multi(x, y, B->K, 1, (long long)n3, LUM_MATMUL_TENSOR, s->stream);
  if (s->kind == 1 && !s->cached.packed && s->cached.precision == LUM_FP64)
    return s->cached.apply_multi(x, y, B->K, 1, (long long)n3, LUM_MATMUL_CUDA_CORES,
                                 s->stream);
  int r = 0;
  for (; r + 1 < B->K; r += 2)
    LUM_TRY(s->apply2(prec, x + r * n3, x + (r + 1) * n3, y + r * n3, y + (r + 1) * n3,
                      nullptr, nullptr));
  if (r < B->K) LUM_TRY(s->apply(prec, x + r * n3, y + r * n3));
  return LUM_OK;
}

// One restart cycle for all systems (the body that is captured as a graph);
// sym != 0 runs its FP32 products on symmetric build sym.
lum_status batch_cycle(lum_batch* B, int mode, int sym) {
  const int prec = (mode == LUM_SOLVE_FP32_REFINE) ? LUM_FP32 : LUM_FP64;
  const size_t len = 3 * (size_t)B->N;
  BatchQueue& qa = (prec == LUM_FP32) ? B->q32 : B->q64;
  BatchGeom g = B->g;
  g.sym32 = sym;
  const BatchFlags* fl = B->flags.as<BatchFlags>();
  LUM_TRY(dispatch_ept<RunStart>(B->ept, B));
  for (int j = 0; j < B->m; ++j) {
    if (B->src)
      LUM_TRY(rhs_apply(B, prec, B->V.as<double2>() + (size_t)j * len, B->w.as<double2>()));
    else
      LUM_TRY(batch_apply(g, prec, B->V.as<double2>() + (size_t)j * len, B->w.as<double2>(),
                          B->part.p, qa, fl, 1, B->stream));
    LUM_TRY(dispatch_ept<RunArnoldi>(B->ept, B, j));
  }
  LUM_TRY(dispatch_ept<RunUpdate>(B->ept, B));
  if (B->src)
    LUM_TRY(rhs_apply(B, LUM_FP64, B->xs.as<double2>(), B->tmp.as<double2>()));
  else
    LUM_TRY(batch_apply(g, LUM_FP64, B->xs.as<double2>(), B->tmp.as<double2>(), B->part.p,
                        B->q64, fl, 2, B->stream));
  LUM_TRY(dispatch_ept<RunResidual>(B->ept, B));
  static_assert(offsetof(BatchCtl, live_items) == offsetof(BatchCtl, active) + sizeof(int),
                "active and live_items are read together");
  LUM_TRY_CUDA(cudaMemcpyAsync(B->h_active, &B->ctl.as<BatchCtl>()->active, 2 * sizeof(int),
                               cudaMemcpyDeviceToHost, B->stream));
  return LUM_OK;
}

// Captures and instantiates the cycle graph of (mode, sym) unless it exists
// for the current restart length.
lum_status batch_graph(lum_batch* B, int mode, int sym) {
  const int gi = (mode == LUM_SOLVE_FP32_REFINE) ? (sym ? 2 : 1) : 0;
  if (!B->graph[gi] || B->graph_m[gi] != B->m) {
    if (B->graph[gi]) {
      cudaGraphExecDestroy(B->graph[gi]);
      B->graph[gi] = nullptr;
    }
    cudaGraph_t gr = nullptr;
    LUM_TRY_CUDA(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
    const uint64_t l0 = g_launches.load();
    lum_status s = batch_cycle(B, mode, sym);
    cudaError_t e = cudaStreamEndCapture(B->stream, &gr);
    if (s != LUM_OK) {
      if (gr) cudaGraphDestroy(gr);
      return s;
    }
    if (e != cudaSuccess) return cuda_status(e, "batch cycle capture", __FILE__, __LINE__);
    B->graph_launches[gi] = g_launches.load() - l0;
    // the captured launches were counted at capture time; count them per replay instead
    g_launches.fetch_sub(B->graph_launches[gi]);
    e = cudaGraphInstantiate(&B->graph[gi], gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) {
      B->graph[gi] = nullptr;
      return cuda_status(e, "batch cycle instantiate", __FILE__, __LINE__);
    }
    B->graph_m[gi] = B->m;
  }
  return LUM_OK;
}

lum_status batch_run_cycle(lum_batch* B, int mode, int sym) {
  const int gi = (mode == LUM_SOLVE_FP32_REFINE) ? (sym ? 2 : 1) : 0;
  if (!B->use_graph) return batch_cycle(B, mode, sym);
  LUM_TRY(batch_graph(B, mode, sym));
  LUM_TRY_CUDA(cudaGraphLaunch(B->graph[gi], B->stream));
  g_launches.fetch_add(B->graph_launches[gi]);
  return LUM_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
int lum_batch_create(lum_ctx* ctx, int n_systems, const int* sys_dipoles, const double* pos,
                     const double* inv_alpha, const double* k, const double* cell, int use_fcd,
                     lum_batch** out) {
  if (bad_arg(ctx, "ctx") || bad_arg(out, "out") || bad_arg(sys_dipoles, "sys_dipoles") ||
      bad_arg(pos, "pos") || bad_arg(inv_alpha, "inv_alpha") || bad_arg(k, "k") ||
      bad_arg(cell, "cell"))
    return LUM_ERR_INVALID;
  *out = nullptr;
  if (n_systems <= 0) {
    set_error("a batch needs at least one system");
    return LUM_ERR_INVALID;
  }
  std::vector<int> off(n_systems + 1, 0);
  int max_len = 0;
  for (int s = 0; s < n_systems; ++s) {
    const int n = sys_dipoles[s];
    if (n <= 0) {
      set_error("system %d has no dipoles", s);
      return LUM_ERR_INVALID;
    }
    if ((long long)off[s] + n > 50000000LL) {
      set_error("batch too large");
      return LUM_ERR_INVALID;
    }
    if (!(std::isfinite(k[s]) && k[s] > 0.0) || !(std::isfinite(cell[s]) && cell[s] >= 0.0)) {
      set_error("system %d: invalid wave number or cell size", s);
      return LUM_ERR_INVALID;
    }
    off[s + 1] = off[s] + n;
    max_len = std::max(max_len, 3 * n);
  }
  const int N = off[n_systems];
  // per-system vector kernels: EPT elements per thread, clusters of <= 8 CTAs
  int ept = 0, clz = 0;
  for (int e : {4, 8, 16, 32}) {
    const int c = (max_len + kBT * e - 1) / (kBT * e);
    if (c <= kMaxCluster) {
      ept = e;
      clz = c;
      break;
    }
  }
  if (!ept) {
    set_error("system of %d dipoles exceeds the batched solver's limit of %d per system",
              max_len / 3, kMaxCluster * kBT * 32 / 3);
    return LUM_ERR_INVALID;
  }
  for (size_t q = 0; q < 3 * (size_t)N; ++q)
    if (!std::isfinite(pos[q])) {
      set_error("non-finite dipole position at index %zu", q / 3);
      return LUM_ERR_INVALID;
    }
  for (size_t q = 0; q < 18 * (size_t)N; ++q)
    if (!std::isfinite(inv_alpha[q])) {
      set_error("non-finite inverse polarisability at dipole %zu", q / 18);
      return LUM_ERR_INVALID;
    }
  lum_batch* B = new (std::nothrow) lum_batch();
  if (!B) return LUM_ERR_OOM;
  B->ctx = ctx;
  B->K = n_systems;
  B->N = N;
  B->off = off;
  B->ept = ept;
  B->cl = clz;
  if (const char* e = std::getenv("LUMINA_BATCH_GRAPH")) B->use_graph = std::atoi(e) != 0;
  auto fail = [&](lum_status s) {
    lum_batch_destroy(B);
    return s;
  };
  cudaError_t ce = cudaSetDevice(ctx->device);
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking);
  if (ce != cudaSuccess) return fail(cuda_status(ce, "batch stream", __FILE__, __LINE__));
  if (lum_status ts = otf_sincos_ready(); ts != LUM_OK) return fail(ts);
  cudaStream_t st = B->stream;

  // host-side layouts
  std::vector<double> p4(4 * (size_t)N, 0.0);
  std::vector<float> h4(4 * (size_t)N, 0.f), l4(4 * (size_t)N, 0.f);
  std::vector<double> ia(18 * (size_t)N);
  std::vector<int> row_sys(N);
  int fast = 1, lofree = 1;
  for (int s = 0; s < n_systems; ++s) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = off[s]; i < off[s + 1]; ++i)
      for (int c = 0; c < 3; ++c) {
        const double v = pos[3 * (size_t)i + c];
        lo[c] = std::min(lo[c], v);
        hi[c] = std::max(hi[c], v);
      }
    double ctr[3], ext2 = 0.0;
    for (int c = 0; c < 3; ++c) {
      ctr[c] = 0.5 * (lo[c] + hi[c]);
      ext2 += (hi[c] - lo[c]) * (hi[c] - lo[c]);
    }
    if (!(k[s] * std::sqrt(ext2) < 3.0)) fast = 0;
    for (int i = off[s]; i < off[s + 1]; ++i) {
      row_sys[i] = s;
      for (int c = 0; c < 3; ++c) {
        const double v = pos[3 * (size_t)i + c];
        p4[4 * (size_t)i + c] = v;
        const double d = v - ctr[c];
        const float h = (float)d;
        const float l = (float)(d - (double)h);
        h4[4 * (size_t)i + c] = h;
        l4[4 * (size_t)i + c] = l;
        if (l != 0.f) lofree = 0;
      }
    }
  }
  for (int i = 0; i < N; ++i)
    for (int e = 0; e < 9; ++e) {
      ia[2 * ((size_t)e * N + i)] = inv_alpha[18 * (size_t)i + 2 * e];
      ia[2 * ((size_t)e * N + i) + 1] = inv_alpha[18 * (size_t)i + 2 * e + 1];
    }
  lum_status s = LUM_OK;
#define LUM_B_TRY(expr)        \
  do {                         \
    s = (expr);                \
    if (s != LUM_OK) return fail(s); \
  } while (0)
#define LUM_B_UP(buf, src, bytes)                                                           \
  do {                                                                                      \
    LUM_B_TRY((buf).alloc(bytes));                                                          \
    ce = cudaMemcpyAsync((buf).p, (src), (bytes), cudaMemcpyHostToDevice, st);              \
    if (ce != cudaSuccess) return fail(cuda_status(ce, "batch upload", __FILE__, __LINE__)); \
  } while (0)
  LUM_B_UP(B->d_off, off.data(), sizeof(int) * off.size());
  LUM_B_UP(B->d_row_sys, row_sys.data(), sizeof(int) * (size_t)N);
  LUM_B_UP(B->d_k, k, sizeof(double) * (size_t)n_systems);
  LUM_B_UP(B->d_cell, cell, sizeof(double) * (size_t)n_systems);
  LUM_B_UP(B->pos64, p4.data(), sizeof(double) * p4.size());
  LUM_B_UP(B->hi, h4.data(), sizeof(float) * h4.size());
  LUM_B_UP(B->lo, l4.data(), sizeof(float) * l4.size());
  LUM_B_UP(B->inv_alpha, ia.data(), sizeof(double) * ia.size());
  BatchGeom& g = B->g;
  g.K = n_systems;
  g.N = N;
  g.fast = fast;
  g.lofree = lofree;
  {  // FP32 pair-kernel build (CTAs per SM): 4 unless LUMINA_BATCH_MINB=6.  On the
     // 256-cluster batch the spill-free 4-CTA build is 3.6 % faster.
    const char* e = std::getenv("LUMINA_BATCH_MINB");
    g.minb32 = (e && std::atoi(e) == 6) ? 6 : 4;
  }
  g.sys_off = B->d_off.as<int>();
  g.row_sys = B->d_row_sys.as<int>();
  g.sys_k = B->d_k.as<double>();
  g.sys_cell = B->d_cell.as<double>();
  g.pos64 = B->pos64.as<double4>();
  g.hi = B->hi.as<float4>();
  g.lo = B->lo.as<float4>();
  g.inv_alpha = B->inv_alpha.as<double2>();
  LUM_B_TRY(batch_near_fcd(g, use_fcd, B->near_j, B->fcd64, B->fcd32, st));
  int sms = ctx->sms > 0 ? ctx->sms : 148;
  std::vector<int> ns32, ch32, ns64, ch64;
  LUM_B_TRY(batch_queue(LUM_FP32, off, sms * batch_occupancy(g, LUM_FP32), B->q32, ns32, ch32, st));
  LUM_B_TRY(batch_queue(LUM_FP64, off, sms * batch_occupancy(g, LUM_FP64), B->q64, ns64, ch64, st));
  LUM_B_UP(B->d_ns32, ns32.data(), sizeof(int) * ns32.size());
  LUM_B_UP(B->d_ch32, ch32.data(), sizeof(int) * ch32.size());
  LUM_B_UP(B->d_ns64, ns64.data(), sizeof(int) * ns64.size());
  LUM_B_UP(B->d_ch64, ch64.data(), sizeof(int) * ch64.size());
  g.sys_ns32 = B->d_ns32.as<int>();
  g.sys_ns64 = B->d_ns64.as<int>();
  g.sys_chunk32 = B->d_ch32.as<int>();
  g.sys_chunk64 = B->d_ch64.as<int>();
  g.nparts32 = *std::max_element(ns32.begin(), ns32.end());
  g.nparts64 = *std::max_element(ns64.begin(), ns64.end());
  // The symmetric FP32 scheme (each unordered pair once, per-system
  // superblock pairs): its work list, and the choice between it and the split
  // kernel by timing one FP32 application of each (best of three after a warm
  // launch).  LUMINA_BATCH_SYM=0 keeps the split kernel, =v forces build v.
  std::vector<int> nb;
  int sym_occ = 1;
  for (int v = 1; v <= batch_sym_variants(); ++v) sym_occ = std::max(sym_occ, batch_sym_occupancy(g, v));
  LUM_B_TRY(batch_queue_sym(off, sms * sym_occ, B->qsym, nb, st));
  LUM_B_UP(B->d_nb, nb.data(), sizeof(int) * nb.size());
  g.sys_nb = B->d_nb.as<int>();
  g.qsym = &B->qsym;
  const int nb_max = *std::max_element(nb.begin(), nb.end());
  const size_t pb = std::max({sizeof(float2) * (size_t)g.nparts32,
                              sizeof(double2) * (size_t)g.nparts64,
                              sizeof(float2) * (size_t)nb_max}) *
                    3 * (size_t)N;
  LUM_B_TRY(B->part.alloc(pb));
  LUM_B_TRY(batch_choose_scheme(B, st));
  B->sym_min_items = 4 * sms * sym_occ;  // four items per CTA slot of the persistent grid
  if (const char* e = std::getenv("LUMINA_BATCH_SYM_MIN_ITEMS")) B->sym_min_items = std::atoi(e);
#undef LUM_B_UP
#undef LUM_B_TRY
  ce = cudaStreamSynchronize(st);
  if (ce != cudaSuccess) return fail(cuda_status(ce, "batch setup", __FILE__, __LINE__));
  *out = B;
  return LUM_OK;
}

int lum_batch_create_rhs(lum_session* s, int nrhs, lum_batch** out) {
  if (bad_arg(s, "session") || bad_arg(out, "out")) return LUM_ERR_INVALID;
  *out = nullptr;
  if (nrhs <= 0) {
    set_error("a right-hand-side batch needs at least one vector");
    return LUM_ERR_INVALID;
  }
  const int n = s->n_dipoles;
  if ((long long)n * nrhs > 50000000LL) {
    set_error("batch too large");
    return LUM_ERR_INVALID;
  }
  int ept = 0, clz = 0;
  for (int e : {4, 8, 16, 32}) {
    const int c = (3 * n + kBT * e - 1) / (kBT * e);
    if (c <= kMaxCluster) {
      ept = e;
      clz = c;
      break;
    }
  }
  if (!ept) {
    set_error("system of %d dipoles exceeds the batched solver's limit of %d per system", n,
              kMaxCluster * kBT * 32 / 3);
    return LUM_ERR_INVALID;
  }
  lum_batch* B = new (std::nothrow) lum_batch();
  if (!B) return LUM_ERR_OOM;
  B->ctx = s->ctx;
  B->K = nrhs;
  B->N = n * nrhs;
  B->ept = ept;
  B->cl = clz;
  B->src = s;
  B->stream = s->stream;  // the session's operator runs on its own stream
  B->own_stream = false;
  B->use_graph = 0;       // the operator may size its workspaces on first use
  B->off.resize(nrhs + 1);
  for (int r = 0; r <= nrhs; ++r) B->off[r] = r * n;
  cudaSetDevice(s->ctx->device);
  lum_status st = B->d_off.alloc(sizeof(int) * B->off.size());
  if (st == LUM_OK) {
    cudaError_t e = cudaMemcpyAsync(B->d_off.p, B->off.data(), sizeof(int) * B->off.size(),
                                    cudaMemcpyHostToDevice, B->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(B->stream);
    if (e != cudaSuccess) st = cuda_status(e, "rhs batch setup", __FILE__, __LINE__);
  }
  if (st != LUM_OK) {
    lum_batch_destroy(B);
    return st;
  }
  *out = B;
  return LUM_OK;
}

int lum_batch_destroy(lum_batch* B) {
  if (!B) return LUM_OK;
  if (B->ctx) cudaSetDevice(B->ctx->device);
  if (B->stream) cudaStreamSynchronize(B->stream);
  cudaStream_t st = B->stream;
  const bool own = B->own_stream;
  delete B;
  if (own && st) cudaStreamDestroy(st);
  return LUM_OK;
}

int lum_batch_set_stream(lum_batch* B, void* stream) {
  if (bad_arg(B, "batch")) return LUM_ERR_INVALID;
  if (B->src) {  // a right-hand-side batch follows its session's stream
    LUM_TRY((lum_status)lum_session_set_stream(B->src, stream));
    B->stream = B->src->stream;
    return LUM_OK;
  }
  cudaSetDevice(B->ctx->device);
  cudaStreamSynchronize(B->stream);
  if (stream) {
    if (B->own_stream && B->stream) cudaStreamDestroy(B->stream);
    B->stream = (cudaStream_t)stream;
    B->own_stream = false;
  } else if (!B->own_stream) {
    LUM_TRY_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
    B->own_stream = true;
  }
  // graphs were captured on the old stream's launches: they remain valid
  // (a graph is not bound to a stream)
  return LUM_OK;
}

int lum_batch_info(lum_batch* B, int* n_systems, int* n_dipoles, int* ell_width, int* cluster,
                   int* elems_per_thread, int* items32, int* grid32, int* items64, int* grid64) {
  if (bad_arg(B, "batch")) return LUM_ERR_INVALID;
  if (n_systems) *n_systems = B->K;
  if (n_dipoles) *n_dipoles = B->N;
  if (ell_width) *ell_width = B->g.ell_w;
  if (cluster) *cluster = B->cl;
  if (elems_per_thread) *elems_per_thread = B->ept;
  const BatchQueue& q32 = B->g.sym32 ? B->qsym : B->q32;
  if (items32) *items32 = q32.nitems;
  if (grid32) *grid32 = q32.grid;
  if (items64) *items64 = B->q64.nitems;
  if (grid64) *grid64 = B->q64.grid;
  return LUM_OK;
}

int lum_batch_kernel_config(lum_batch* B, char* buf, size_t len) {
  if (bad_arg(B, "batch") || bad_arg(buf, "buf") || len == 0) return LUM_ERR_INVALID;
  const BatchGeom& g = B->g;
  snprintf(buf, len, "kind=%s fp32_scheme=%s sym32=%d items32=%d grid32=%d items64=%d grid64=%d "
           "minb32=%d lofree=%d fast_trig=%d",
           B->src ? "rhs" : "clusters", g.sym32 ? "symmetric" : "split",
           g.sym32, g.sym32 ? B->qsym.nitems : B->q32.nitems,
           g.sym32 ? B->qsym.grid : B->q32.grid, B->q64.nitems, B->q64.grid, g.minb32, g.lofree,
           g.fast);
  if (g.sym32) {
    const size_t used = strlen(buf);
    if (used + 1 < len)
      snprintf(buf + used, len - used, " sym_variant=%s sym_min_items=%d split_items32=%d",
               batch_sym_name(g.sym32), B->sym_min_items, B->q32.nitems);
  }
  return LUM_OK;
}

int lum_batch_matvec_device(lum_batch* B, int precision, const void* x_dev, void* y_dev) {
  if (bad_arg(B, "batch") || bad_arg(x_dev, "x") || bad_arg(y_dev, "y")) return LUM_ERR_INVALID;
  if (precision != LUM_FP32 && precision != LUM_FP64) {
    set_error("invalid precision %d", precision);
    return LUM_ERR_INVALID;
  }
  cudaSetDevice(B->ctx->device);
  if (B->src)
    return rhs_apply(B, precision, static_cast<const double2*>(x_dev),
                     static_cast<double2*>(y_dev));
  return batch_apply(B->g, precision, static_cast<const double2*>(x_dev),
                     static_cast<double2*>(y_dev), B->part.p,
                     precision == LUM_FP32 ? B->q32 : B->q64, nullptr, 0, B->stream);
}

int lum_batch_matvec(lum_batch* B, int precision, const double* x, double* y) {
  if (bad_arg(B, "batch") || bad_arg(x, "x") || bad_arg(y, "y")) return LUM_ERR_INVALID;
  cudaSetDevice(B->ctx->device);
  const size_t bytes = sizeof(double2) * 3 * (size_t)B->N;
  if (!B->xin.p) {
    LUM_TRY(B->xin.alloc(bytes));
    LUM_TRY(B->yout.alloc(bytes));
  }
  LUM_TRY_CUDA(cudaMemcpyAsync(B->xin.p, x, bytes, cudaMemcpyHostToDevice, B->stream));
  LUM_TRY((lum_status)lum_batch_matvec_device(B, precision, B->xin.p, B->yout.p));
  LUM_TRY_CUDA(cudaMemcpyAsync(y, B->yout.p, bytes, cudaMemcpyDeviceToHost, B->stream));
  LUM_TRY_CUDA(cudaStreamSynchronize(B->stream));
  if (B->src && B->src->kind == 1) return lum::cgemm_status(B->src->cached, B->stream);
  return LUM_OK;
}

int lum_batch_solve_device(lum_batch* B, const void* b_dev, void* x_dev, double tol, int max_iter,
                           int restart, int mode, lum_solve_info* info) {
  if (bad_arg(B, "batch") || bad_arg(b_dev, "b") || bad_arg(x_dev, "x")) return LUM_ERR_INVALID;
  if (mode != LUM_SOLVE_FP64 && mode != LUM_SOLVE_FP32_REFINE) {
    set_error("invalid solve mode %d", mode);
    return LUM_ERR_INVALID;
  }
  if (!(tol > 0.0) || !std::isfinite(tol)) {
    set_error("invalid tolerance");
    return LUM_ERR_INVALID;
  }
  auto t0 = std::chrono::steady_clock::now();
  cudaSetDevice(B->ctx->device);
  cudaStream_t st = B->stream;
  if (restart <= 0) restart = 30;
  // the graph runs m steps per cycle; a system's own restart is min(m, 3N_s)
  int max_len = 0;
  for (int s = 0; s < B->K; ++s) max_len = std::max(max_len, 3 * (B->off[s + 1] - B->off[s]));
  const int m = std::min(std::min(restart, max_len), kBM);
  LUM_TRY(batch_workspace(B, m));
  if (B->m != m) {
    // a smaller restart than the workspace was sized for: graphs depend on m
    B->m = m;
  }
  const size_t bytes = sizeof(double2) * 3 * (size_t)B->N;
  LUM_TRY_CUDA(cudaMemcpyAsync(B->bs.p, b_dev, bytes, cudaMemcpyDeviceToDevice, st));
  BatchCtl c{};
  c.tol = tol;
  c.inner_rel = 1e-5;
  c.max_iter = max_iter;
  c.m = m;
  c.refine = (mode == LUM_SOLVE_FP32_REFINE);
  c.active = 0;
  LUM_TRY_CUDA(cudaMemcpyAsync(B->ctl.p, &c, sizeof(c), cudaMemcpyHostToDevice, st));
  LUM_TRY(dispatch_ept<RunInit>(B->ept, B, B->bs.as<const double2>()));
  // every active cycle advances each active system by >= 1 step
  const long max_cycles = (long)std::max(max_iter, 0) + 1;
  // a tensor-core product whose pipeline wait gave up leaves tiles of its
  // result unwritten: the cycle's status is read after every cycle
  const bool tensor = B->src && B->src->kind == 1 && !B->src->cached.packed &&
                      B->src->cached.precision == LUM_FP32 && mode == LUM_SOLVE_FP32_REFINE;
  // symmetric items of the systems still active (all of them at the start)
  long live = 0;
  if (!B->src)
    for (int s = 0; s < B->K; ++s) {
      const long nb = (B->off[s + 1] - B->off[s] + kBatchSymRows - 1) / kBatchSymRows;
      live += nb * (nb + 1) / 2;
    }
  if (B->use_graph && mode == LUM_SOLVE_FP32_REFINE && B->g.sym32) {
    // both FP32 cycle graphs before the first cycle: none is captured mid-solve
    LUM_TRY(batch_graph(B, mode, B->g.sym32));
    LUM_TRY(batch_graph(B, mode, 0));
  }
  for (long cyc = 0; cyc < max_cycles; ++cyc) {
    const int sym = (mode == LUM_SOLVE_FP32_REFINE && B->g.sym32 && live >= B->sym_min_items)
                        ? B->g.sym32
                        : 0;
    LUM_TRY(batch_run_cycle(B, mode, sym));
    LUM_TRY_CUDA(cudaStreamSynchronize(st));
    if (tensor) LUM_TRY(lum::cgemm_status(B->src->cached, st));
    if (B->h_active[0] == 0) break;
    live = B->h_active[1];
  }
  LUM_TRY_CUDA(cudaMemcpyAsync(x_dev, B->xs.p, bytes, cudaMemcpyDeviceToDevice, st));
  LUM_TRY_CUDA(cudaMemcpyAsync(B->h_state, B->state.p, sizeof(BatchSysState) * (size_t)B->K,
                               cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaMemcpyAsync(B->h_flags, B->flags.p, sizeof(BatchFlags) * (size_t)B->K,
                               cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  int n_bad = 0, n_fail = 0, first_bad = -1, first_fail = -1;
  for (int s = 0; s < B->K; ++s) {
    const BatchSysState& S = B->h_state[s];
    const BatchFlags& F = B->h_flags[s];
    if (F.bad) {
      if (first_bad < 0) first_bad = s;
      ++n_bad;
    } else if (!S.converged) {
      if (first_fail < 0) first_fail = s;
      ++n_fail;
    }
    if (info) {
      lum_solve_info& o = info[s];
      o = lum_solve_info{};
      o.iterations = S.total;
      o.restarts = S.restarts;
      o.converged = S.converged;
      o.rel_residual = S.rhs_norm > 0.0 ? S.beta / S.rhs_norm : 0.0;
      o.matvecs_fp64 = S.mv_fp64 + (mode == LUM_SOLVE_FP64 ? S.mv_arnoldi : 0);
      o.matvecs_fp32 = (mode == LUM_SOLVE_FP32_REFINE) ? S.mv_arnoldi : 0;
      o.matvecs_reference = S.total + 2 * S.restarts + (S.restarts == 0 ? 1 : 0);
      o.seconds = secs;
    }
  }
  if (n_bad) {
    set_error("GMRES breakdown (non-finite residual) in %d system(s), first %d", n_bad, first_bad);
    return LUM_ERR_DEVICE;
  }
  if (n_fail) {
    set_error("Solver failed to converge after %d iterations in %d system(s), first %d "
              "(residual: %.2e)", max_iter, n_fail, first_fail,
              B->h_state[first_fail].beta / B->h_state[first_fail].rhs_norm);
    return LUM_ERR_NOT_CONVERGED;
  }
  return LUM_OK;
}

int lum_batch_solve(lum_batch* B, const double* b, double tol, int max_iter, int restart, int mode,
                    double* x, lum_solve_info* info) {
  if (bad_arg(B, "batch") || bad_arg(b, "b") || bad_arg(x, "x")) return LUM_ERR_INVALID;
  cudaSetDevice(B->ctx->device);
  const size_t bytes = sizeof(double2) * 3 * (size_t)B->N;
  if (!B->xin.p) {
    LUM_TRY(B->xin.alloc(bytes));
    LUM_TRY(B->yout.alloc(bytes));
  }
  LUM_TRY_CUDA(cudaMemcpyAsync(B->xin.p, b, bytes, cudaMemcpyHostToDevice, B->stream));
  const int st = lum_batch_solve_device(B, B->xin.p, B->yout.p, tol, max_iter, restart, mode, info);
  if (st != LUM_OK && st != LUM_ERR_NOT_CONVERGED) return st;
  LUM_TRY_CUDA(cudaMemcpyAsync(x, B->yout.p, bytes, cudaMemcpyDeviceToHost, B->stream));
  LUM_TRY_CUDA(cudaStreamSynchronize(B->stream));
  return st;
}
