// noalloc.cu -- a matrix-free matvec for callers that cannot allocate device
// memory.
//
// Every other entry point of this library owns device buffers (sessions,
// Krylov workspaces, scratch).  Some callers cannot let a library call
// cudaMalloc: their GPU memory is already claimed by another allocator (a
// framework's caching pool, or an arena reserved up front so a large cached
// matrix fits in HBM), or they run in code where an allocation, with the
// device-wide synchronisation cudaFree can imply, is not allowed.  For them,
// lum_matvec_onthefly_noalloc computes the FP64 point-dipole product
//
//   y_i = alpha_i^-1 x_i - sum_{j != i} G(r_i - r_j) x_j
//
// from caller-owned inputs and output only.  It is the same computation as the
// FP64 on-the-fly session with use_fcd = 0 (otf_pairs_f64 + otf_epilogue in
// otf.cu), and it keeps its only scratch -- the per-split partial sums -- in
// the file-scope device array below, so it allocates nothing per call.
//
// Limits and sharing: the array holds 2^19 double2 (8 MiB); a call accepts at
// most 174,762 dipoles (3N entries must fit one split) and uses fewer splits
// when N is large.  Every GPU that loads this library holds the array until
// the process exits.  All calls share it and it keeps the last call's
// contents; every entry a call reads was written earlier in the same call,
// so nothing needs clearing.  Calls whose kernels overlap on a GPU (two
// streams, two threads) race on the array: serialise them.
#include "lumina_internal.cuh"

#include <cmath>
#include <mutex>

namespace lum {

constexpr int kNaBlock = 128;
constexpr size_t kNoAllocEntries = size_t(1) << 19;  // double2 entries (8 MiB)

static __device__ __align__(256) double2 g_noalloc_scratch[kNoAllocEntries];

// Pair pass: positions read as N x 3 doubles (the ABI layout), partial sums
// of +G x per split into partial[split][3N].
__global__ void __launch_bounds__(kNaBlock)
noalloc_pairs_f64(int n, const double* __restrict__ pos, const double2* __restrict__ x, double k,
                  double inv_k, double s0, int chunk, double2* __restrict__ partial) {
  __shared__ double sP[3 * kNaBlock];
  __shared__ double2 sX[3 * kNaBlock];
  const int tid = threadIdx.x;
  const int i = blockIdx.x * kNaBlock + tid;
  const int ic = min(i, n - 1);
  const double rx = pos[3 * ic], ry = pos[3 * ic + 1], rz = pos[3 * ic + 2];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const int j_begin = blockIdx.y * chunk;
  const int j_end = min(n, j_begin + chunk);
  for (int jt = j_begin; jt < j_end; jt += kNaBlock) {
    const int cnt = min(kNaBlock, j_end - jt);
    __syncthreads();
    if (tid < cnt) {
      const int j = jt + tid;
      sP[3 * tid] = pos[3 * j];
      sP[3 * tid + 1] = pos[3 * j + 1];
      sP[3 * tid + 2] = pos[3 * j + 2];
      sX[3 * tid] = x[3 * j];
      sX[3 * tid + 1] = x[3 * j + 1];
      sX[3 * tid + 2] = x[3 * j + 2];
    }
    __syncthreads();
    for (int jj = 0; jj < cnt; ++jj) {
      const double2 xa = sX[3 * jj], xb = sX[3 * jj + 1], xc = sX[3 * jj + 2];
      double dx = rx - sP[3 * jj], dy = ry - sP[3 * jj + 1], dz = rz - sP[3 * jj + 2];
      double r2 = dx * dx + dy * dy + dz * dz;
      const bool self = (jt + jj == i);
      if (self) r2 = 1.0;
      double ir = rsqrt(r2);
      double Rr = r2 * ir;
      double u = ir * inv_k;
      double u2 = u * u;
      double sn, cs;
      sincos(k * Rr, &sn, &cs);
      double su = self ? 0.0 : s0 * u;
      double pr = su * cs, pi = su * sn;
      double ar = 1.0 - u2;
      double Ar = pr * ar - pi * u, Ai = pr * u + pi * ar;
      double br = 3.0 * u2 - 1.0, bi = -3.0 * u;
      double ir2 = ir * ir;
      double Br = (pr * br - pi * bi) * ir2, Bi = (pr * bi + pi * br) * ir2;
      double dxr = dx * xa.x + dy * xb.x + dz * xc.x;
      double dxi = dx * xa.y + dy * xb.y + dz * xc.y;
      double tr = Br * dxr - Bi * dxi, ti = Br * dxi + Bi * dxr;
      acc[0] += Ar * xa.x - Ai * xa.y + tr * dx;
      acc[1] += Ar * xa.y + Ai * xa.x + ti * dx;
      acc[2] += Ar * xb.x - Ai * xb.y + tr * dy;
      acc[3] += Ar * xb.y + Ai * xb.x + ti * dy;
      acc[4] += Ar * xc.x - Ai * xc.y + tr * dz;
      acc[5] += Ar * xc.y + Ai * xc.x + ti * dz;
    }
  }
  if (i < n) {
    double2* out = partial + (size_t)blockIdx.y * (3 * (size_t)n);
    out[3 * i + 0] = make_double2(acc[0], acc[1]);
    out[3 * i + 1] = make_double2(acc[2], acc[3]);
    out[3 * i + 2] = make_double2(acc[4], acc[5]);
  }
}

// y = alpha^-1 x (alpha^-1 as N x 9 complex, row-major per dipole) minus the
// splits summed in a fixed order.
__global__ void __launch_bounds__(256)
noalloc_epilogue(int n, const double2* __restrict__ x, const double2* __restrict__ inv_alpha,
                 const double2* __restrict__ partial, int nparts, double2* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double2 xi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
  const size_t stride = 3 * (size_t)n;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double sr = 0.0, si = 0.0;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const double2 m = inv_alpha[9 * (size_t)i + 3 * a + b];
      sr += m.x * xi[b].x - m.y * xi[b].y;
      si += m.x * xi[b].y + m.y * xi[b].x;
    }
    double gr = 0.0, gi = 0.0;
    for (int s = 0; s < nparts; ++s) {
      const double2 p = partial[s * stride + 3 * i + a];
      gr += p.x;
      gi += p.y;
    }
    y[3 * i + a] = make_double2(sr - gr, si - gi);
  }
}

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
// Per device: the resolved address and the context it belongs to.  A device
// reset (cudaDeviceReset) or a new primary context reloads this library's
// device code, and the array may then sit at another address, so the address
// is looked up again whenever the current context is not the recorded one.
double2* g_noalloc_ptr[kMaxDevices] = {};
void* g_noalloc_ctx[kMaxDevices] = {};

using CtxGetCurrentFn = int (*)(void**);  // CUresult cuCtxGetCurrent(CUcontext*)

CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrentFn>(p);
  }
  return fn;
}
}  // namespace

}  // namespace lum

using namespace lum;

extern "C" int lum_matvec_onthefly_noalloc(int n_dipoles, const double* pos,
                                           const double* inv_alpha, double k, const double* x,
                                           double* y, void* stream) {
  const size_t max_dipoles = kNoAllocEntries / 3;
  if (n_dipoles <= 0 || (size_t)n_dipoles > max_dipoles) {
    set_error("lum_matvec_onthefly_noalloc: n_dipoles = %d is outside 1..%zu (the fixed "
              "no-alloc scratch holds %zu complex entries)", n_dipoles, max_dipoles,
              kNoAllocEntries);
    return LUM_ERR_INVALID;
  }
  if (!pos || !inv_alpha || !x || !y) {
    set_error("lum_matvec_onthefly_noalloc: pos, inv_alpha, x and y must be device pointers");
    return LUM_ERR_INVALID;
  }
  if (!(k > 0.0) || !std::isfinite(k)) {
    set_error("lum_matvec_onthefly_noalloc: wavenumber must be positive and finite (got %g)", k);
    return LUM_ERR_INVALID;
  }
  int dev = 0;
  LUM_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("lum_matvec_onthefly_noalloc: device %d out of range", dev);
    return LUM_ERR_INVALID;
  }
  double2* scratch = nullptr;
  {
    // First call on a device (or in a new context of it): resolve the device
    // address of the file-scope array (the host-side symbol is only a
    // stand-in) with that device current.
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    void* ctx = nullptr;
    if (CtxGetCurrentFn get = ctx_get_current()) get(&ctx);
    if (!g_noalloc_ptr[dev] || ctx != g_noalloc_ctx[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        return cuda_status(e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                           "cudaGetSymbolAddress(no-alloc scratch)", __FILE__, __LINE__);
      }
      g_noalloc_ptr[dev] = static_cast<double2*>(p);
      if (!ctx && ctx_get_current()) ctx_get_current()(&ctx);  // created by the lookup
      g_noalloc_ctx[dev] = ctx;
    }
    scratch = g_noalloc_ptr[dev];
  }
  int sms = 148;
  LUM_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int n = n_dipoles;
  const int ntiles = (n + kNaBlock - 1) / kNaBlock;
  const int fit = (int)std::min<size_t>(64, kNoAllocEntries / (3 * (size_t)n));
  int nsplit = (4 * sms + ntiles - 1) / ntiles;
  nsplit = std::max(1, std::min(nsplit, std::min(fit, ntiles)));
  const int chunk = ((ntiles + nsplit - 1) / nsplit) * kNaBlock;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const double s0 = k * k * k / (4.0 * kPi);
  noalloc_pairs_f64<<<dim3(ntiles, nsplit), kNaBlock, 0, st>>>(
      n, pos, reinterpret_cast<const double2*>(x), k, 1.0 / k, s0, chunk, scratch);
  LUM_CHECK_LAUNCH();
  noalloc_epilogue<<<(n + 255) / 256, 256, 0, st>>>(
      n, reinterpret_cast<const double2*>(x), reinterpret_cast<const double2*>(inv_alpha),
      scratch, nsplit, reinterpret_cast<double2*>(y));
  LUM_CHECK_LAUNCH();
  return LUM_OK;
}
