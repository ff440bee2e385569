// capi.cu -- extern "C" surface of liblumina_b200 (declared in
// include/lumina_b200.h).  Every entry point validates its arguments,
// converts CUDA failures into lum_status codes with a thread-local message
// (lum_last_error) and never throws or aborts across the ABI.
#include "lumina_internal.cuh"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstring>
#include <new>

namespace lum {

std::atomic<uint64_t> g_launches{0};
static thread_local std::string t_last_error = "";
static thread_local size_t t_oom_requested = 0, t_oom_available = 0;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  t_last_error = buf;
}

lum_status cuda_status(cudaError_t e, const char* what, const char* file, int line) {
  set_error("%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();  // clear the sticky-free allocation error
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    t_oom_requested = 0;
    t_oom_available = fr;
    return LUM_ERR_OOM;
  }
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return LUM_ERR_UNAVAILABLE;
  return LUM_ERR_DEVICE;
}

lum_status DevBuf::alloc(size_t nbytes) {
  release();
  if (nbytes == 0) return LUM_OK;
  cudaError_t e = cudaMalloc(&p, nbytes);
  if (e != cudaSuccess) {
    p = nullptr;
    size_t fr = 0, tot = 0;
    cudaGetLastError();
    cudaMemGetInfo(&fr, &tot);
    set_error("Out of memory: requested %zu bytes, available %zu", nbytes, fr);
    t_oom_requested = nbytes;
    t_oom_available = fr;
    return LUM_ERR_OOM;
  }
  bytes = nbytes;
  return LUM_OK;
}

// --- FMA-chain microbenchmark (roofline denominator for CUDA-core kernels) --
template <typename T>
__global__ void fma_chain(T* out, int iters, T a, T b) {
  T x0 = (T)threadIdx.x * (T)1e-7, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
  T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
      x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
    }
  }
  T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == (T)-12345.678) out[0] = s;  // keeps the chain live; never true
}

// Packed FP32 variant: eight float2 chains of f32x2 FMAs (the instruction the
// FP32 pair kernels are built from).
__global__ void fma2_chain(float* out, int iters, float a, float b) {
  const float t = (float)threadIdx.x * 1e-7f;
  float2 x0 = make_float2(t, t + 0.5f), x1 = make_float2(t + 1.f, t + 1.5f),
         x2 = make_float2(t + 2.f, t + 2.5f), x3 = make_float2(t + 3.f, t + 3.5f),
         x4 = make_float2(t + 4.f, t + 4.5f), x5 = make_float2(t + 5.f, t + 5.5f),
         x6 = make_float2(t + 6.f, t + 6.5f), x7 = make_float2(t + 7.f, t + 7.5f);
  const float2 A = make_float2(a, a), B = make_float2(b, b);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x0 = __ffma2_rn(x0, A, B); x1 = __ffma2_rn(x1, A, B); x2 = __ffma2_rn(x2, A, B);
      x3 = __ffma2_rn(x3, A, B); x4 = __ffma2_rn(x4, A, B); x5 = __ffma2_rn(x5, A, B);
      x6 = __ffma2_rn(x6, A, B); x7 = __ffma2_rn(x7, A, B);
    }
  }
  const float s = x0.x + x1.x + x2.x + x3.x + x4.x + x5.x + x6.x + x7.x + x0.y + x1.y + x2.y +
                  x3.y + x4.y + x5.y + x6.y + x7.y;
  if (s == -12345.678f) out[0] = s;  // keeps the chains live; never true
}

// --- L2 read microbenchmark (roofline denominator for the table gathers) --
// Every thread streams 16-byte loads that bypass L1 (ld.global.cg) over a
// buffer far smaller than L2, so after the first pass every load hits L2.
__global__ void l2_read(const float4* __restrict__ buf, size_t n4, int reps,
                        float* __restrict__ out) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  float acc = 0.f;
  for (int r = 0; r < reps; ++r)
    for (size_t i = (t0 + (size_t)r * 4099) % n4, c = 0; c < n4; c += stride) {
      const float4 v = __ldcg(buf + i);
      acc += v.x + v.y + v.z + v.w;
      i += stride;
      if (i >= n4) i -= n4;
    }
  if (acc == -12345.678f) out[0] = acc;  // keeps the loads live; never true
}

}  // namespace lum

using namespace lum;

lum_status lum_gmres_device(lum_session* s, const double2* b, double2* x, double tol,
                            int max_iter, int restart, int mode, lum_solve_info* info,
                            cudaStream_t st);

lum_status lum_session::apply(int precision, const double2* x, double2* y, const int* skip) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (profile) {
    if (ev_used + 1 > ev_pool.size()) {
      for (int q = 0; q < 64; ++q) {
        EvRec r;
        LUM_TRY_CUDA(cudaEventCreate(&r.a));
        LUM_TRY_CUDA(cudaEventCreate(&r.b));
        ev_pool.push_back(r);
      }
    }
    EvRec& r = ev_pool[ev_used++];
    r.precision = precision;
    e0 = r.a;
    e1 = r.b;
  }
  if (kind == 0) {
    LUM_TRY(otf.apply(precision, x, y, stream, e0, e1, skip));
    return otf.somm_apply(precision, x, y, stream, skip);
  }
  if (kind == 2) return fft.apply(precision, x, y, stream, e0, e1, skip);
  // cached session
  if (otf.has_somm && otf.somm_stale) return otf.somm_apply(precision, x, y, stream, skip);
  if (precision == LUM_FP64 && cached.precision == LUM_FP32 && otf.inv_alpha.p) {
    LUM_TRY(otf.apply(LUM_FP64, x, y, stream, nullptr, nullptr, skip));
    return otf.somm_apply(LUM_FP64, x, y, stream, skip);
  }
  if (e0) cudaEventRecord(e0, stream);
  LUM_TRY(cached.apply(x, y, stream, skip));
  if (e1) cudaEventRecord(e1, stream);
  return LUM_OK;
}

// Two vectors per application; profiled under precision + 2 (the two-vector
// kernels), so the single-vector records stay comparable.
lum_status lum_session::apply2(int precision, const double2* x, const double2* x2, double2* y,
                               double2* y2, const int* skip, const int* skip2) {
  if (kind != 0) {
    LUM_TRY(apply(precision, x, y, skip));
    return apply(precision, x2, y2, skip2);
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (profile) {
    if (ev_used + 1 > ev_pool.size()) {
      for (int q = 0; q < 64; ++q) {
        EvRec r;
        LUM_TRY_CUDA(cudaEventCreate(&r.a));
        LUM_TRY_CUDA(cudaEventCreate(&r.b));
        ev_pool.push_back(r);
      }
    }
    EvRec& r = ev_pool[ev_used++];
    r.precision = precision + 2;
    e0 = r.a;
    e1 = r.b;
  }
  LUM_TRY(otf.apply2(precision, x, x2, y, y2, stream, e0, e1, skip, skip2));
  LUM_TRY(otf.somm_apply(precision, x, y, stream, skip));
  return otf.somm_apply(precision, x2, y2, stream, skip2);
}

static bool bad_ptr(const void* p, const char* what) {
  if (!p) {
    set_error("%s must not be NULL", what);
    return true;
  }
  return false;
}

extern "C" {

const char* lum_last_error(void) { return t_last_error.c_str(); }

int lum_last_oom(size_t* requested, size_t* available) {
  if (requested) *requested = t_oom_requested;
  if (available) *available = t_oom_available;
  return LUM_OK;
}
uint64_t lum_launch_count(void) { return g_launches.load(); }

int lum_ctx_create(int device, lum_ctx** out) {
  if (bad_ptr(out, "out")) return LUM_ERR_INVALID;
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    set_error("No CUDA device found (%s)", cudaGetErrorString(e));
    return LUM_ERR_UNAVAILABLE;
  }
  if (device < 0 || device >= count) {
    set_error("device %d out of range (count %d)", device, count);
    return LUM_ERR_INVALID;
  }
  cudaDeviceProp prop;
  LUM_TRY_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) {
    set_error("device %d (%s, sm_%d%d) is not an sm_100 part", device, prop.name, prop.major,
              prop.minor);
    return LUM_ERR_UNAVAILABLE;
  }
  LUM_TRY_CUDA(cudaSetDevice(device));
  lum_ctx* c = new (std::nothrow) lum_ctx();
  if (!c) return LUM_ERR_OOM;
  c->device = device;
  c->name = prop.name;
  c->mem_bytes = prop.totalGlobalMem;
  c->sms = prop.multiProcessorCount;
  *out = c;
  return LUM_OK;
}

int lum_ctx_destroy(lum_ctx* ctx) {
  delete ctx;
  return LUM_OK;
}

int lum_device_info(lum_ctx* ctx, char* name, size_t name_len, size_t* memory_bytes,
                    int* compute_units) {
  if (bad_ptr(ctx, "ctx")) return LUM_ERR_INVALID;
  if (name && name_len) {
    std::string s = "GPU (" + ctx->name + ")";
    std::strncpy(name, s.c_str(), name_len - 1);
    name[name_len - 1] = '\0';
  }
  if (memory_bytes) *memory_bytes = ctx->mem_bytes;
  if (compute_units) *compute_units = ctx->sms;
  return LUM_OK;
}

// ---- host helpers ---------------------------------------------------------
using cd = std::complex<double>;

static bool invert3(const cd m[9], cd o[9]) {  // assembly.rs:335-363
  cd a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], k = m[8];
  cd det = a * (e * k - f * h) - b * (d * k - f * g) + c * (d * h - e * g);
  if (!(std::abs(det) > 1e-30)) return false;
  cd id = 1.0 / det;
  o[0] = id * (e * k - f * h);
  o[1] = id * (c * h - b * k);
  o[2] = id * (b * f - c * e);
  o[3] = id * (f * g - d * k);
  o[4] = id * (a * k - c * g);
  o[5] = id * (c * d - a * f);
  o[6] = id * (d * h - e * g);
  o[7] = id * (b * g - a * h);
  o[8] = id * (a * e - b * d);
  return true;
}

int lum_invert_polarisability(int n, const double* alpha, double* inv_alpha) {
  if (n < 0 || (n > 0 && (bad_ptr(alpha, "alpha") || bad_ptr(inv_alpha, "inv_alpha"))))
    return LUM_ERR_INVALID;
  for (int i = 0; i < n; ++i) {
    cd m[9], o[9];
    for (int e = 0; e < 9; ++e) m[e] = cd(alpha[18 * (size_t)i + 2 * e], alpha[18 * (size_t)i + 2 * e + 1]);
    if (!invert3(m, o)) {
      set_error("Singular polarisability tensor at dipole %d", i);
      return LUM_ERR_INVALID;
    }
    for (int e = 0; e < 9; ++e) {
      inv_alpha[18 * (size_t)i + 2 * e] = o[e].real();
      inv_alpha[18 * (size_t)i + 2 * e + 1] = o[e].imag();
    }
  }
  return LUM_OK;
}

int lum_incident_field(int n, const double* pos, const double direction[3],
                       const double polarisation[3], double amplitude, double k, double* rhs) {
  if (n < 0 || bad_ptr(direction, "direction") || bad_ptr(polarisation, "polarisation"))
    return LUM_ERR_INVALID;
  if (n > 0 && (bad_ptr(pos, "pos") || bad_ptr(rhs, "rhs"))) return LUM_ERR_INVALID;
  for (int i = 0; i < n; ++i) {
    const double* p = pos + 3 * (size_t)i;
    double kdotr = k * (direction[0] * p[0] + direction[1] * p[1] + direction[2] * p[2]);
    double c = std::cos(kdotr), s = std::sin(kdotr);
    for (int q = 0; q < 3; ++q) {
      double e0 = amplitude * polarisation[q];
      rhs[2 * (3 * (size_t)i + q)] = e0 * c;
      rhs[2 * (3 * (size_t)i + q) + 1] = e0 * s;
    }
  }
  return LUM_OK;
}

int lum_cross_sections(int n, const double* pos, const double* inv_alpha, const double* moments,
                       double k, const double direction[3], const double polarisation[3],
                       double amplitude, double out[3]) {
  if (n <= 0 || bad_ptr(pos, "pos") || bad_ptr(inv_alpha, "inv_alpha") ||
      bad_ptr(moments, "moments") || bad_ptr(out, "out") || bad_ptr(direction, "direction") ||
      bad_ptr(polarisation, "polarisation"))
    return LUM_ERR_INVALID;
  const double e0_sq = amplitude * amplitude;
  double c_ext = 0.0, c_abs = 0.0;
  const double k3 = k * k * k;
  for (int i = 0; i < n; ++i) {
    const double* p = pos + 3 * (size_t)i;
    double kdotr = k * (direction[0] * p[0] + direction[1] * p[1] + direction[2] * p[2]);
    cd phase(std::cos(kdotr), std::sin(kdotr));
    cd m[3];
    for (int c = 0; c < 3; ++c)
      m[c] = cd(moments[2 * (3 * (size_t)i + c)], moments[2 * (3 * (size_t)i + c) + 1]);
    for (int c = 0; c < 3; ++c) {
      cd e = amplitude * polarisation[c] * phase;
      c_ext += (std::conj(e) * m[c]).imag();
    }
    cd acc = 0.0;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        cd ia(inv_alpha[18 * (size_t)i + 2 * (3 * a + b)], inv_alpha[18 * (size_t)i + 2 * (3 * a + b) + 1]);
        acc += m[a] * std::conj(ia) * std::conj(m[b]);
      }
    double psq = std::norm(m[0]) + std::norm(m[1]) + std::norm(m[2]);
    c_abs += acc.imag() - (2.0 / 3.0) * k3 * psq;
  }
  c_ext *= k / e0_sq;
  c_abs *= k / e0_sq;
  out[0] = c_ext;
  out[1] = c_abs;
  out[2] = std::max(c_ext - c_abs, 0.0);
  return LUM_OK;
}

// ---- sessions -------------------------------------------------------------
static lum_status new_session(lum_ctx* ctx, int kind, int dim, lum_session** out) {
  lum_session* s = new (std::nothrow) lum_session();
  if (!s) return LUM_ERR_OOM;
  s->ctx = ctx;
  s->kind = kind;
  s->dim = dim;
  s->n_dipoles = dim / 3;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete s;
    return cuda_status(e, "stream create", __FILE__, __LINE__);
  }
  *out = s;
  return LUM_OK;
}

int lum_session_destroy(lum_session* s) {
  if (!s) return LUM_OK;
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->stream);
  for (auto& r : s->ev_pool) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return LUM_OK;
}

int lum_session_set_stream(lum_session* s, void* stream) {
  if (bad_ptr(s, "session")) return LUM_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->stream);
  if (stream) {
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    s->stream = (cudaStream_t)stream;
    s->own_stream = false;
  } else if (!s->own_stream) {
    LUM_TRY_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    s->own_stream = true;
  }
  return LUM_OK;
}

int lum_session_create_cached(lum_ctx* ctx, int dim, int precision, lum_session** out) {
  if (bad_ptr(ctx, "ctx") || bad_ptr(out, "out")) return LUM_ERR_INVALID;
  *out = nullptr;
  if (dim <= 0 || (precision != LUM_FP32 && precision != LUM_FP64)) {
    set_error("invalid cached session (dim %d, precision %d)", dim, precision);
    return LUM_ERR_INVALID;
  }
  lum_session* s = nullptr;
  LUM_TRY(new_session(ctx, 1, dim, &s));
  lum_status st = s->cached.allocate(dim, precision);
  if (st != LUM_OK) {
    lum_session_destroy(s);
    return st;
  }
  *out = s;
  return LUM_OK;
}

int lum_session_upload_matrix(lum_session* s, const double* A) {
  if (bad_ptr(s, "session") || bad_ptr(A, "matrix")) return LUM_ERR_INVALID;
  if (s->kind != 1) {
    set_error("upload_matrix needs a cached session");
    return LUM_ERR_INVALID;
  }
  if (s->cached.packed) {
    set_error("upload_matrix takes dense rows; this session keeps symmetric tiles");
    return LUM_ERR_INVALID;
  }
  cudaSetDevice(s->ctx->device);
  return s->cached.upload(A, s->stream);
}

static lum_status check_physics(int n, const double* inv_alpha, double k) {
  if (bad_ptr(inv_alpha, "inv_alpha")) return LUM_ERR_INVALID;
  if (!(k > 0.0) || !std::isfinite(k)) {
    set_error("wavenumber must be positive and finite (got %g)", k);
    return LUM_ERR_INVALID;
  }
  for (size_t q = 0; q < 18 * (size_t)n; ++q)
    if (!std::isfinite(inv_alpha[q])) {
      set_error("non-finite inverse polarisability at dipole %zu", q / 18);
      return LUM_ERR_INVALID;
    }
  return LUM_OK;
}

static lum_status check_inputs(int n, const double* pos, const double* inv_alpha, double k) {
  if (n <= 0) {
    set_error("No dipoles provided");
    return LUM_ERR_INVALID;
  }
  if (bad_ptr(pos, "pos")) return LUM_ERR_INVALID;
  return check_physics(n, inv_alpha, k);
}

int lum_session_create_onthefly(lum_ctx* ctx, int n, const double* pos, const double* inv_alpha,
                                double k, int use_fcd, double cell, const lum_lattice* lattice,
                                const double k_bloch[3], const lum_substrate* substrate,
                                lum_session** out) {
  if (bad_ptr(ctx, "ctx") || bad_ptr(out, "out")) return LUM_ERR_INVALID;
  *out = nullptr;
  LUM_TRY(check_inputs(n, pos, inv_alpha, k));
  if (n > 100000000) {
    set_error("too many dipoles (%d)", n);
    return LUM_ERR_INVALID;
  }
  lum_session* s = nullptr;
  LUM_TRY(new_session(ctx, 0, 3 * n, &s));
  lum_status st = s->otf.build_geometry(pos, n, s->stream);
  if (st == LUM_OK)
    st = s->otf.set_physics(k, inv_alpha, use_fcd, cell, lattice, k_bloch, substrate, s->stream);
  if (st == LUM_OK) {
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) st = cuda_status(e, "session setup", __FILE__, __LINE__);
  }
  if (st != LUM_OK) {
    lum_session_destroy(s);
    return st;
  }
  *out = s;
  return LUM_OK;
}

int lum_session_set_wavelength(lum_session* s, double k, const double* inv_alpha,
                               const lum_substrate* substrate) {
  if (bad_ptr(s, "session")) return LUM_ERR_INVALID;
  if (s->kind == 2) {
    LUM_TRY(check_physics(s->n_dipoles, inv_alpha, k));
    if (substrate && s->fft.refl_mode == 2) {
      set_error("a Sommerfeld session takes no Fresnel substrate");
      return LUM_ERR_INVALID;
    }
    cudaSetDevice(s->ctx->device);
    LUM_TRY(s->fft.set_physics(k, inv_alpha, s->stream));
    // the reflected spectra: Fresnel rebuilt here, Sommerfeld waits for
    // lum_session_set_sommerfeld
    if (substrate) LUM_TRY(s->fft.set_reflection(1, substrate, nullptr, s->stream));
    else if (s->fft.refl_mode == 2) s->fft.refl_stale = 1;
    else if (s->fft.refl_mode == 1) LUM_TRY(s->fft.set_reflection(0, nullptr, nullptr, s->stream));
    LUM_TRY_CUDA(cudaStreamSynchronize(s->stream));
    return LUM_OK;
  }
  if (!s->otf.inv_alpha.p) {
    set_error("set_wavelength needs a geometry session");
    return LUM_ERR_INVALID;
  }
  LUM_TRY(check_physics(s->n_dipoles, inv_alpha, k));
  if (s->otf.has_somm && substrate) {
    set_error("a Sommerfeld session takes no Fresnel substrate");
    return LUM_ERR_INVALID;
  }
  if (s->kind == 1 && s->cached.packed && substrate) {
    set_error("symmetric tile storage needs a free-space system (no substrate)");
    return LUM_ERR_INVALID;
  }
  cudaSetDevice(s->ctx->device);
  LUM_TRY(s->otf.set_physics(k, inv_alpha, s->otf.use_fcd, s->otf.cell, nullptr, nullptr,
                             substrate, s->stream));
  // The Sommerfeld table (and a matrix built from it) waits for
  // lum_session_set_sommerfeld with this wavelength's substrate.
  if (s->otf.has_somm) s->otf.somm_stale = 1;
  else if (s->kind == 1) LUM_TRY(s->cached.assemble(s->otf, s->stream));
  LUM_TRY_CUDA(cudaStreamSynchronize(s->stream));
  return LUM_OK;
}

int lum_session_create_fft(lum_ctx* ctx, int n, const double* pos, const double* inv_alpha,
                           double k, int use_fcd, double cell, double spacing,
                           lum_session** out) {
  if (bad_ptr(ctx, "ctx") || bad_ptr(out, "out")) return LUM_ERR_INVALID;
  *out = nullptr;
  LUM_TRY(check_inputs(n, pos, inv_alpha, k));
  lum_session* s = nullptr;
  LUM_TRY(new_session(ctx, 2, 3 * n, &s));
  lum_status st = s->fft.build(pos, n, spacing, cell, use_fcd, s->stream);
  if (st == LUM_OK) st = s->fft.set_physics(k, inv_alpha, s->stream);
  if (st != LUM_OK) {
    lum_session_destroy(s);
    return st;
  }
  *out = s;
  return LUM_OK;
}

int lum_session_assemble(lum_ctx* ctx, int n, const double* pos, const double* inv_alpha,
                         double k, int use_fcd, double cell, const lum_lattice* lattice,
                         const double k_bloch[3], const lum_substrate* substrate, int precision,
                         lum_session** out) {
  if (bad_ptr(ctx, "ctx") || bad_ptr(out, "out")) return LUM_ERR_INVALID;
  *out = nullptr;
  LUM_TRY(check_inputs(n, pos, inv_alpha, k));
  const bool sym = (precision & LUM_STORAGE_SYMMETRIC) != 0;
  precision &= ~LUM_STORAGE_SYMMETRIC;
  if (precision != LUM_FP32 && precision != LUM_FP64) {
    set_error("invalid storage precision %d", precision);
    return LUM_ERR_INVALID;
  }
  if (sym && (lattice || substrate)) {
    set_error("symmetric tile storage needs a free-space system (no lattice sum, no "
              "substrate)");
    return LUM_ERR_INVALID;
  }
  lum_session* s = nullptr;
  LUM_TRY(new_session(ctx, 1, 3 * n, &s));
  lum_status st = s->otf.build_geometry(pos, n, s->stream);
  if (st == LUM_OK)
    st = s->otf.set_physics(k, inv_alpha, use_fcd, cell, lattice, k_bloch, substrate, s->stream);
  if (st == LUM_OK) st = s->cached.allocate(3 * n, precision, sym);
  if (st == LUM_OK) st = s->cached.assemble(s->otf, s->stream);
  if (st == LUM_OK) {
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) st = cuda_status(e, "assembly", __FILE__, __LINE__);
  }
  if (st != LUM_OK) {
    lum_session_destroy(s);
    return st;
  }
  *out = s;
  return LUM_OK;
}

// Sessions with the Sommerfeld substrate runtime (assembly.rs:157-166 and
// :296-303): the free-space or lattice operator plus -G_refl from the
// device table (sommerfeld.cu).
int lum_session_create_onthefly_sommerfeld(lum_ctx* ctx, int n, const double* pos,
                                           const double* inv_alpha, double k, int use_fcd,
                                           double cell, const lum_lattice* lattice,
                                           const double k_bloch[3], const lum_sommerfeld* somm,
                                           lum_session** out) {
  if (bad_ptr(ctx, "ctx") || bad_ptr(out, "out") || bad_ptr(somm, "somm")) return LUM_ERR_INVALID;
  *out = nullptr;
  lum_session* s = nullptr;
  LUM_TRY((lum_status)lum_session_create_onthefly(ctx, n, pos, inv_alpha, k, use_fcd, cell,
                                                  lattice, k_bloch, nullptr, &s));
  lum_status st = s->otf.somm_build(somm, s->stream);
  if (st == LUM_OK) {
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) st = cuda_status(e, "Sommerfeld table", __FILE__, __LINE__);
  }
  if (st != LUM_OK) {
    lum_session_destroy(s);
    return st;
  }
  *out = s;
  return LUM_OK;
}

int lum_session_assemble_sommerfeld(lum_ctx* ctx, int n, const double* pos,
                                    const double* inv_alpha, double k, int use_fcd, double cell,
                                    const lum_lattice* lattice, const double k_bloch[3],
                                    const lum_sommerfeld* somm, int precision,
                                    lum_session** out) {
  if (bad_ptr(ctx, "ctx") || bad_ptr(out, "out") || bad_ptr(somm, "somm")) return LUM_ERR_INVALID;
  *out = nullptr;
  LUM_TRY(check_inputs(n, pos, inv_alpha, k));
  if (precision != LUM_FP32 && precision != LUM_FP64) {
    set_error("invalid storage precision %d", precision);
    return LUM_ERR_INVALID;
  }
  lum_session* s = nullptr;
  LUM_TRY(new_session(ctx, 1, 3 * n, &s));
  lum_status st = s->otf.build_geometry(pos, n, s->stream);
  if (st == LUM_OK)
    st = s->otf.set_physics(k, inv_alpha, use_fcd, cell, lattice, k_bloch, nullptr, s->stream);
  if (st == LUM_OK) st = s->otf.somm_build(somm, s->stream);
  if (st == LUM_OK) st = s->cached.allocate(3 * n, precision);
  if (st == LUM_OK) st = s->cached.assemble(s->otf, s->stream);
  if (st == LUM_OK) {
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) st = cuda_status(e, "assembly", __FILE__, __LINE__);
  }
  if (st != LUM_OK) {
    lum_session_destroy(s);
    return st;
  }
  *out = s;
  return LUM_OK;
}

int lum_session_set_sommerfeld(lum_session* s, const lum_sommerfeld* somm) {
  if (bad_ptr(s, "session") || bad_ptr(somm, "somm")) return LUM_ERR_INVALID;
  if (s->kind == 1 && s->cached.packed) {
    set_error("symmetric tile storage needs a free-space system (no substrate)");
    return LUM_ERR_INVALID;
  }
  if (s->kind == 2) {
    if (s->fft.refl_mode == 1) {
      set_error("the session already has a Fresnel substrate");
      return LUM_ERR_INVALID;
    }
    lum::SommDev S;
    LUM_TRY(lum::somm_params(somm, &S));
    cudaSetDevice(s->ctx->device);
    LUM_TRY(s->fft.set_reflection(2, nullptr, &S, s->stream));
    LUM_TRY_CUDA(cudaStreamSynchronize(s->stream));
    return LUM_OK;
  }
  if (!s->otf.inv_alpha.p) {
    set_error("the Sommerfeld substrate needs an on-the-fly or assembled session");
    return LUM_ERR_INVALID;
  }
  if (s->otf.has_substrate) {
    set_error("the session already has a Fresnel substrate");
    return LUM_ERR_INVALID;
  }
  cudaSetDevice(s->ctx->device);
  LUM_TRY(s->otf.somm_build(somm, s->stream));
  if (s->kind == 1) LUM_TRY(s->cached.assemble(s->otf, s->stream));
  LUM_TRY_CUDA(cudaStreamSynchronize(s->stream));
  return LUM_OK;
}

int lum_session_matvec_device(lum_session* s, int precision, const void* x, void* y,
                              void* stream) {
  if (bad_ptr(s, "session") || bad_ptr(x, "x") || bad_ptr(y, "y")) return LUM_ERR_INVALID;
  if (precision != LUM_FP32 && precision != LUM_FP64) {
    set_error("invalid precision %d", precision);
    return LUM_ERR_INVALID;
  }
  cudaSetDevice(s->ctx->device);
  cudaStream_t keep = s->stream;
  if (stream) s->stream = (cudaStream_t)stream;
  lum_status st = s->apply(precision, (const double2*)x, (double2*)y);
  s->stream = keep;
  return st;
}

// Host-path staging buffers of a session: grown on demand and kept, since a
// cudaMalloc / cudaFree pair per call costs far more than the copies.
static lum_status grow_buf(lum::DevBuf& b, size_t bytes) {
  return b.bytes >= bytes ? LUM_OK : b.alloc(bytes);
}

int lum_session_matvec(lum_session* s, int precision, const double* x, double* y) {
  if (bad_ptr(s, "session") || bad_ptr(x, "x") || bad_ptr(y, "y")) return LUM_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  const size_t bytes = sizeof(double2) * (size_t)s->dim;
  LUM_TRY(grow_buf(s->xbuf, bytes));
  LUM_TRY(grow_buf(s->ybuf, bytes));
  LUM_TRY_CUDA(cudaMemcpyAsync(s->xbuf.p, x, bytes, cudaMemcpyHostToDevice, s->stream));
  LUM_TRY(s->apply(precision, s->xbuf.as<double2>(), s->ybuf.as<double2>()));
  LUM_TRY_CUDA(cudaMemcpyAsync(y, s->ybuf.p, bytes, cudaMemcpyDeviceToHost, s->stream));
  LUM_TRY_CUDA(cudaStreamSynchronize(s->stream));
  return LUM_OK;
}

static lum_status check_matmul(lum_session* s, const void* X, const void* Y, int nrhs,
                               int method) {
  if (bad_ptr(s, "session") || bad_ptr(X, "X") || bad_ptr(Y, "Y")) return LUM_ERR_INVALID;
  if (s->kind != 1 || nrhs <= 0) {
    set_error("matmul needs a cached session and nrhs > 0");
    return LUM_ERR_INVALID;
  }
  if (method != LUM_MATMUL_AUTO && method != LUM_MATMUL_TENSOR &&
      method != LUM_MATMUL_CUDA_CORES) {
    set_error("invalid matmul method %d", method);
    return LUM_ERR_INVALID;
  }
  if (s->otf.has_somm && s->otf.somm_stale) {
    set_error("the matrix was not re-assembled for the new wavelength: call "
              "lum_session_set_sommerfeld after lum_session_set_wavelength");
    return LUM_ERR_INVALID;
  }
  return LUM_OK;
}

int lum_session_matmul_device(lum_session* s, const void* X, void* Y, int nrhs, void* stream) {
  LUM_TRY(check_matmul(s, X, Y, nrhs, LUM_MATMUL_AUTO));
  cudaSetDevice(s->ctx->device);
  return s->cached.apply_multi((const double2*)X, (double2*)Y, nrhs, nrhs, 1, LUM_MATMUL_AUTO,
                               stream ? (cudaStream_t)stream : s->stream);
}

int lum_session_matmul_vectors_device(lum_session* s, const void* X, void* Y, int nrhs,
                                      int method, void* stream) {
  LUM_TRY(check_matmul(s, X, Y, nrhs, method));
  cudaSetDevice(s->ctx->device);
  return s->cached.apply_multi((const double2*)X, (double2*)Y, nrhs, 1, s->dim, method,
                               stream ? (cudaStream_t)stream : s->stream);
}

int lum_session_matmul_vectors(lum_session* s, const double* X, double* Y, int nrhs,
                               int method) {
  LUM_TRY(check_matmul(s, X, Y, nrhs, method));
  cudaSetDevice(s->ctx->device);
  const size_t bytes = sizeof(double2) * (size_t)s->dim * nrhs;
  LUM_TRY(grow_buf(s->xbuf, bytes));
  LUM_TRY(grow_buf(s->ybuf, bytes));
  LUM_TRY_CUDA(cudaMemcpyAsync(s->xbuf.p, X, bytes, cudaMemcpyHostToDevice, s->stream));
  LUM_TRY(s->cached.apply_multi(s->xbuf.as<double2>(), s->ybuf.as<double2>(), nrhs, 1, s->dim,
                                method, s->stream));
  LUM_TRY_CUDA(cudaMemcpyAsync(Y, s->ybuf.p, bytes, cudaMemcpyDeviceToHost, s->stream));
  LUM_TRY_CUDA(cudaStreamSynchronize(s->stream));
  return lum::cgemm_status(s->cached, s->stream);
}

// nrhs right-hand sides of one session, two at a time in lockstep.
int lum_solve_gmres_multi_device(lum_session* s, int nrhs, const void* b_dev, void* x_dev,
                                 double tol, int max_iter, int restart, int mode,
                                 lum_solve_info* info, void* stream) {
  if (bad_ptr(s, "session") || bad_ptr(b_dev, "b") || bad_ptr(x_dev, "x")) return LUM_ERR_INVALID;
  if (nrhs < 1 || (mode != LUM_SOLVE_FP64 && mode != LUM_SOLVE_FP32_REFINE) || !(tol > 0.0)) {
    set_error("invalid multi-RHS solve (nrhs %d, mode %d, tol %g)", nrhs, mode, tol);
    return LUM_ERR_INVALID;
  }
  cudaSetDevice(s->ctx->device);
  cudaStream_t keep = s->stream;
  if (stream) s->stream = (cudaStream_t)stream;
  const double2* b = static_cast<const double2*>(b_dev);
  double2* x = static_cast<double2*>(x_dev);
  const size_t len = (size_t)s->dim;
  lum_status worst = LUM_OK;
  for (int r = 0; r < nrhs; r += 2) {
    const int g = std::min(2, nrhs - r);
    const double2* bb[2] = {b + r * len, b + (r + g - 1) * len};
    double2* xx[2] = {x + r * len, x + (r + g - 1) * len};
    lum_status st = lum_gmres_device_multi(s, g, bb, xx, tol, max_iter, restart, mode,
                                           info ? info + r : nullptr, s->stream);
    if (st == LUM_ERR_NOT_CONVERGED) {
      worst = st;
    } else if (st != LUM_OK) {
      s->stream = keep;
      return st;
    }
  }
  s->stream = keep;
  return worst;
}

int lum_solve_gmres_multi(lum_session* s, int nrhs, const double* b, double tol, int max_iter,
                          int restart, int mode, double* x, lum_solve_info* info) {
  if (bad_ptr(s, "session") || bad_ptr(b, "b") || bad_ptr(x, "x")) return LUM_ERR_INVALID;
  if (nrhs < 1) {
    set_error("nrhs must be positive");
    return LUM_ERR_INVALID;
  }
  cudaSetDevice(s->ctx->device);
  const size_t bytes = sizeof(double2) * (size_t)s->dim * nrhs;
  LUM_TRY(grow_buf(s->bbuf, bytes));
  LUM_TRY(grow_buf(s->xbuf, bytes));
  LUM_TRY_CUDA(cudaMemcpyAsync(s->bbuf.p, b, bytes, cudaMemcpyHostToDevice, s->stream));
  int st = lum_solve_gmres_multi_device(s, nrhs, s->bbuf.p, s->xbuf.p, tol, max_iter, restart,
                                        mode, info, nullptr);
  if (st == LUM_OK || st == LUM_ERR_NOT_CONVERGED) {
    LUM_TRY_CUDA(cudaMemcpyAsync(x, s->xbuf.p, bytes, cudaMemcpyDeviceToHost, s->stream));
    LUM_TRY_CUDA(cudaStreamSynchronize(s->stream));
  }
  return st;
}

int lum_solve_gmres_device(lum_session* s, const void* b, void* x, double tol, int max_iter,
                           int restart, int mode, lum_solve_info* info, void* stream) {
  if (bad_ptr(s, "session") || bad_ptr(b, "b") || bad_ptr(x, "x")) return LUM_ERR_INVALID;
  if (!(tol > 0.0) || max_iter < 0 || restart < 0 || restart > kMaxRestart ||
      (mode != LUM_SOLVE_FP64 && mode != LUM_SOLVE_FP32_REFINE)) {
    set_error("invalid solve arguments (tol %g, max_iter %d, restart %d, mode %d)", tol,
              max_iter, restart, mode);
    return LUM_ERR_INVALID;
  }
  cudaSetDevice(s->ctx->device);
  cudaStream_t keep = s->stream;
  if (stream) s->stream = (cudaStream_t)stream;
  lum_status st = lum_gmres_device(s, (const double2*)b, (double2*)x, tol, max_iter, restart,
                                   mode, info, s->stream);
  s->stream = keep;
  return st;
}

int lum_solve_gmres(lum_session* s, const double* b, double tol, int max_iter, int restart,
                    int mode, double* x, lum_solve_info* info) {
  if (bad_ptr(s, "session") || bad_ptr(b, "b") || bad_ptr(x, "x")) return LUM_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  const size_t bytes = sizeof(double2) * (size_t)s->dim;
  LUM_TRY(grow_buf(s->bbuf, bytes));
  LUM_TRY(grow_buf(s->xbuf, bytes));
  LUM_TRY(grow_buf(s->ybuf, bytes));
  LUM_TRY_CUDA(cudaMemcpyAsync(s->bbuf.p, b, bytes, cudaMemcpyHostToDevice, s->stream));
  int st = lum_solve_gmres_device(s, s->bbuf.p, s->xbuf.p, tol, max_iter, restart, mode, info,
                                  nullptr);
  if (st == LUM_OK || st == LUM_ERR_NOT_CONVERGED) {
    LUM_TRY_CUDA(cudaMemcpyAsync(x, s->xbuf.p, bytes, cudaMemcpyDeviceToHost, s->stream));
    LUM_TRY_CUDA(cudaStreamSynchronize(s->stream));
  }
  return st;
}

int lum_session_profile(lum_session* s, int enable) {
  if (bad_ptr(s, "session")) return LUM_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  LUM_TRY_CUDA(cudaStreamSynchronize(s->stream));
  s->profile = enable != 0;
  s->ev_used = 0;
  return LUM_OK;
}

int lum_session_kernel_time(lum_session* s, int precision, int* launches, double* total_ms) {
  if (bad_ptr(s, "session")) return LUM_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  LUM_TRY_CUDA(cudaStreamSynchronize(s->stream));
  double tot = 0.0;
  int cnt = 0;
  for (size_t q = 0; q < s->ev_used; ++q) {
    const auto& r = s->ev_pool[q];
    if (r.precision != precision) continue;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      tot += ms;
      ++cnt;
    } else {
      cudaGetLastError();
    }
  }
  if (launches) *launches = cnt;
  if (total_ms) *total_ms = tot;
  return LUM_OK;
}

int lum_session_stats(lum_session* s, long long* near_pairs, int* ell_width, int* nsplit32,
                      int* nsplit64) {
  if (bad_ptr(s, "session")) return LUM_ERR_INVALID;
  cudaSetDevice(s->ctx->device);
  LUM_TRY_CUDA(cudaStreamSynchronize(s->stream));
  if (near_pairs) {
    long long np = 0;
    if (s->otf.ell_w > 0) {
      std::vector<int> nj((size_t)s->otf.ell_w * s->otf.n);
      LUM_TRY_CUDA(cudaMemcpy(nj.data(), s->otf.near_j.p, sizeof(int) * nj.size(),
                              cudaMemcpyDeviceToHost));
      for (int v : nj) np += (v >= 0);
    }
    *near_pairs = np;
  }
  if (ell_width) *ell_width = s->otf.ell_w;
  if (nsplit32) *nsplit32 = s->otf.nsplit32;
  if (nsplit64) *nsplit64 = s->otf.nsplit64;
  return LUM_OK;
}

int lum_session_kernel_config(lum_session* s, char* buf, size_t len) {
  if (bad_ptr(s, "session") || bad_ptr(buf, "buf") || len == 0) return LUM_ERR_INVALID;
  const lum::OtfOperator& o = s->otf;
  snprintf(buf, len,
           "kind=%s f32_variant=%s tuned_ms=%.4f nsplit32=%d nsplit64=%d ell_w=%d lofree=%d "
           "fast_trig=%d f32x2_variant=%s tuned_x2_ms=%.4f nsplit_x2=%d f32_sym=%d "
           "sym_variant=%s tuned_sym_ms=%.4f f64_sym=%d tuned_f64_ms=%.4f f32x2_sym=%d "
           "sym2_variant=%s sym_superblocks=%d sommerfeld=%s somm_records=%lld",
           s->kind == 0 ? "onthefly" : (s->kind == 1 ? "cached" : "fft"),
           lum::f32_variant_name(o.f32_variant),
           (double)o.tuned_ms, o.nsplit32, o.nsplit64, o.ell_w, o.lofree, o.fast_trig,
           lum::f32x2_variant_name(o.f32x2_variant), (double)o.tuned_x2_ms, o.nsplit_x2,
           o.f32_sym, lum::sym_variant_name(o.f32_sym), (double)o.tuned_sym_ms, o.f64_sym,
           (double)o.tuned_f64_ms, o.f32x2_sym, lum::sym2_variant_name(o.f32x2_sym), o.sym_nb,
           o.has_somm ? (o.somm_keyed ? "lattice_keys" : "pairs") : "none",
           (long long)o.somm_records);
  return LUM_OK;
}

int lum_measure_fma2_peak(lum_ctx* ctx, double* gflops) {
  if (bad_ptr(ctx, "ctx") || bad_ptr(gflops, "gflops")) return LUM_ERR_INVALID;
  LUM_TRY_CUDA(cudaSetDevice(ctx->device));
  DevBuf out;
  LUM_TRY(out.alloc(16));
  cudaEvent_t e0, e1;
  LUM_TRY_CUDA(cudaEventCreate(&e0));
  LUM_TRY_CUDA(cudaEventCreate(&e1));
  const int threads = 256, blocks = ctx->sms * 8, iters = 2048;
  lum_status st = LUM_OK;
  float ms = 0.f;
  for (int rep = 0; rep < 2 && st == LUM_OK; ++rep) {
    cudaEventRecord(e0);
    fma2_chain<<<blocks, threads>>>(out.as<float>(), iters, 0.999999f, 1e-7f);
    cudaEventRecord(e1);
    const cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) st = cuda_status(e, "packed FMA microbenchmark", __FILE__, __LINE__);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
  if (st == LUM_OK) {
    cudaEventElapsedTime(&ms, e0, e1);
    // 8 chains x 16 unrolled x 2 lanes x 2 flops per f32x2 FMA
    *gflops = 2.0 * 2.0 * 8 * 16 * (double)iters * threads * blocks / (ms * 1e-3) / 1e9;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

int lum_measure_l2_peak(lum_ctx* ctx, double* gbs) {
  if (bad_ptr(ctx, "ctx") || bad_ptr(gbs, "gbs")) return LUM_ERR_INVALID;
  LUM_TRY_CUDA(cudaSetDevice(ctx->device));
  const size_t bytes = size_t(16) << 20;  // 16 MiB: L2-resident
  const size_t n4 = bytes / sizeof(float4);
  DevBuf buf, out;
  LUM_TRY(buf.alloc(bytes));
  LUM_TRY(out.alloc(16));
  LUM_TRY_CUDA(cudaMemset(buf.p, 0, bytes));
  cudaEvent_t e0, e1;
  LUM_TRY_CUDA(cudaEventCreate(&e0));
  LUM_TRY_CUDA(cudaEventCreate(&e1));
  const int threads = 512, blocks = ctx->sms * 4, reps = 64;
  float ms = 0.f;
  lum_status st = LUM_OK;
  for (int rep = 0; rep < 2 && st == LUM_OK; ++rep) {  // the first launch warms L2
    cudaEventRecord(e0);
    l2_read<<<blocks, threads>>>(buf.as<float4>(), n4, reps, out.as<float>());
    cudaEventRecord(e1);
    const cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) st = cuda_status(e, "L2 microbenchmark", __FILE__, __LINE__);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
  if (st == LUM_OK) {
    cudaEventElapsedTime(&ms, e0, e1);
    // each thread reads ceil(n4 / threads in the grid) entries per pass
    const size_t grid = (size_t)blocks * threads;
    const double read = (double)grid * (double)((n4 + grid - 1) / grid) * sizeof(float4) * reps;
    *gbs = read / (ms * 1e-3) / 1e9;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

int lum_measure_fma_peak(lum_ctx* ctx, double* fp32_gflops, double* fp64_gflops) {
  if (bad_ptr(ctx, "ctx")) return LUM_ERR_INVALID;
  LUM_TRY_CUDA(cudaSetDevice(ctx->device));
  DevBuf out;
  LUM_TRY(out.alloc(16));
  cudaEvent_t e0, e1;
  LUM_TRY_CUDA(cudaEventCreate(&e0));
  LUM_TRY_CUDA(cudaEventCreate(&e1));
  const int threads = 256;
  const int blocks = ctx->sms * 8;
  auto run = [&](bool dbl, int iters, double* gflops) -> lum_status {
    for (int rep = 0; rep < 2; ++rep) {
      cudaEventRecord(e0);
      if (dbl)
        fma_chain<double><<<blocks, threads>>>(out.as<double>(), iters, 0.999999, 1e-7);
      else
        fma_chain<float><<<blocks, threads>>>(out.as<float>(), iters, 0.999999f, 1e-7f);
      LUM_CHECK_LAUNCH();
      cudaEventRecord(e1);
      LUM_TRY_CUDA(cudaEventSynchronize(e1));
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    *gflops = flops / (ms * 1e-3) / 1e9;
    return LUM_OK;
  };
  double g32 = 0, g64 = 0;
  lum_status st = run(false, 4096, &g32);
  if (st == LUM_OK) st = run(true, 1024, &g64);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (fp32_gflops) *fp32_gflops = g32;
  if (fp64_gflops) *fp64_gflops = g64;
  return st;
}

}  // extern "C"
