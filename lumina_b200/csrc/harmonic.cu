// harmonic.cu -- nonlinear (SHG / THG) source moments on the device.
//
// compute_shg_sources / compute_thg_sources (crates/lumina-core/src/
// nonlinear.rs:61-86, :233-258) with Chi2Tensor::contract /
// Chi3Tensor::contract (types.rs:355-365, :461-472):
//   order 2: p_a = sum_{b,c}   chi_{abc}  E_b E_c     (27 components, a*9+b*3+c)
//   order 3: p_a = sum_{b,c,d} chi_{abcd} E_b E_c E_d (81 components)
// per dipole, in FP64, the products formed left to right as the reference
// does ((chi * E_b) * E_c ...).  One thread per dipole; the tensor is shared
// by all dipoles or given per dipole.  The harmonic solve itself is an
// ordinary session solve with these moments as the right-hand side.
#include "lumina_internal.cuh"

namespace lum {
namespace {

__device__ __forceinline__ double2 zm(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

template <int ORDER>
__global__ void harmonic_sources(int n, const double2* __restrict__ e_loc, int per_dipole,
                                 const double2* __restrict__ chi, double2* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  constexpr int NC = ORDER == 2 ? 27 : 81;
  const double2* t = chi + (per_dipole ? (size_t)i * NC : 0);
  const double2 e[3] = {e_loc[3 * (size_t)i], e_loc[3 * (size_t)i + 1], e_loc[3 * (size_t)i + 2]};
  for (int a = 0; a < 3; ++a) {
    double2 p = make_double2(0.0, 0.0);
    for (int b = 0; b < 3; ++b)
      for (int c = 0; c < 3; ++c) {
        if (ORDER == 2) {
          const double2 v = zm(zm(t[a * 9 + b * 3 + c], e[b]), e[c]);
          p.x += v.x;
          p.y += v.y;
        } else {
          for (int d = 0; d < 3; ++d) {
            const double2 v = zm(zm(zm(t[a * 27 + b * 9 + c * 3 + d], e[b]), e[c]), e[d]);
            p.x += v.x;
            p.y += v.y;
          }
        }
      }
    out[3 * (size_t)i + a] = p;
  }
}

}  // namespace
}  // namespace lum

using namespace lum;

int lum_harmonic_sources(lum_ctx* ctx, int order, int n, const double* local_fields,
                         int n_tensors, const double* chi, double* sources) {
  if (!ctx || (order != 2 && order != 3) || n < 0 ||
      (n > 0 && (!local_fields || !chi || !sources)) || (n_tensors != 1 && n_tensors != n)) {
    set_error("invalid harmonic-source arguments (order %d, n %d, tensors %d)", order, n,
              n_tensors);
    return LUM_ERR_INVALID;
  }
  if (n == 0) return LUM_OK;
  const int nc = order == 2 ? 27 : 81;
  for (size_t q = 0; q < 6 * (size_t)n; ++q)
    if (!std::isfinite(local_fields[q])) {
      set_error("non-finite local field at dipole %zu", q / 6);
      return LUM_ERR_INVALID;
    }
  LUM_TRY_CUDA(cudaSetDevice(ctx->device));
  FieldWork* fw = nullptr;
  LUM_TRY(ctx_work(ctx, &fw));
  std::lock_guard<std::mutex> lk(fw->mu);
  cudaStream_t st = fw->stream;
  DevBuf &de = fw->h_e, &dc = fw->h_chi, &dp = fw->h_p;
  const size_t vb = sizeof(double2) * 3 * (size_t)n, cb = sizeof(double2) * nc * (size_t)n_tensors;
  auto grow = [](DevBuf& b, size_t bytes) { return b.bytes >= bytes ? LUM_OK : b.alloc(bytes); };
  LUM_TRY(grow(de, vb));
  LUM_TRY(grow(dc, cb));
  LUM_TRY(grow(dp, vb));
  LUM_TRY_CUDA(cudaMemcpyAsync(de.p, local_fields, vb, cudaMemcpyHostToDevice, st));
  LUM_TRY_CUDA(cudaMemcpyAsync(dc.p, chi, cb, cudaMemcpyHostToDevice, st));
  const int per = n_tensors == n && n > 1 ? 1 : 0;
  if (order == 2)
    harmonic_sources<2><<<(n + 127) / 128, 128, 0, st>>>(n, de.as<double2>(), per,
                                                         dc.as<double2>(), dp.as<double2>());
  else
    harmonic_sources<3><<<(n + 127) / 128, 128, 0, st>>>(n, de.as<double2>(), per,
                                                         dc.as<double2>(), dp.as<double2>());
  LUM_CHECK_LAUNCH();
  LUM_TRY_CUDA(cudaMemcpyAsync(sources, dp.p, vb, cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));
  return LUM_OK;
}
