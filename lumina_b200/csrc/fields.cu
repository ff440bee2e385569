// fields.cu -- fields from solved dipole moments (fields.rs) on the device.
//
// Near field (field_at_point, fields.rs:18-49): E(r) = E_inc(r) + sum_i
// G(r - r_i) p_i over every dipole with |r - r_i|^2 >= 1e-20, with the
// point-dipole tensor of greens.rs:34-71 in the contracted form
//   G p = A p + B' d (d . p),  A = pf (1 - u^2 + i u),
//   B' = pf (3u^2 - 1 - 3iu) / R^2,  pf = k^2 e^{ikR} / (4 pi R),  u = 1/(kR),
// in FP64.  One thread per observation point; the dipoles (position and
// moment) are staged through shared memory in tiles, and the dipole range is
// split over gridDim.y so that small maps still fill the SMs; the splits are
// summed in a fixed order with the incident field (types.rs:60-73).
//
// Far field (compute_far_field, fields.rs:147-221): per direction
// r = (sin t cos p, sin t sin p, cos t), F = sum_i p_i e^{-ik r.r_i} in FP64,
// then |(I - r r) . F|^2, with the same tiling and split summation.
//
// The near-field map (compute_near_field_map, fields.rs:52-139) builds its
// plane grid on the host exactly as the reference does and evaluates it with
// the near-field kernel.
#include "lumina_internal.cuh"
#include "device_sincos.cuh"

#include <algorithm>
#include <new>
#include <cmath>

namespace lum {

lum_status ctx_work(lum_ctx* ctx, FieldWork** out) {
  static std::mutex create_mu;
  std::lock_guard<std::mutex> lk(create_mu);
  if (!ctx->fields) {
    std::unique_ptr<FieldWork> fw(new (std::nothrow) FieldWork());
    if (!fw) return LUM_ERR_OOM;
    LUM_TRY_CUDA(cudaStreamCreateWithFlags(&fw->stream, cudaStreamNonBlocking));
    ctx->fields = std::move(fw);
  }
  *out = ctx->fields.get();
  return LUM_OK;
}

namespace {

constexpr int kFieldBlock = 128;

struct SrcTile {
  double4 pos[kFieldBlock];
  double2 mom[3][kFieldBlock];
};

__global__ void __launch_bounds__(kFieldBlock)
near_field_part(int n, const double4* __restrict__ pos, const double2* __restrict__ mom,
                double k, int m, const double4* __restrict__ obs, int chunk,
                double2* __restrict__ part) {
  __shared__ SrcTile t;
  __shared__ double2 sTab[kScTab];
  sincos_table_stage(sTab);  // the first tile's barrier precedes its use
  const int q = blockIdx.x * kFieldBlock + threadIdx.x;
  const double4 o = obs[min(q, m - 1)];
  const int j0 = blockIdx.y * chunk, j1 = min(n, j0 + chunk);
  const double s0 = k * k * k / (4.0 * kPi), ik = 1.0 / k;
  double er[3] = {0.0, 0.0, 0.0}, ei[3] = {0.0, 0.0, 0.0};
  for (int jt = j0; jt < j1; jt += kFieldBlock) {
    const int cnt = min(kFieldBlock, j1 - jt);
    __syncthreads();
    if (threadIdx.x < cnt) {
      const int j = jt + threadIdx.x;
      t.pos[threadIdx.x] = pos[j];
      for (int c = 0; c < 3; ++c) t.mom[c][threadIdx.x] = mom[3 * j + c];
    }
    __syncthreads();
    for (int jj = 0; jj < cnt; ++jj) {
      const double4 r = t.pos[jj];
      const double dx = o.x - r.x, dy = o.y - r.y, dz = o.z - r.z;
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 < 1e-20) continue;  // fields.rs:35-37
      const double ir = rsqrt(r2);
      const double R = r2 * ir;
      const double u = ir * ik, u2 = u * u;
      double sn, cs;
      sincos_tab(k * R, sTab, &sn, &cs);
      const double qf = s0 * u;  // k^2 / (4 pi R)
      const double pr = qf * cs, pi = qf * sn;
      const double ar = 1.0 - u2;
      const double Ar = pr * ar - pi * u, Ai = pr * u + pi * ar;
      const double br = 3.0 * u2 - 1.0, bi = -3.0 * u;
      const double ir2 = ir * ir;
      const double Br = (pr * br - pi * bi) * ir2, Bi = (pr * bi + pi * br) * ir2;
      const double2 p0 = t.mom[0][jj], p1 = t.mom[1][jj], p2 = t.mom[2][jj];
      const double sr = dx * p0.x + dy * p1.x + dz * p2.x;
      const double si = dx * p0.y + dy * p1.y + dz * p2.y;
      const double tr = Br * sr - Bi * si, ti = Br * si + Bi * sr;
      er[0] += Ar * p0.x - Ai * p0.y + tr * dx;
      ei[0] += Ar * p0.y + Ai * p0.x + ti * dx;
      er[1] += Ar * p1.x - Ai * p1.y + tr * dy;
      ei[1] += Ar * p1.y + Ai * p1.x + ti * dy;
      er[2] += Ar * p2.x - Ai * p2.y + tr * dz;
      ei[2] += Ar * p2.y + Ai * p2.x + ti * dz;
    }
  }
  if (q < m)
    for (int c = 0; c < 3; ++c)
      part[(size_t)blockIdx.y * 3 * m + 3 * (size_t)q + c] = make_double2(er[c], ei[c]);
}

// E = E_inc + sum of the splits (split order); |E|^2 when `intensity` is set.
__global__ void near_field_finish(int m, const double4* __restrict__ obs, int nsplit,
                                  const double2* __restrict__ part, double k, double d0,
                                  double d1, double d2, double e0, double e1, double e2,
                                  double amplitude, double2* __restrict__ field,
                                  double* __restrict__ intensity) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= m) return;
  const double4 o = obs[q];
  // IncidentField::at_position (types.rs:60-73): E0 e exp(i k d.r)
  double sn, cs;
  sincos(k * (d0 * o.x + d1 * o.y + d2 * o.z), &sn, &cs);
  const double pol[3] = {e0, e1, e2};
  double inten = 0.0;
  for (int c = 0; c < 3; ++c) {
    double vr = amplitude * pol[c] * cs, vi = amplitude * pol[c] * sn;
    for (int s = 0; s < nsplit; ++s) {
      const double2 v = part[(size_t)s * 3 * m + 3 * (size_t)q + c];
      vr += v.x;
      vi += v.y;
    }
    field[3 * (size_t)q + c] = make_double2(vr, vi);
    inten += vr * vr + vi * vi;
  }
  if (intensity) intensity[q] = inten;
}

__global__ void __launch_bounds__(kFieldBlock)
far_field_part(int n, const double4* __restrict__ pos, const double2* __restrict__ mom,
               double k, int n_theta, int n_phi, int chunk, double2* __restrict__ part) {
  __shared__ SrcTile t;
  __shared__ double2 sTab[kScTab];
  sincos_table_stage(sTab);  // the first tile's barrier precedes its use
  const int m = n_theta * n_phi;
  const int q = min(blockIdx.x * kFieldBlock + (int)threadIdx.x, m - 1);
  const int it = q / n_phi, ip = q % n_phi;
  const double th = kPi * (double)it / (double)max(n_theta - 1, 1);
  const double ph = 2.0 * kPi * (double)ip / (double)n_phi;
  double st, ct, sp, cp;
  sincos(th, &st, &ct);
  sincos(ph, &sp, &cp);
  const double rx = k * st * cp, ry = k * st * sp, rz = k * ct;
  const int j0 = blockIdx.y * chunk, j1 = min(n, j0 + chunk);
  double fr[3] = {0.0, 0.0, 0.0}, fi[3] = {0.0, 0.0, 0.0};
  for (int jt = j0; jt < j1; jt += kFieldBlock) {
    const int cnt = min(kFieldBlock, j1 - jt);
    __syncthreads();
    if (threadIdx.x < cnt) {
      const int j = jt + threadIdx.x;
      t.pos[threadIdx.x] = pos[j];
      for (int c = 0; c < 3; ++c) t.mom[c][threadIdx.x] = mom[3 * j + c];
    }
    __syncthreads();
    for (int jj = 0; jj < cnt; ++jj) {
      const double4 r = t.pos[jj];
      double sn, cs;
      // phase e^{-i k r.r_i} = cs - i sn
      sincos_tab(rx * r.x + ry * r.y + rz * r.z, sTab, &sn, &cs);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double2 p = t.mom[c][jj];
        fr[c] += p.x * cs + p.y * sn;
        fi[c] += p.y * cs - p.x * sn;
      }
    }
  }
  if (blockIdx.x * kFieldBlock + (int)threadIdx.x < m)
    for (int c = 0; c < 3; ++c)
      part[(size_t)blockIdx.y * 3 * m + 3 * (size_t)q + c] = make_double2(fr[c], fi[c]);
}

__global__ void far_field_finish(int n_theta, int n_phi, int nsplit,
                                 const double2* __restrict__ part, double* __restrict__ theta,
                                 double* __restrict__ phi, double* __restrict__ intensity) {
  const int m = n_theta * n_phi;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= m) return;
  const int it = q / n_phi, ip = q % n_phi;
  const double th = kPi * (double)it / (double)max(n_theta - 1, 1);
  const double ph = 2.0 * kPi * (double)ip / (double)n_phi;
  double st, ct, sp, cp;
  sincos(th, &st, &ct);
  sincos(ph, &sp, &cp);
  const double rh[3] = {st * cp, st * sp, ct};
  double fr[3], fi[3];
  for (int c = 0; c < 3; ++c) {
    fr[c] = fi[c] = 0.0;
    for (int s = 0; s < nsplit; ++s) {
      const double2 v = part[(size_t)s * 3 * m + 3 * (size_t)q + c];
      fr[c] += v.x;
      fi[c] += v.y;
    }
  }
  const double dr = rh[0] * fr[0] + rh[1] * fr[1] + rh[2] * fr[2];
  const double di = rh[0] * fi[0] + rh[1] * fi[1] + rh[2] * fi[2];
  double inten = 0.0;
  for (int c = 0; c < 3; ++c) {
    const double tr = fr[c] - dr * rh[c], ti = fi[c] - di * rh[c];
    inten += tr * tr + ti * ti;
  }
  theta[q] = th;
  phi[q] = ph;
  intensity[q] = inten;
}

// dipole splits so that (row blocks x splits) covers the SMs about twice
int field_splits(int blocks, int n, int sms) {
  const int tiles = std::max(1, (n + kFieldBlock - 1) / kFieldBlock);
  const int want = std::max(1, (2 * 4 * sms + blocks - 1) / blocks);
  return std::max(1, std::min(tiles, std::min(64, want)));
}

lum_status grow(DevBuf& b, size_t bytes) { return b.bytes >= bytes ? LUM_OK : b.alloc(bytes); }

lum_status field_work(lum_ctx* ctx, FieldWork** out) { return ctx_work(ctx, out); }

lum_status upload_sources(int n, const double* pos, const double* moments, DevBuf& dpos,
                          DevBuf& dmom, cudaStream_t st) {
  std::vector<double> p4(4 * (size_t)std::max(n, 1), 0.0);
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      const double v = pos[3 * (size_t)i + c];
      if (!std::isfinite(v)) {
        set_error("non-finite dipole position at index %d", i);
        return LUM_ERR_INVALID;
      }
      p4[4 * (size_t)i + c] = v;
    }
  for (size_t q = 0; q < 6 * (size_t)n; ++q)
    if (!std::isfinite(moments[q])) {
      set_error("non-finite dipole moment at dipole %zu", q / 6);
      return LUM_ERR_INVALID;
    }
  LUM_TRY(grow(dpos, sizeof(double) * p4.size()));
  LUM_TRY(grow(dmom, sizeof(double2) * 3 * (size_t)std::max(n, 1)));
  LUM_TRY_CUDA(cudaMemcpyAsync(dpos.p, p4.data(), sizeof(double) * p4.size(),
                               cudaMemcpyHostToDevice, st));
  if (n > 0)
    LUM_TRY_CUDA(cudaMemcpyAsync(dmom.p, moments, sizeof(double2) * 3 * (size_t)n,
                                 cudaMemcpyHostToDevice, st));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));  // p4 is freed on return
  return LUM_OK;
}

lum_status near_field_device(lum_ctx* ctx, int n, const double* pos, const double* moments,
                             double k, const double dir[3], const double pol[3],
                             double amplitude, int m, const double* obs, double* field,
                             double* intensity) {
  LUM_TRY(sincos_table_ready());
  FieldWork* fw = nullptr;
  LUM_TRY(field_work(ctx, &fw));
  std::lock_guard<std::mutex> lk(fw->mu);
  cudaStream_t st = fw->stream;
  DevBuf &dpos = fw->pos, &dmom = fw->mom, &dobs = fw->obs, &dpart = fw->part,
         &dfield = fw->field, &dint = fw->inten;
  LUM_TRY(upload_sources(n, pos, moments, dpos, dmom, st));
  std::vector<double> o4(4 * (size_t)m, 0.0);
  for (int q = 0; q < m; ++q)
    for (int c = 0; c < 3; ++c) {
      const double v = obs[3 * (size_t)q + c];
      if (!std::isfinite(v)) {
        set_error("non-finite observation point at index %d", q);
        return LUM_ERR_INVALID;
      }
      o4[4 * (size_t)q + c] = v;
    }
  LUM_TRY(grow(dobs, sizeof(double) * o4.size()));
  LUM_TRY_CUDA(cudaMemcpyAsync(dobs.p, o4.data(), sizeof(double) * o4.size(),
                               cudaMemcpyHostToDevice, st));
  const int blocks = (m + kFieldBlock - 1) / kFieldBlock;
  const int ns = n > 0 ? field_splits(blocks, n, ctx->sms) : 0;
  const int chunk = ns > 0 ? ((n + ns - 1) / ns + kFieldBlock - 1) / kFieldBlock * kFieldBlock : 0;
  const int nsplit = ns > 0 ? (n + chunk - 1) / chunk : 0;
  LUM_TRY(grow(dpart, sizeof(double2) * 3 * (size_t)m * std::max(nsplit, 1)));
  LUM_TRY(grow(dfield, sizeof(double2) * 3 * (size_t)m));
  if (intensity) LUM_TRY(grow(dint, sizeof(double) * (size_t)m));
  if (nsplit > 0) {
    near_field_part<<<dim3(blocks, nsplit), kFieldBlock, 0, st>>>(
        n, dpos.as<double4>(), dmom.as<double2>(), k, m, dobs.as<double4>(), chunk,
        dpart.as<double2>());
    LUM_CHECK_LAUNCH();
  }
  near_field_finish<<<(m + 255) / 256, 256, 0, st>>>(
      m, dobs.as<double4>(), nsplit, dpart.as<double2>(), k, dir[0], dir[1], dir[2], pol[0],
      pol[1], pol[2], amplitude, dfield.as<double2>(), intensity ? dint.as<double>() : nullptr);
  LUM_CHECK_LAUNCH();
  if (field)
    LUM_TRY_CUDA(cudaMemcpyAsync(field, dfield.p, sizeof(double2) * 3 * (size_t)m,
                                 cudaMemcpyDeviceToHost, st));
  if (intensity)
    LUM_TRY_CUDA(cudaMemcpyAsync(intensity, dint.p, sizeof(double) * (size_t)m,
                                 cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));
  return LUM_OK;
}

bool finite3(const double* v) {
  return v && std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]);
}

lum_status check_field_args(lum_ctx* ctx, int n, const double* pos, const double* moments,
                            double k) {
  if (!ctx) {
    set_error("null context");
    return LUM_ERR_INVALID;
  }
  if (n < 0 || (n > 0 && (!pos || !moments))) {
    set_error("invalid dipole arrays (n = %d)", n);
    return LUM_ERR_INVALID;
  }
  if (!(k > 0.0) || !std::isfinite(k)) {
    set_error("wavenumber must be positive and finite (got %g)", k);
    return LUM_ERR_INVALID;
  }
  return LUM_OK;
}

}  // namespace
}  // namespace lum

using namespace lum;

int lum_near_field(lum_ctx* ctx, int n, const double* pos, const double* moments, double k,
                   const double direction[3], const double polarisation[3], double amplitude,
                   int m, const double* obs, double* field, double* intensity) {
  LUM_TRY(check_field_args(ctx, n, pos, moments, k));
  if (m < 0 || (m > 0 && !obs) || !finite3(direction) || !finite3(polarisation) ||
      !std::isfinite(amplitude)) {
    set_error("invalid observation points or incident field");
    return LUM_ERR_INVALID;
  }
  if (m == 0) return LUM_OK;
  LUM_TRY_CUDA(cudaSetDevice(ctx->device));
  return near_field_device(ctx, n, pos, moments, k, direction, polarisation, amplitude, m, obs,
                           field, intensity);
}

int lum_near_field_map(lum_ctx* ctx, int n, const double* pos, const double* moments, double k,
                       const double direction[3], const double polarisation[3],
                       double amplitude, const double centre[3], const double normal[3],
                       double half_width, double half_height, int nx, int ny, double* positions,
                       double* intensity, double extent[4]) {
  LUM_TRY(check_field_args(ctx, n, pos, moments, k));
  if (!finite3(centre) || !finite3(normal) || !std::isfinite(half_width) ||
      !std::isfinite(half_height) || nx < 0 || ny < 0 || !finite3(direction) ||
      !finite3(polarisation) || !std::isfinite(amplitude)) {
    set_error("invalid near-field plane or incident field");
    return LUM_ERR_INVALID;
  }
  const double nl = std::sqrt(normal[0] * normal[0] + normal[1] * normal[1] +
                              normal[2] * normal[2]);
  if (!(nl > 0.0)) {
    set_error("near-field plane normal is zero");
    return LUM_ERR_INVALID;
  }
  // plane_basis (fields.rs:111-139)
  const double nv[3] = {normal[0] / nl, normal[1] / nl, normal[2] / nl};
  double seed[3] = {0.0, 1.0, 0.0};
  if (std::fabs(nv[0]) < 0.9) {
    seed[0] = 1.0;
    seed[1] = 0.0;
  }
  const double dot = seed[0] * nv[0] + seed[1] * nv[1] + seed[2] * nv[2];
  const double ur[3] = {seed[0] - dot * nv[0], seed[1] - dot * nv[1], seed[2] - dot * nv[2]};
  const double ul = std::sqrt(ur[0] * ur[0] + ur[1] * ur[1] + ur[2] * ur[2]);
  const double u[3] = {ur[0] / ul, ur[1] / ul, ur[2] / ul};
  const double v[3] = {nv[1] * u[2] - nv[2] * u[1], nv[2] * u[0] - nv[0] * u[2],
                       nv[0] * u[1] - nv[1] * u[0]};
  // the grid of compute_near_field_map (fields.rs:61-95): iy outer, ix inner
  const double x_min = -half_width, x_max = half_width;
  const double y_min = -half_height, y_max = half_height;
  const double dx = nx > 1 ? (x_max - x_min) / (double)(nx - 1) : 0.0;
  const double dy = ny > 1 ? (y_max - y_min) / (double)(ny - 1) : 0.0;
  const size_t m = (size_t)nx * ny;
  if (m > 0x7fffffff) {
    set_error("near-field map too large");
    return LUM_ERR_INVALID;
  }
  std::vector<double> grid(3 * m);
  size_t q = 0;
  for (int iy = 0; iy < ny; ++iy)
    for (int ix = 0; ix < nx; ++ix) {
      const double uu = x_min + (double)ix * dx, vv = y_min + (double)iy * dy;
      for (int c = 0; c < 3; ++c) grid[3 * q + c] = centre[c] + uu * u[c] + vv * v[c];
      ++q;
    }
  if (extent) {
    extent[0] = centre[0] + x_min * u[0] + y_min * v[0];
    extent[1] = centre[0] + x_max * u[0] + y_max * v[0];
    extent[2] = centre[1] + x_min * u[1] + y_min * v[1];
    extent[3] = centre[1] + x_max * u[1] + y_max * v[1];
  }
  if (positions) std::copy(grid.begin(), grid.end(), positions);
  if (m == 0) return LUM_OK;
  LUM_TRY_CUDA(cudaSetDevice(ctx->device));
  return near_field_device(ctx, n, pos, moments, k, direction, polarisation, amplitude, (int)m,
                           grid.data(), nullptr, intensity);
}

int lum_far_field(lum_ctx* ctx, int n, const double* pos, const double* moments, double k,
                  int n_theta, int n_phi, double* theta, double* phi, double* intensity) {
  LUM_TRY(check_field_args(ctx, n, pos, moments, k));
  if (n_theta < 0 || n_phi < 0 || !theta || !phi || !intensity) {
    set_error("invalid far-field grid or output arrays");
    return LUM_ERR_INVALID;
  }
  const size_t m = (size_t)n_theta * n_phi;
  if (m == 0) return LUM_OK;
  if (m > 0x7fffffff) {
    set_error("far-field grid too large");
    return LUM_ERR_INVALID;
  }
  LUM_TRY_CUDA(cudaSetDevice(ctx->device));
  LUM_TRY(sincos_table_ready());
  FieldWork* fw = nullptr;
  LUM_TRY(field_work(ctx, &fw));
  std::lock_guard<std::mutex> lk(fw->mu);
  cudaStream_t st = fw->stream;
  DevBuf &dpos = fw->pos, &dmom = fw->mom, &dpart = fw->part, &dth = fw->th, &dph = fw->ph,
         &dint = fw->inten;
  LUM_TRY(upload_sources(n, pos, moments, dpos, dmom, st));
  const int blocks = (int)((m + kFieldBlock - 1) / kFieldBlock);
  const int ns = n > 0 ? field_splits(blocks, n, ctx->sms) : 0;
  const int chunk = ns > 0 ? ((n + ns - 1) / ns + kFieldBlock - 1) / kFieldBlock * kFieldBlock : 0;
  const int nsplit = ns > 0 ? (n + chunk - 1) / chunk : 0;
  LUM_TRY(grow(dpart, sizeof(double2) * 3 * m * std::max(nsplit, 1)));
  LUM_TRY(grow(dth, sizeof(double) * m));
  LUM_TRY(grow(dph, sizeof(double) * m));
  LUM_TRY(grow(dint, sizeof(double) * m));
  if (nsplit > 0) {
    far_field_part<<<dim3(blocks, nsplit), kFieldBlock, 0, st>>>(
        n, dpos.as<double4>(), dmom.as<double2>(), k, n_theta, n_phi, chunk,
        dpart.as<double2>());
    LUM_CHECK_LAUNCH();
  }
  far_field_finish<<<(unsigned)((m + 255) / 256), 256, 0, st>>>(
      n_theta, n_phi, nsplit, dpart.as<double2>(), dth.as<double>(), dph.as<double>(),
      dint.as<double>());
  LUM_CHECK_LAUNCH();
  LUM_TRY_CUDA(cudaMemcpyAsync(theta, dth.p, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaMemcpyAsync(phi, dph.p, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaMemcpyAsync(intensity, dint.p, sizeof(double) * m, cudaMemcpyDeviceToHost,
                               st));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));
  return LUM_OK;
}
