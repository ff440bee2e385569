// grad.cu -- adjoint gradients of the extinction cross-section.
//
// No counterpart in the reference (it has no gradient code).  With
// A p = E (E the incident field, A = alpha^-1 - G), the extinction
// C_ext = k/|E0|^2 Im(E^H p) (cda/mod.rs:175-236, with a complex
// polarisation allowed) has
//   dC_ext = k/|E0|^2 Im( dE^H p + mu^T (dE - dA p) ),   A mu = conj(E),
// because A is complex symmetric (G(d) = G(d)^T = G(-d), alpha symmetric,
// the FCD cell average symmetric in its two dipoles): the adjoint solve is a
// forward solve of the same operator with the conjugate right-hand side, and
// both run in lockstep so each operator application serves the two.
//
// Positions.  Row i and column i of A depend on r_i; with d = r_i - r_j and
// G odd in its first derivative,
//   -mu^T (dA/dr_ic) p = sum_{j != i} [ mu_i^T dG_c(d) p_j + mu_j^T dG_c(d) p_i ],
// and the plane wave adds i k dhat_c (mu_i . E_i - conj(E_i) . p_i).
// Writing G(d) = A(R) I + B(R) d d^T (A, B the radial functions of the
// point tensor, greens.rs:34-71),
//   mu^T dG_c p = (d_c/R) [A' (mu.p) + B' (mu.d)(d.p)]
//                + B [mu_c (d.p) + (mu.d) p_c].
// The pair sum is one FP64 pass over all pairs that recomputes the tensor
// derivatives and contracts them with the moments (nothing N^2 is stored);
// FCD near pairs (greens.rs:94-167) swap the point derivative for the
// 27-node average of the derivative, applied in the finishing kernel.  The
// near/far switch at 2*cell is a step in A: the gradient is that of the
// branch each pair is on.
//
// Permittivity.  dC_ext/d eps_i = -k/|E0|^2 mu_i^T (d alpha_i^-1/d eps) p_i,
// reported as the derivatives with respect to Re(eps_i) and Im(eps_i)
// (C_ext is the imaginary part of a holomorphic function of eps).
#include "lumina_internal.cuh"
#include "device_physics.cuh"
#include "device_sincos.cuh"

#include <cmath>
#include <vector>

namespace lum {
namespace {

constexpr int kGradBlock = 128;

__device__ __forceinline__ double2 c_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 c_scale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// a . b over three components, no conjugation
__device__ __forceinline__ double2 c_dot3(const double2* a, const double2* b) {
  double2 s = cmul(a[0], b[0]);
  s = c_add(s, cmul(a[1], b[1]));
  return c_add(s, cmul(a[2], b[2]));
}
__device__ __forceinline__ double2 r_dot3(const double d[3], const double2* a) {
  return make_double2(d[0] * a[0].x + d[1] * a[1].x + d[2] * a[2].x,
                      d[0] * a[0].y + d[1] * a[1].y + d[2] * a[2].y);
}

// Radial functions A, B of the point tensor and their R-derivatives:
//   A = e^{ikR}/(4 pi) (k^2/R - 1/R^3 + i k/R^2)
//   B = e^{ikR}/(4 pi) (-k^2/R^3 + 3/R^5 - 3ik/R^4)
//   X' = e^{ikR} (ik x + x') for X = e^{ikR} x.
struct Radial {
  double2 A, dA, B, dB;
};

__device__ __forceinline__ Radial radial(double R, double k, const double2* __restrict__ sTab) {
  const double ir = 1.0 / R, ir2 = ir * ir, ir3 = ir2 * ir, ir4 = ir2 * ir2, ir5 = ir4 * ir,
               ir6 = ir3 * ir3, k2 = k * k;
  double sn, cs;
  sincos_tab(k * R, sTab, &sn, &cs);
  const double f = 1.0 / (4.0 * kPi);
  const double2 e = make_double2(cs * f, sn * f);
  const double2 a = make_double2(k2 * ir - ir3, k * ir2);
  const double2 ap = make_double2(-k2 * ir2 + 3.0 * ir4, -2.0 * k * ir3);
  const double2 b = make_double2(-k2 * ir3 + 3.0 * ir5, -3.0 * k * ir4);
  const double2 bp = make_double2(3.0 * k2 * ir4 - 15.0 * ir6, 12.0 * k * ir5);
  Radial r;
  r.A = cmul(e, a);
  r.dA = cmul(e, make_double2(ap.x - k * a.y, ap.y + k * a.x));
  r.B = cmul(e, b);
  r.dB = cmul(e, make_double2(bp.x - k * b.y, bp.y + k * b.x));
  return r;
}

// g_c += mu_i^T dG_c(d) p_j + mu_j^T dG_c(d) p_i, scaled by w.
__device__ __forceinline__ void pair_grad(const double d[3], double k, const double2* mi,
                                          const double2* pi, const double2* mj,
                                          const double2* pj, double w, double2 g[3],
                                          const double2* __restrict__ sTab) {
  const double R = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  const Radial rf = radial(R, k, sTab);
  const double2 mid = r_dot3(d, mi), pid = r_dot3(d, pi);
  const double2 mjd = r_dot3(d, mj), pjd = r_dot3(d, pj);
  const double2 s1 = c_add(c_dot3(mi, pj), c_dot3(mj, pi));
  const double2 u1 = c_add(cmul(mid, pjd), cmul(mjd, pid));
  const double2 T = c_scale(c_add(cmul(rf.dA, s1), cmul(rf.dB, u1)), w / R);
  const double2 Bw = c_scale(rf.B, w);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double2 W = cmul(mi[c], pjd);
    W = c_add(W, cmul(mid, pj[c]));
    W = c_add(W, cmul(mj[c], pid));
    W = c_add(W, cmul(mjd, pi[c]));
    g[c] = c_add(g[c], c_add(c_scale(T, d[c]), cmul(Bw, W)));
  }
}

// Pair pass: thread per dipole i, sources [blockIdx.y*chunk, +chunk) staged
// through shared memory; partial[blockIdx.y][3i+c].
__global__ void __launch_bounds__(kGradBlock)
grad_pairs(int n, const double4* __restrict__ pos, const double2* __restrict__ p,
           const double2* __restrict__ mu, double k, int chunk, double2* __restrict__ partial) {
  __shared__ double4 sP[kGradBlock];
  __shared__ double2 sPm[3 * kGradBlock], sMu[3 * kGradBlock];
  __shared__ double2 sTab[kScTab];
  sincos_table_stage(sTab);  // the first tile's barrier precedes its use
  const int tid = threadIdx.x;
  const int i = blockIdx.x * kGradBlock + tid;
  const int ic = min(i, n - 1);
  const double4 ri = pos[ic];
  const double2 pi[3] = {p[3 * ic], p[3 * ic + 1], p[3 * ic + 2]};
  const double2 mi[3] = {mu[3 * ic], mu[3 * ic + 1], mu[3 * ic + 2]};
  double2 g[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
  const int j_begin = blockIdx.y * chunk, j_end = min(n, j_begin + chunk);
  for (int jt = j_begin; jt < j_end; jt += kGradBlock) {
    const int cnt = min(kGradBlock, j_end - jt);
    __syncthreads();
    if (tid < cnt) {
      const int j = jt + tid;
      sP[tid] = pos[j];
      for (int a = 0; a < 3; ++a) {
        sPm[3 * tid + a] = p[3 * j + a];
        sMu[3 * tid + a] = mu[3 * j + a];
      }
    }
    __syncthreads();
    for (int jj = 0; jj < cnt; ++jj) {
      if (jt + jj == i) continue;
      const double4 rj = sP[jj];
      const double d[3] = {ri.x - rj.x, ri.y - rj.y, ri.z - rj.z};
      pair_grad(d, k, mi, pi, sMu + 3 * jj, sPm + 3 * jj, 1.0, g, sTab);
    }
  }
  if (i < n) {
    const size_t off = (size_t)blockIdx.y * 3 * n + 3 * (size_t)i;
    for (int c = 0; c < 3; ++c) partial[off + c] = g[c];
  }
}

// Sum of the pair partials, FCD near-pair replacement, plane-wave and
// permittivity terms; outputs dC_ext/dr (3N) and dC_ext/dRe,Im(eps) (2N).
__global__ void __launch_bounds__(128)
grad_finish(int n, const double4* __restrict__ pos, const double2* __restrict__ p,
            const double2* __restrict__ mu, const double2* __restrict__ E, double k,
            double dx, double dy, double dz, const double2* __restrict__ partial, int nparts,
            int ell_w, const int* __restrict__ near_j, double cell,
            const double2* __restrict__ dinv, double scale, double* __restrict__ grad_r,
            double* __restrict__ grad_eps) {
  __shared__ double2 sTab[kScTab];
  sincos_table_stage(sTab);
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double2 pi[3] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
  const double2 mi[3] = {mu[3 * i], mu[3 * i + 1], mu[3 * i + 2]};
  double2 g[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
  for (int s = 0; s < nparts; ++s)
    for (int c = 0; c < 3; ++c) g[c] = c_add(g[c], partial[(size_t)s * 3 * n + 3 * (size_t)i + c]);
  // FCD: near pairs use the cell-averaged derivative (same nodes, weights
  // and node skip as the forward filter)
  const double4 ro = pos[i];
  const double nodes[3] = {-sqrt(3.0 / 5.0), 0.0, sqrt(3.0 / 5.0)};
  const double wts[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  const double half_d = cell / 2.0;
  for (int w = 0; w < ell_w; ++w) {
    const int j = near_j[(size_t)w * n + i];
    if (j < 0) break;
    const double4 rs = pos[j];
    const double2 pj[3] = {p[3 * j], p[3 * j + 1], p[3 * j + 2]};
    const double2 mj[3] = {mu[3 * j], mu[3 * j + 1], mu[3 * j + 2]};
    double2 ga[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    double tw = 0.0;
    for (int ix = 0; ix < 3; ++ix)
      for (int iy = 0; iy < 3; ++iy)
        for (int iz = 0; iz < 3; ++iz) {
          const double px = rs.x + half_d * nodes[ix];
          const double py = rs.y + half_d * nodes[iy];
          const double pz = rs.z + half_d * nodes[iz];
          const double d[3] = {ro.x - px, ro.y - py, ro.z - pz};
          if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < 1e-20) continue;
          const double wt = wts[ix] * wts[iy] * wts[iz];
          pair_grad(d, k, mi, pi, mj, pj, wt, ga, sTab);
          tw += wt;
        }
    const double inv = (tw > 1e-30) ? 1.0 / tw : 0.0;
    const double d0[3] = {ro.x - rs.x, ro.y - rs.y, ro.z - rs.z};
    for (int c = 0; c < 3; ++c) g[c] = c_add(g[c], c_scale(ga[c], inv));
    pair_grad(d0, k, mi, pi, mj, pj, -1.0, g, sTab);
  }
  // plane wave: i k dhat_c (mu_i . E_i - conj(E_i) . p_i)
  const double2 Ei[3] = {E[3 * i], E[3 * i + 1], E[3 * i + 2]};
  double2 q = c_dot3(mi, Ei);
  for (int a = 0; a < 3; ++a) {
    q.x -= Ei[a].x * pi[a].x + Ei[a].y * pi[a].y;
    q.y -= Ei[a].x * pi[a].y - Ei[a].y * pi[a].x;
  }
  const double dh[3] = {dx, dy, dz};
  for (int c = 0; c < 3; ++c) {
    const double2 inc = make_double2(-k * dh[c] * q.y, k * dh[c] * q.x);
    grad_r[3 * (size_t)i + c] = scale * (g[c].y + inc.y);
  }
  if (grad_eps) {
    double2 f = make_double2(0.0, 0.0);
    if (dinv) {
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
          f = c_add(f, cmul(mi[a], cmul(dinv[(size_t)(3 * a + b) * n + i], pi[b])));
    }
    // df/d eps = -mu^T D p
    grad_eps[2 * (size_t)i] = -scale * f.y;      // d C_ext / d Re(eps_i)
    grad_eps[2 * (size_t)i + 1] = -scale * f.x;  // d C_ext / d Im(eps_i)
  }
}

// E_i = amp e exp(i k dhat . r_i) with a complex polarisation e; Ec = conj(E).
__global__ void grad_incident(int n, const double4* __restrict__ pos, double k, double dx,
                              double dy, double dz, double2 e0, double2 e1, double2 e2,
                              double2* __restrict__ E, double2* __restrict__ Ec) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 r = pos[i];
  const double kdotr = k * (dx * r.x + dy * r.y + dz * r.z);
  double sn, cs;
  sincos(kdotr, &sn, &cs);
  const double2 ph = make_double2(cs, sn);
  const double2 e[3] = {e0, e1, e2};
  for (int a = 0; a < 3; ++a) {
    const double2 v = cmul(e[a], ph);
    E[3 * (size_t)i + a] = v;
    Ec[3 * (size_t)i + a] = make_double2(v.x, -v.y);
  }
}

}  // namespace
}  // namespace lum

using namespace lum;

int lum_grad_cext(lum_session* s, const double direction[3], const double polarisation[6],
                  double amplitude, const double* dinv_alpha_deps, double tol, int max_iter,
                  int restart, int mode, double* c_ext, double* moments, double* grad_r,
                  double* grad_eps, lum_solve_info* info_fwd, lum_solve_info* info_adj) {
  if (!s || !direction || !polarisation || !grad_r) {
    set_error("null pointer passed to lum_grad_cext");
    return LUM_ERR_INVALID;
  }
  OtfOperator& op = s->otf;
  if (s->kind != 0 || !op.pos64.p) {
    set_error("lum_grad_cext needs an on-the-fly session");
    return LUM_ERR_INVALID;
  }
  if (op.has_lattice || op.has_substrate) {
    set_error("lum_grad_cext covers isolated systems (no lattice, no substrate)");
    return LUM_ERR_INVALID;
  }
  if (!(amplitude > 0.0) || !std::isfinite(amplitude)) {
    set_error("invalid amplitude");
    return LUM_ERR_INVALID;
  }
  for (int q = 0; q < 3; ++q)
    if (!std::isfinite(direction[q])) {
      set_error("invalid direction");
      return LUM_ERR_INVALID;
    }
  for (int q = 0; q < 6; ++q)
    if (!std::isfinite(polarisation[q])) {
      set_error("invalid polarisation");
      return LUM_ERR_INVALID;
    }
  cudaSetDevice(s->ctx->device);
  LUM_TRY(sincos_table_ready());
  cudaStream_t st = s->stream;
  const int n = op.n;
  const size_t len = 3 * (size_t)n;
  // workspaces kept by the session: no allocation once they have grown
  auto grow = [](DevBuf& b, size_t bytes) { return b.bytes >= bytes ? LUM_OK : b.alloc(bytes); };
  DevBuf &E = s->gE, &Ec = s->gEc, &P = s->gP, &Mu = s->gMu, &part = s->gPart,
         &dinv = s->gDinv, &gr = s->gR, &ge = s->gEps;
  LUM_TRY(grow(E, sizeof(double2) * len));
  LUM_TRY(grow(Ec, sizeof(double2) * len));
  LUM_TRY(grow(P, sizeof(double2) * len));
  LUM_TRY(grow(Mu, sizeof(double2) * len));
  LUM_TRY(grow(gr, sizeof(double) * len));
  if (grad_eps) LUM_TRY(grow(ge, sizeof(double) * 2 * (size_t)n));
  if (dinv_alpha_deps) {
    std::vector<double> h(18 * (size_t)n);
    for (int i = 0; i < n; ++i)
      for (int e = 0; e < 9; ++e) {
        h[2 * ((size_t)e * n + i)] = dinv_alpha_deps[18 * (size_t)i + 2 * e];
        h[2 * ((size_t)e * n + i) + 1] = dinv_alpha_deps[18 * (size_t)i + 2 * e + 1];
      }
    LUM_TRY(grow(dinv, sizeof(double) * h.size()));
    LUM_TRY_CUDA(cudaMemcpyAsync(dinv.p, h.data(), sizeof(double) * h.size(),
                                 cudaMemcpyHostToDevice, st));
    LUM_TRY_CUDA(cudaStreamSynchronize(st));  // h is freed on scope exit
  }
  const double2 e0 = make_double2(amplitude * polarisation[0], amplitude * polarisation[1]);
  const double2 e1 = make_double2(amplitude * polarisation[2], amplitude * polarisation[3]);
  const double2 e2 = make_double2(amplitude * polarisation[4], amplitude * polarisation[5]);
  grad_incident<<<(n + 255) / 256, 256, 0, st>>>(n, op.pos64.as<double4>(), op.k, direction[0],
                                                 direction[1], direction[2], e0, e1, e2,
                                                 E.as<double2>(), Ec.as<double2>());
  LUM_CHECK_LAUNCH();
  // forward and adjoint solves in lockstep: every operator application
  // serves both right-hand sides
  lum_solve_info inf[2] = {};
  const double2* bb[2] = {E.as<double2>(), Ec.as<double2>()};
  double2* xx[2] = {P.as<double2>(), Mu.as<double2>()};
  lum_status rs = lum_gmres_device_multi(s, 2, bb, xx, tol, max_iter, restart, mode, inf, st);
  if (info_fwd) *info_fwd = inf[0];
  if (info_adj) *info_adj = inf[1];
  if (rs != LUM_OK) return rs;
  // pair pass: split the sources until the grid covers the SMs twice
  const int tiles = (n + kGradBlock - 1) / kGradBlock;
  const int sms = s->ctx->sms > 0 ? s->ctx->sms : 148;
  int ns = std::max(1, std::min(32, (4 * sms + tiles - 1) / tiles));
  const int chunk = ((tiles + ns - 1) / ns) * kGradBlock;
  ns = (n + chunk - 1) / chunk;
  LUM_TRY(grow(part, sizeof(double2) * (size_t)ns * len));
  grad_pairs<<<dim3(tiles, ns), kGradBlock, 0, st>>>(n, op.pos64.as<double4>(), P.as<double2>(),
                                                     Mu.as<double2>(), op.k, chunk,
                                                     part.as<double2>());
  LUM_CHECK_LAUNCH();
  const double scale = op.k / (amplitude * amplitude);
  grad_finish<<<(n + 127) / 128, 128, 0, st>>>(
      n, op.pos64.as<double4>(), P.as<double2>(), Mu.as<double2>(), E.as<double2>(), op.k,
      direction[0], direction[1], direction[2], part.as<double2>(), ns,
      op.use_fcd ? op.ell_w : 0, op.near_j.as<int>(), op.cell,
      dinv_alpha_deps ? dinv.as<double2>() : nullptr, scale,
      gr.as<double>(), grad_eps ? ge.as<double>() : nullptr);
  LUM_CHECK_LAUNCH();
  std::vector<double> hp(2 * len), he(2 * len);
  // exact sizes: the session's workspaces may be larger than this system
  LUM_TRY_CUDA(cudaMemcpyAsync(hp.data(), P.p, sizeof(double2) * len, cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaMemcpyAsync(he.data(), E.p, sizeof(double2) * len, cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaMemcpyAsync(grad_r, gr.p, sizeof(double) * len, cudaMemcpyDeviceToHost, st));
  if (grad_eps)
    LUM_TRY_CUDA(cudaMemcpyAsync(grad_eps, ge.p, sizeof(double) * 2 * (size_t)n,
                                 cudaMemcpyDeviceToHost, st));
  LUM_TRY_CUDA(cudaStreamSynchronize(st));
  // C_ext = k/|E0|^2 sum Im(conj(E) . p)  (cda/mod.rs:196-203)
  double acc = 0.0;
  for (size_t q = 0; q < len; ++q) acc += he[2 * q] * hp[2 * q + 1] - he[2 * q + 1] * hp[2 * q];
  if (c_ext) *c_ext = scale * acc;
  if (moments) std::copy(hp.begin(), hp.end(), moments);
  return LUM_OK;
}
