// lumina_internal.cuh -- shared declarations of the sm_100a CDA library.
//
// Device data layout (HBM):
//   * complex vectors (3N entries) are interleaved double2/float2, entry 3*i+c
//     holds component c of dipole i -- the same order as the reference's
//     Array1<Complex64> (assembly.rs:178-194);
//   * dipole positions are stored twice: double4 (x, y, z, 0) for the FP64
//     kernels, and a centred FP32 hi/lo pair (float4 each) for the FP32
//     kernels, so an FP32 displacement keeps ~1 ulp of its own magnitude;
//   * per-dipole 3x3 blocks (alpha^-1) are stored element-major [9][N] so a
//     warp reading one element of 32 consecutive dipoles is coalesced;
//   * the FCD near-pair corrections are an ELL table [W][N] of source
//     indices and [W][9][N] complex tensors (W = max near pairs per dipole).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>
#include <atomic>
#include <memory>
#include <mutex>

#include "../../include/lumina_b200.h"

namespace lum {

constexpr double kPi = 3.14159265358979323846;
constexpr int kMaxRestart = 64;

// --- error plumbing --------------------------------------------------------
void set_error(const char* fmt, ...);
lum_status cuda_status(cudaError_t e, const char* what, const char* file, int line);
extern std::atomic<uint64_t> g_launches;

#define LUM_TRY_CUDA(call)                                                  \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess) return ::lum::cuda_status(e_, #call, __FILE__, __LINE__); \
  } while (0)

#define LUM_CHECK_LAUNCH()                                                  \
  do {                                                                      \
    ::lum::g_launches.fetch_add(1, std::memory_order_relaxed);              \
    cudaError_t e_ = cudaGetLastError();                                    \
    if (e_ != cudaSuccess) return ::lum::cuda_status(e_, "kernel launch", __FILE__, __LINE__); \
  } while (0)

#define LUM_TRY(expr)                 \
  do {                                \
    lum_status s_ = (expr);           \
    if (s_ != LUM_OK) return s_;      \
  } while (0)

// --- device buffer ---------------------------------------------------------
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  lum_status alloc(size_t nbytes);   // frees the old buffer first; zero-size ok
  template <typename T> T* as() const { return reinterpret_cast<T*>(p); }
};

// --- physics configuration on the device ----------------------------------
struct LatticeDev {
  int is_2d;
  double eta;
  int n_real;          // number of real-space lattice points
  int n_recip;         // number of reciprocal points (2D) or modes (1D)
  double area;         // cell measure: area (2D) or |a1| (1D)
  double a1[3];
  double e_hat[3];     // 1D chain axis
  double a1_len;
  long m_max;          // 1D spectral modes
};

struct SubstrateDev {
  double z_interface;
  double refl_re, refl_im;
};

// SommerfeldGreens (sommerfeld.rs:215-241) with the interface height.
struct SommDev {
  double z0;
  double k_env;
  double eps_env;
  double2 eps_sub;
  double2 k_sub;
};

// --- on-the-fly operator ----------------------------------------------------
struct OtfOperator {
  int n = 0;                // dipoles
  double k = 0.0;
  int use_fcd = 0;
  double cell = 0.0;
  int has_lattice = 0;
  int has_substrate = 0;
  lum_lattice lattice{};
  double kbloch[3] = {0, 0, 0};
  SubstrateDev substrate{};
  LatticeDev latdev{};
  double center[3] = {0, 0, 0};
  double extent = 0.0;      // bounding-box diagonal (nm)
  int fast_trig = 1;        // k*extent within the fast FP32 sincos range
  int lofree = 0;           // every centred position is exact in FP32 (lo == 0)
  int img_lofree = 0;       // same for the substrate image positions

  DevBuf pos64;             // double4[n]
  DevBuf pos_hi, pos_lo;    // float4[n] (centred)
  DevBuf img_hi, img_lo;    // float4[n] image positions (substrate), centred
  DevBuf inv_alpha;         // double2[9][n]
  int ell_w = 0;            // max near pairs per dipole
  DevBuf near_j;            // int[ell_w][n], -1 padded
  DevBuf fcd64;             // double2[ell_w][9][n]
  DevBuf fcd32;             // float2[ell_w][9][n]
  DevBuf lat_real;          // double4[n_real] real-space lattice points
  DevBuf lat_recip;         // double4[n_recip] reciprocal points
  DevBuf partial;           // scratch: FP32 or FP64 partial sums [nsplit][3n]
  int nsplit32 = 1, nsplit64 = 1;
  int f32_variant = 0;      // FP32 pair-kernel variant chosen by the tuner
  int nsplit_v[8] = {1, 1, 1, 1, 1, 1, 1, 1};
  float tuned_ms = 0.f;     // tuned FP32 pair-kernel time (ms), 0 if untuned
  // Symmetric scheme (pairs_f32_sym.cuh): each unordered pair evaluated once
  // over superblock pairs; chosen by the tuner when it is faster.
  int f32_sym = 0;          // 0: split kernel; v >= 1: symmetric build v (sym_variant_name)
  int f64_sym = 0;          // 1: the FP64 operator runs the symmetric scheme too
  int f32x2_sym = 0;        // two-vector FP32 applications: v >= 1 symmetric build v
  int sym_nb = 0, sym_nitems = 0;
  float tuned_sym_ms = 0.f;
  float tuned_f64_ms = 0.f;
  DevBuf sym_items;         // int2 [sym_nitems] superblock pairs (I <= J)
  DevBuf sym_slots;         // [sym_nb][3n] per-superblock partial sums (double2; float2 for FP32)
  DevBuf sym_slots2;        // the second vector's FP64 slots (two-vector applications)
  lum_status sym_prepare(cudaStream_t st);
  void sym_launch(int variant, const double2* x, const int* skip, cudaStream_t st);
  void sym64_launch(const double2* x, const int* skip, cudaStream_t st);
  void sym2_launch(int variant, const double2* x, const double2* x2, const int* skip,
                   const int* skip2, cudaStream_t st);
  lum_status tune_f32(cudaStream_t st);
  lum_status tune_f64(cudaStream_t st);
  std::vector<double> host_pos;  // double4 host copy (image positions are built from it)

  // Sommerfeld substrate (sommerfeld.cu): the reflected-tensor integrals
  // depend on a pair only through (rho, z_i + z_j).  On a cubic dipole
  // lattice they are tabulated once per wavelength per key
  // (da^2 + db^2, c_i + c_j) -- a table of a few MB that stays in L2 -- else
  // per unordered pair (an HBM table of n(n+1)/2 records).  Records are four
  // complex values; each application gathers them (y -= G_refl x).
  int has_somm = 0;
  int somm_stale = 0;        // the physics changed after the table was built
  SommDev somm{};
  int somm_keyed = 0;        // 1: lattice keys, 0: per unordered pair
  int somm_T = 0;            // keyed: number of height sums (2 max c + 1)
  double somm_d = 0.0;       // keyed: lattice pitch
  double somm_zlo = 0.0;     // keyed: lowest dipole height
  long long somm_records = 0;
  DevBuf somm_idx;           // keyed: int4 [n] integer lattice coordinates
  DevBuf somm_tab;           // double2 [records][4]
  DevBuf somm_tab32;         // keyed: float2 [records][4]
  lum_status somm_build(const lum_sommerfeld* s, cudaStream_t st);
  lum_status somm_apply(int precision, const double2* x, double2* y, cudaStream_t st,
                        const int* skip) const;

  // Periodic (Ewald) operator on a dipole lattice: every displacement is
  // d*(da, db, dc) with integer steps, so the periodic tensor is tabulated
  // once per unique displacement (FP64, with an FP32 copy) and the matvec
  // gathers from the table (table.cu).  Off-lattice geometries use the
  // per-pair Ewald kernel instead.
  int table_ok = 0;
  double lat_d = 0.0, lat_org[3] = {0, 0, 0};
  int tdim[3] = {0, 0, 0};   // table extent per axis: 2*(max index) + 1
  int tsdim = 0;             // image table z extent: 2*(max z index) + 1
  DevBuf lidx;               // int4[n] integer lattice coordinates
  DevBuf tab64, tab32, img64, img32;
  int nsplit_tab = 1;
  lum_status table_detect(cudaStream_t st);        // host: lattice test + lidx upload
  lum_status table_build(cudaStream_t st);         // per wavelength / Bloch vector
  lum_status table_apply(int precision, const double2* x, double2* part, cudaStream_t st,
                         const int* skip, int* nparts);

  lum_status build_geometry(const double* pos_host, int n, cudaStream_t st);
  lum_status set_physics(double k, const double* inv_alpha_host, int use_fcd, double cell,
                         const lum_lattice* lat, const double* kb, const lum_substrate* sub,
                         cudaStream_t st);
  // skip: optional device flag; when it is nonzero at kernel start every
  // kernel of this application returns at once (y is left untouched).
  lum_status apply(int precision, const double2* x, double2* y, cudaStream_t st,
                   cudaEvent_t ev0, cudaEvent_t ev1, const int* skip = nullptr);

  // Two right-hand sides at once (y = A x, y2 = A x2) with one skip flag
  // each: the dense pair kernels evaluate each tensor once for both vectors.
  DevBuf partial2;             // partial sums of the second vector
  int f32x2_variant = -1;      // tuned two-vector FP32 variant (-1: not yet tuned)
  int nsplit_x2 = 1;
  float tuned_x2_ms = 0.f;
  lum_status tune_f32_x2(cudaStream_t st);
  lum_status apply2(int precision, const double2* x, const double2* x2, double2* y, double2* y2,
                    cudaStream_t st, cudaEvent_t ev0, cudaEvent_t ev1, const int* skip,
                    const int* skip2);
};

// --- cached (dense matrix) operator ----------------------------------------
// Workspace of the tensor-core product (cgemm_tc.cu): the right-hand sides
// split into TF32 hi/lo operands, split-K partial sums, the TMA maps and a
// device status word.
struct TcWork {
  DevBuf bhi, blo;          // float [npad][2 ld] each (K-major B operand)
  DevBuf part;              // float2 [ksplit][nrhs][dim] split-K partials
  DevBuf status;            // int: nonzero after a pipeline wait gave up
  int npad = 0;             // rows of bhi/blo the TMA maps describe
  size_t part_bytes = 0;
  const void* mapped_a = nullptr;
  alignas(64) unsigned char map_a[128];
  alignas(64) unsigned char map_bhi[128];
  alignas(64) unsigned char map_blo[128];
  void release() {
    bhi.release();
    blo.release();
    part.release();
    npad = 0;
    part_bytes = 0;
    mapped_a = nullptr;
  }
};

// Right-hand sides from which the automatic method takes the tensor cores.
constexpr int kTcMinRhs = 4;

// Symmetric tile storage of a cached matrix: tiles of kSymTile x kSymTile
// complex entries (kSymTile / 3 dipoles a side, so no 3x3 dipole block
// straddles two tiles); only the tiles (I, J) with I <= J are stored.
constexpr int kSymTile = 192;

struct CachedOperator {
  int dim = 0;              // 3N
  size_t ld = 0;            // row pitch in complex entries (dim rounded up to 16)
  int precision = LUM_FP32; // storage precision of A
  DevBuf A;                 // float2 or double2 [dim][ld] row-major, zero padding
  TcWork tc;
  int gemv_chunks = 0;      // column chunks of the GEMV (0: not yet chosen)
  int gemv_chunk = 0;       // complex entries per chunk
  DevBuf gemv_part_buf;     // double2 [gemv_chunks][dim] per-chunk partial sums
  // Symmetric tile storage (A = A^T): A holds the upper-triangle tiles,
  // packed row by row, each tile row-major with zero padding past dim.
  bool packed = false;
  int nt = 0;               // tiles (blocks) per side, ceil(dim / kSymTile)
  DevBuf tile_items;        // int2 (I, J) per tile product block
  DevBuf tile_part;         // double2 [nt][dim]: slot S, row r (see cached.cu)
  lum_status allocate(int dim, int precision, bool packed = false);
  lum_status tile_blocks(bool upper);
  lum_status upload(const double* host, cudaStream_t st);
  lum_status assemble(const OtfOperator& geo, cudaStream_t st);
  lum_status apply(const double2* x, double2* y, cudaStream_t st, const int* skip = nullptr);
  // Y = A X; element (c, r) of X and Y at [c * sc + r * sr].
  lum_status apply_multi(const double2* X, double2* Y, int nrhs, long long sc, long long sr,
                         int method, cudaStream_t st);
  lum_status apply_multi_cuda_cores(const double2* X, double2* Y, int nrhs, long long sc,
                                    long long sr, cudaStream_t st);
};

// Tensor-core product Y = A X of an FP32-storage cached matrix (cgemm_tc.cu).
lum_status cgemm_tf32x3(CachedOperator& op, const double2* X, long long sxc, long long sxr,
                        double2* Y, long long syc, long long syr, int nrhs, cudaStream_t st);
// LUM_ERR_TIMEOUT when a pipeline wait of an earlier product gave up (and
// clears the record); synchronises `st`.
lum_status cgemm_status(CachedOperator& op, cudaStream_t st);

// --- block-Toeplitz operator through 3D FFTs (fft.cu) -----------------------
struct FftOperator {
  int n = 0;                // dipoles
  int gn[3] = {1, 1, 1};    // lattice nodes per axis (bounding box of the dipoles)
  int M[3] = {1, 1, 1};     // circulant dimensions: powers of two >= 2 gn - 1
  size_t mtot = 1;          // M[0] M[1] M[2]
  double spacing = 0.0, cell = 0.0, k = 0.0;
  int use_fcd = 0;
  size_t tw_off[3] = {0, 0, 0};
  DevBuf d_node_dip;        // int [mtot]: dipole on each node, -1 if none
  DevBuf d_grid_of;         // int [n]: node of each dipole
  DevBuf inv_alpha;         // double2 [9][n]
  DevBuf kern64, kern32;    // kernel spectra: 6 components (xx xy xz yy yz zz) x mtot
  DevBuf buf64, buf32;      // 3 vector components x mtot
  DevBuf tw64, tw32;        // twiddles exp(-2 pi i q / M[c]), q < M[c]/2, per axis
  // Substrate term: R(da, db, c_i + c_j) is a convolution in the z-mirrored
  // coordinate, applied as R^ . (m o X)(kx, ky, -kz) in the spectral product.
  int refl_mode = 0;        // 0 none, 1 Fresnel image dipole, 2 Sommerfeld
  int refl_stale = 0;       // Sommerfeld spectra of another wavelength
  double lo_z = 0.0;        // lowest lattice node height (z of c = 0)
  double2 refl_m[3] = {{1, 0}, {1, 0}, {1, 0}};  // column factors of the mirrored input
  DevBuf refl64, refl32;    // reflected spectra: 6 components x mtot
  lum_status set_reflection(int mode, const lum_substrate* fresnel, const SommDev* somm,
                            cudaStream_t st);
  lum_status build(const double* pos_host, int n, double spacing, double cell, int use_fcd,
                   cudaStream_t st);
  lum_status set_physics(double k, const double* inv_alpha_host, cudaStream_t st);
  lum_status apply(int precision, const double2* x, double2* y, cudaStream_t st,
                   cudaEvent_t ev0, cudaEvent_t ev1, const int* skip);
};

// --- GMRES workspace --------------------------------------------------------
struct GmresState {
  double2 H[(kMaxRestart + 1) * kMaxRestart];
  double cs[kMaxRestart];
  double2 sn[kMaxRestart];
  double2 g[kMaxRestart + 1];
  double2 y[kMaxRestart];
  double scal[8];   // 0: last norm, 1: h_{j+1,j}, 2: |g[j+1]|, 3: residual norm
  int done;         // the cycle has met its test: later kernels of the cycle exit at once
  int jdone;        // Arnoldi steps completed in the current cycle
  int bad;          // a non-finite residual estimate was produced
  int pad;
};

struct GmresWork {
  int len = 0;      // complex entries (3N)
  int m = 0;
  DevBuf V, w, r, tmp, partials, counter, state;
  DevBuf coop_part;                // double2 [2][nblk]: block sums of the fused step kernel
  GmresState* h_state = nullptr;   // pinned mirror of a few scalars
  int nblk = 0;
  lum_status ensure(int len, int m, cudaStream_t st);
  ~GmresWork();
};

// --- batched systems (batch.cu + the batched kernels in otf.cu) ------------
// Per-system control flags of a batched solve: `done` ends the system's
// current restart cycle, `frozen` removes it from all further work.
struct BatchFlags {
  int done;
  int frozen;
  int jdone;
  int bad;
};

// Device view of K systems concatenated into one dipole range [0, N): system
// s owns dipoles [sys_off[s], sys_off[s+1]).  Vectors are 3N complex, and the
// per-dipole arrays (positions, alpha^-1, near lists) are indexed globally.
// FP32 positions are centred per system.
struct BatchGeom {
  int K = 0, N = 0;
  int ell_w = 0;
  int lofree = 0, fast = 1;
  int minb32 = 4;                      // FP32 pair kernel: CTAs per SM it is built for (4 or 6)
  int sym32 = 0;                       // FP32: v >= 1 runs symmetric build v (batch_sym_name)
  const int* sys_nb = nullptr;         // [K] superblocks of each system (symmetric scheme)
  const struct BatchQueue* qsym = nullptr;  // symmetric work list
  int nparts32 = 1, nparts64 = 1;      // partial slices (max splits of any system)
  const int* sys_off = nullptr;        // [K+1]
  const int* row_sys = nullptr;        // [N]
  const int* sys_ns32 = nullptr;       // [K] source splits of each system (FP32 items)
  const int* sys_ns64 = nullptr;       // [K]
  const int* sys_chunk32 = nullptr;    // [K] sources per split (multiple of 128)
  const int* sys_chunk64 = nullptr;    // [K]
  const double* sys_k = nullptr;       // [K]
  const double* sys_cell = nullptr;    // [K]
  const double4* pos64 = nullptr;
  const float4 *hi = nullptr, *lo = nullptr;
  const double2* inv_alpha = nullptr;  // [9][N]
  const int* near_j = nullptr;         // [W][N] global source indices, -1 padded
  const double2* fcd64 = nullptr;      // [W][9][N]
  const float2* fcd32 = nullptr;
};

// A pair-kernel work list: int4 items (system, first row, split, 0), ordered
// by decreasing cost, consumed by a persistent grid through an atomic
// counter (the last CTA to leave resets it, so the list can be replayed).
struct BatchQueue {
  DevBuf items;
  int nitems = 0;
  int grid = 0;
  DevBuf counters;   // unsigned[2]: next item, CTAs finished
};

// skip_mode: 0 apply to every system, 1 skip systems whose cycle is done or
// that are frozen, 2 skip frozen systems only.
lum_status batch_near_fcd(BatchGeom& g, int use_fcd, DevBuf& near_j, DevBuf& fcd64,
                          DevBuf& fcd32, cudaStream_t st);                           // otf.cu
lum_status batch_queue(int precision, const std::vector<int>& off, int slots, BatchQueue& q,
                       std::vector<int>& ns, std::vector<int>& chunk,
                       cudaStream_t st);                                             // otf.cu
lum_status batch_apply(const BatchGeom& g, int precision, const double2* x, double2* y,
                       void* partial, BatchQueue& q, const BatchFlags* flags, int skip_mode,
                       cudaStream_t st);                                             // otf.cu
int batch_occupancy(const BatchGeom& g, int precision);                              // otf.cu
// Rows (and sources) of a superblock of the symmetric scheme; a system of n
// dipoles has ceil(n / kBatchSymRows) superblocks and nb (nb + 1) / 2 items.
constexpr int kBatchSymRows = 512;
lum_status otf_sincos_ready();  // otf.cu: its FP64 pair kernels' sin / cos table
lum_status batch_queue_sym(const std::vector<int>& off, int slots, BatchQueue& q,
                           std::vector<int>& nb, cudaStream_t st);                   // otf.cu
int batch_sym_variants();                                                            // otf.cu
const char* batch_sym_name(int v);                                                   // otf.cu
int batch_sym_occupancy(const BatchGeom& g, int v);                                  // otf.cu

const char* f32_variant_name(int v);    // otf.cu
const char* f32x2_variant_name(int v);  // otf.cu
const char* sym_variant_name(int v);    // otf.cu (1-based; "none" for 0)
const char* sym2_variant_name(int v);   // otf.cu (1-based; "none" for 0)
// Persistent tuner choices (tune_cache.cu).
std::string tune_device_tag();
bool tune_lookup(const std::string& key, int* value);
void tune_store(const std::string& key, int value);
lum_status somm_assemble(const OtfOperator& g, int precision, void* A, size_t ld,
                         cudaStream_t st);
lum_status somm_params(const lum_sommerfeld* s, SommDev* out);
lum_status assemble_from_table(const OtfOperator& g, int precision, void* A, size_t ld,
                               cudaStream_t st);  // table.cu

// vector kernels (gmres.cu)
lum_status vec_norm(const double2* v, int len, GmresWork& W, int slot, cudaStream_t st);
lum_status read_scalars(GmresWork& W, cudaStream_t st);

}  // namespace lum

// Session (opaque to callers).
namespace lum {
// Workspaces of a context's own entry points (the fields of fields.cu, the
// harmonic sources of harmonic.cu): one stream and buffers that grow on
// demand, used by one caller at a time (hold mu).
struct FieldWork {
  std::mutex mu;
  cudaStream_t stream = nullptr;
  DevBuf pos, mom, obs, part, field, inten, th, ph;
  DevBuf h_e, h_chi, h_p;
  ~FieldWork() {
    if (stream) cudaStreamDestroy(stream);
  }
};
}  // namespace lum

struct lum_ctx {
  int device = 0;
  std::string name;
  size_t mem_bytes = 0;
  int sms = 0;
  std::unique_ptr<lum::FieldWork> fields;  // created by the first call that needs it
};

namespace lum {
// The context's workspace, created on first use (fields.cu); the caller has
// made the context's device current.
lum_status ctx_work(lum_ctx* ctx, FieldWork** out);
}  // namespace lum

struct lum_session {
  lum_ctx* ctx = nullptr;
  int kind = 0;                 // 0 on-the-fly, 1 cached, 2 FFT (lattice)
  int n_dipoles = 0;
  int dim = 0;                  // 3N
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  lum::OtfOperator otf;
  lum::CachedOperator cached;
  lum::FftOperator fft;
  lum::GmresWork gw;
  lum::DevBuf xbuf, ybuf, bbuf; // host-path staging
  // profiling of the dominant kernel
  bool profile = false;
  struct EvRec {
    cudaEvent_t a, b;
    int precision;
  };
  std::vector<EvRec> ev_pool;
  size_t ev_used = 0;
  lum_status apply(int precision, const double2* x, double2* y, const int* skip = nullptr);
  lum_status apply2(int precision, const double2* x, const double2* x2, double2* y, double2* y2,
                    const int* skip, const int* skip2);
  lum::GmresWork gw2;           // workspace of the second right-hand side
  // lum_grad_cext workspaces (incident field and its conjugate, forward and
  // adjoint solutions, pair partials, d alpha^-1 / d eps, outputs); they
  // grow on demand and live with the session
  lum::DevBuf gE, gEc, gP, gMu, gPart, gDinv, gR, gEps;
};

// Device GMRES drivers (gmres.cu): one right-hand side, or one or two in
// lockstep sharing every operator application.
lum_status lum_gmres_device(lum_session* s, const double2* b, double2* x, double tol,
                            int max_iter, int restart, int mode, lum_solve_info* info,
                            cudaStream_t st);
lum_status lum_gmres_device_multi(lum_session* s, int nrhs, const double2* const* b,
                                  double2* const* x, double tol, int max_iter, int restart,
                                  int mode, lum_solve_info* info, cudaStream_t st);
