/* lumina_b200.h -- C ABI of the B200 (sm_100a) coupled-dipole solve library.
 *
 * This is the drop-in boundary for the reference's compute backend
 * (crates/lumina-compute/src/backend.rs) and the two solver hooks its
 * on-the-fly path lacks.  Plain pointers and sizes only; every function
 * returns a lum_status and never aborts across the ABI.
 *
 * Conventions
 *  - complex arrays are interleaved (re, im) doubles, the memory layout of
 *    ndarray's Array1<Complex64> / Array2<Complex64> (row-major);
 *  - a vector of the CDA system has 3N complex entries, entry 3*i+c holding
 *    component c of dipole i (assembly.rs:178-194);
 *  - positions are N*3 doubles in nm; alpha^-1 / alpha blocks are N*9
 *    complex, row-major 3x3 per dipole (types.rs:12-18);
 *  - "_device" variants take device pointers and an optional cudaStream_t
 *    (passed as void*; NULL = the session's stream).
 */
#ifndef LUMINA_B200_H
#define LUMINA_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define LUM_API __attribute__((visibility("default")))
#else
#define LUM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  Map onto ComputeError (backend.rs:13-22) and SolverError
 * (solver/mod.rs:18-30):
 *   UNAVAILABLE -> ComputeError::Unavailable, DEVICE -> DeviceError,
 *   OOM -> OutOfMemory, NOT_CONVERGED -> SolverError::ConvergenceFailure,
 *   INVALID -> SolverError::InvalidGeometry / LinAlgError. */
typedef enum {
  LUM_OK = 0,
  LUM_ERR_UNAVAILABLE = 1,
  LUM_ERR_DEVICE = 2,
  LUM_ERR_OOM = 3,
  LUM_ERR_NOT_CONVERGED = 4,
  LUM_ERR_TIMEOUT = 5,
  LUM_ERR_INVALID = 6
} lum_status;

/* Arithmetic of a matvec / matrix storage. */
enum { LUM_FP64 = 0, LUM_FP32 = 1 };
/* OR-ed into lum_session_assemble's storage precision: keep only the upper
 * triangle of the matrix, as tiles of 192 x 192 entries (64 dipoles a side),
 * for a free-space system, whose matrix is complex symmetric.  Half the
 * device memory and half the bytes per product of dense rows.  No
 * counterpart in the reference, which stores dense rows (gpu.rs:303-399). */
enum { LUM_STORAGE_SYMMETRIC = 0x10 };

/* Solve modes of lum_solve_gmres. */
enum {
  LUM_SOLVE_FP64 = 0,        /* plain FP64 GMRES(m): Arnoldi and matvecs in FP64 */
  LUM_SOLVE_FP32_REFINE = 1  /* FP32 matvecs inside FP64 Arnoldi/Givens, every
                                restart residual r = b - A x in FP64 */
};

typedef struct lum_ctx lum_ctx;
typedef struct lum_session lum_session;

/* LatticeSpec (crates/lumina-geometry/src/lattice.rs:29-44). is_2d=0 is a
 * 1D chain along a1 (a2 ignored).  has_eta=0 selects eta = sqrt(pi/A). */
typedef struct {
  double a1[3];
  double a2[3];
  int is_2d;
  int has_eta;
  double eta;
  int truncation_real;
  int truncation_recip;
} lum_lattice;

/* SubstrateRuntime::Fresnel (solver/substrate.rs:103-107): interface plane
 * and the scalar reflection factor (quasi-static delta-eps or retarded r). */
typedef struct {
  double z_interface;
  double refl_re;
  double refl_im;
} lum_substrate;

/* SubstrateRuntime::Sommerfeld (solver/substrate.rs:109-113, built by
 * from_spec at :126-130 as SommerfeldGreens::new(wavelength_nm, eps_sub,
 * eps_env), sommerfeld.rs:236-241): the full reflected Green's tensor by the
 * Sommerfeld integral over k_par. */
typedef struct {
  double z_interface;
  double wavelength_nm;
  double eps_sub_re;
  double eps_sub_im;
  double eps_env;
} lum_sommerfeld;

typedef struct {
  int iterations;          /* Arnoldi steps, counted as iterative.rs:129 does */
  int restarts;            /* restart cycles completed */
  int matvecs_fp64;        /* FP64 operator applications */
  int matvecs_fp32;        /* FP32 operator applications */
  int matvecs_reference;   /* matvecs the reference loop would have issued
                              (it recomputes the cycle-start residual) */
  int converged;
  double rel_residual;     /* final true residual / ||b||, FP64 */
  double seconds;          /* wall time of the solve */
} lum_solve_info;

/* ---- context ------------------------------------------------------------ */
/* Creates a context on CUDA device `device`; fails with UNAVAILABLE when no
 * sm_100 device exists.  Replaces GpuBackend::new_blocking (gpu.rs:115-290). */
LUM_API int lum_ctx_create(int device, lum_ctx** out);
LUM_API int lum_ctx_destroy(lum_ctx* ctx);
/* ComputeBackend::device_info (backend.rs:64, gpu.rs:493-500). */
LUM_API int lum_device_info(lum_ctx* ctx, char* name, size_t name_len, size_t* memory_bytes,
                    int* compute_units);
/* Message of the last failing call on this thread (never NULL). */
LUM_API const char* lum_last_error(void);
/* The sizes behind the last LUM_ERR_OOM on this thread, for
 * ComputeError::OutOfMemory { requested, available } (backend.rs:13-22):
 * the bytes the failed allocation asked for (0 when a CUDA call other than
 * an allocation ran out) and the device's free bytes at that moment. */
LUM_API int lum_last_oom(size_t* requested, size_t* available);
/* Kernels this library has launched since load (all threads). */
LUM_API uint64_t lum_launch_count(void);

/* ---- host-side inputs (types.rs, assembly.rs) ---------------------------- */
/* compute_diagonal_blocks / invert_3x3 (assembly.rs:325-363): alpha^-1 per
 * dipole; INVALID when |det| <= 1e-30 (the reference panics there). */
LUM_API int lum_invert_polarisability(int n_dipoles, const double* alpha, double* inv_alpha);
/* build_incident_field_vector + IncidentField::at_position
 * (assembly.rs:178-194, types.rs:60-73). */
LUM_API int lum_incident_field(int n_dipoles, const double* pos, const double direction[3],
                       const double polarisation[3], double amplitude, double k,
                       double* rhs);
/* OpticalSolver::compute_cross_sections (cda/mod.rs:175-236) from solved
 * moments: out[0]=C_ext, out[1]=C_abs, out[2]=max(C_ext-C_abs,0). */
LUM_API int lum_cross_sections(int n_dipoles, const double* pos, const double* inv_alpha,
                       const double* moments, double k, const double direction[3],
                       const double polarisation[3], double amplitude, double out[3]);

/* ---- sessions (MatvecSession, backend.rs:47-55) -------------------------- */
/* ComputeBackend::create_session(n) (backend.rs:70-72, gpu.rs:303-399):
 * a cached-matrix session of dimension dim=3N, storage LUM_FP32 or LUM_FP64. */
LUM_API int lum_session_create_cached(lum_ctx* ctx, int dim, int storage_precision,
                              lum_session** out);
/* MatvecSession::upload_matrix (backend.rs:51, gpu.rs:410-421). */
LUM_API int lum_session_upload_matrix(lum_session* s, const double* A);
/* ComputeBackend::assemble_and_create_session (backend.rs:109-117,
 * gpu.rs:502-610), widened to the FCD / lattice / substrate terms of
 * assemble_interaction_matrix (assembly.rs:45-175): the whole 3N x 3N matrix
 * is built on the device.  inv_alpha = compute_diagonal_blocks output.
 * storage_precision | LUM_STORAGE_SYMMETRIC stores the upper-triangle tiles
 * only; INVALID with a lattice sum (which is not symmetric) or a substrate
 * (the tile assembly covers free space only).
 * Such a session applies its matrix one vector per product: a tensor-core
 * product, or a lum_session_matmul_device of more than one vector, returns
 * INVALID, and lum_session_matmul_vectors and the right-hand-side batches
 * run one tile product per vector. */
LUM_API int lum_session_assemble(lum_ctx* ctx, int n_dipoles, const double* pos,
                         const double* inv_alpha, double k, int use_fcd, double cell_size,
                         const lum_lattice* lattice, const double k_bloch[3],
                         const lum_substrate* substrate, int storage_precision,
                         lum_session** out);
/* New backend hook (the reference's on-the-fly path bypasses the backend,
 * cda/mod.rs:329-344 and :375-390): a matrix-free session whose matvec is
 * matvec_on_the_fly (assembly.rs:209-318).  O(N) device memory. */
LUM_API int lum_session_create_onthefly(lum_ctx* ctx, int n_dipoles, const double* pos,
                                const double* inv_alpha, double k, int use_fcd,
                                double cell_size, const lum_lattice* lattice,
                                const double k_bloch[3], const lum_substrate* substrate,
                                lum_session** out);
/* The reference's FftMatvecPlan (crates/lumina-core/src/solver/cda/
 * fft_matvec.rs:77-258, chosen at cda/mod.rs:286-298) as a session: A x by a
 * circulant-embedded 3D FFT convolution, O(N log N), FP64 or FP32.  Widened
 * to FCD (the filtered tensor is a function of the displacement too, so the
 * product equals the on-the-fly FCD operator) and to any set of nodes of a
 * cubic lattice (empty nodes hold zero), not only a full box.  `spacing` is
 * the lattice pitch (<= 0: cell_size, as detect_regular_grid takes it,
 * fft_matvec.rs:19); every dipole must lie within 1e-6 spacing of a node,
 * at most 512 nodes per axis, no lattice sum.  The session supports matvec,
 * the solves and set_wavelength.  A planar substrate is added as a second
 * convolution in the z-mirrored coordinate (six more spectra, no further FFT
 * per product): the Fresnel image term through lum_session_set_wavelength's
 * substrate argument, the Sommerfeld term through lum_session_set_sommerfeld.
 * Neither is in the reference's FFT plan, which declines substrates
 * (cda/mod.rs:286-298). */
LUM_API int lum_session_create_fft(lum_ctx* ctx, int n_dipoles, const double* pos,
                                   const double* inv_alpha, double k, int use_fcd,
                                   double cell_size, double spacing, lum_session** out);
/* Re-targets a session to a new wavelength (k, alpha^-1, Fresnel substrate
 * factor or NULL) keeping the geometry, near-pair list and buffers (the
 * runner's per-wavelength loop, runner.rs:150-183): an on-the-fly session
 * rebuilds its wavelength tables, an assembled session re-assembles its
 * matrix, an FFT session rebuilds its kernel (and reflected) spectra.  A
 * session with a Sommerfeld term keeps it stale -- its applications fail
 * with INVALID -- until lum_session_set_sommerfeld gives this wavelength's
 * substrate. */
LUM_API int lum_session_set_wavelength(lum_session* s, double k, const double* inv_alpha,
                               const lum_substrate* substrate);
/* The Sommerfeld substrate runtime in the sessions.  Replaces the
 * SubstrateRuntime::Sommerfeld arms of assemble_interaction_matrix
 * (assembly.rs:157-166) and matvec_on_the_fly (assembly.rs:296-303): every
 * block (i, j), i == j included, gets -G_refl(r_i, r_j).  The integrals of
 * each unordered pair are evaluated once on the device into a table of
 * 32 N(N+1) bytes (N <= 65535), which the on-the-fly application streams and
 * the dense assembly folds into the matrix.  Arguments as
 * lum_session_assemble / lum_session_create_onthefly with `somm` in place of
 * the Fresnel substrate. */
LUM_API int lum_session_assemble_sommerfeld(lum_ctx* ctx, int n_dipoles, const double* pos,
                                            const double* inv_alpha, double k, int use_fcd,
                                            double cell_size, const lum_lattice* lattice,
                                            const double k_bloch[3], const lum_sommerfeld* somm,
                                            int storage_precision, lum_session** out);
LUM_API int lum_session_create_onthefly_sommerfeld(lum_ctx* ctx, int n_dipoles,
                                                   const double* pos, const double* inv_alpha,
                                                   double k, int use_fcd, double cell_size,
                                                   const lum_lattice* lattice,
                                                   const double k_bloch[3],
                                                   const lum_sommerfeld* somm,
                                                   lum_session** out);
/* Rebuilds the Sommerfeld table of an on-the-fly session for new substrate
 * parameters (after lum_session_set_wavelength, which marks the table stale:
 * until it is rebuilt the session's applications fail with INVALID),
 * re-assembles a cached session's matrix with them, or builds an FFT
 * session's reflected spectra. */
LUM_API int lum_session_set_sommerfeld(lum_session* s, const lum_sommerfeld* somm);
/* SommerfeldGreens::evaluate (sommerfeld.rs:254-300) on the device for
 * npairs point pairs: ri, rj are npairs x 3, g receives npairs x 3 x 3
 * interleaved complex values. */
LUM_API int lum_sommerfeld_tensor(lum_ctx* ctx, const lum_sommerfeld* somm, int npairs,
                                  const double* ri, const double* rj, double* g);
/* MatvecSession::matvec (backend.rs:54, gpu.rs:428-488) on host vectors,
 * precision LUM_FP64 or LUM_FP32 (FP32 arithmetic, FP64 in/out). */
LUM_API int lum_session_matvec(lum_session* s, int precision, const double* x, double* y);
LUM_API int lum_session_matvec_device(lum_session* s, int precision, const void* x_dev, void* y_dev,
                              void* stream);
/* Multi-RHS cached matvec Y = A X, X and Y row-major dim x nrhs (device).
 * Method as LUM_MATMUL_AUTO below.  Asynchronous: a tensor-core pipeline
 * wait that gave up is reported as TIMEOUT by the session's next
 * synchronising product (lum_session_matmul_vectors, lum_batch_matvec,
 * lum_batch_solve). */
LUM_API int lum_session_matmul_device(lum_session* s, const void* X_dev, void* Y_dev, int nrhs,
                              void* stream);
/* Methods of a multi-RHS cached product.  TENSOR runs on the tensor cores
 * (tcgen05, TF32 operands split hi + lo, three products per pair: about FP32
 * accuracy) and needs FP32 matrix storage; CUDA_CORES streams the matrix once
 * per 8 vectors with FP64 accumulation; AUTO takes TENSOR for FP32 storage
 * and nrhs >= 4. */
enum { LUM_MATMUL_AUTO = 0, LUM_MATMUL_TENSOR = 1, LUM_MATMUL_CUDA_CORES = 2 };
/* No single counterpart in the reference, which applies the cached matrix
 * one vector per MatvecSession::matvec call (backend.rs:54, gpu.rs:428-488):
 * Y = A X for nrhs vectors stored back to back (vector r at 3N*r complex,
 * the layout of lum_solve_gmres_multi).  The device variant runs on `stream`
 * (NULL = the session stream) without synchronising; the host variant
 * synchronises and returns TIMEOUT if a tensor-core pipeline wait gave up. */
LUM_API int lum_session_matmul_vectors_device(lum_session* s, const void* X_dev, void* Y_dev,
                                              int nrhs, int method, void* stream);
LUM_API int lum_session_matmul_vectors(lum_session* s, const double* X, double* Y, int nrhs,
                                       int method);
/* Use the caller's stream for all later work of this session (NULL resets). */
LUM_API int lum_session_set_stream(lum_session* s, void* stream);
LUM_API int lum_session_destroy(lum_session* s);

/* ---- solve (iterative.rs:33-206; fills the dense_solve slot,
 *      backend.rs:123-133) -------------------------------------------------- */
/* Restarted GMRES(min(restart,3N)) with x0 = 0, modified Gram-Schmidt and
 * complex Givens rotations, |g| < tol*||b|| inside a cycle and the true
 * residual at its end, as iterative.rs does.  NOT_CONVERGED carries
 * info->rel_residual.  Host vectors. */
LUM_API int lum_solve_gmres(lum_session* s, const double* b, double tol, int max_iter, int restart,
                    int mode, double* x, lum_solve_info* info);
LUM_API int lum_solve_gmres_device(lum_session* s, const void* b_dev, void* x_dev, double tol,
                           int max_iter, int restart, int mode, lum_solve_info* info,
                           void* stream);

/* ---- batched systems ------------------------------------------------------ */
/* No single counterpart in the reference: its callers solve independent
 * systems (clusters, wavelengths of a sweep, polarisations) one
 * CdaSolver::solve_dipoles call at a time (cda/mod.rs:304-389, runner.rs
 * 134-148 runs one per rayon thread).  A batch holds K isolated systems of
 * uneven size, each with its own positions, alpha^-1, wave number and FCD
 * cell (no lattice, no substrate), concatenated in system order: pos is
 * 3*sum(N_s) doubles, inv_alpha 18*sum(N_s) (row-major 3x3 complex per
 * dipole, as lum_session_create_onthefly), k and cell K doubles.  Vectors
 * are 3*sum(N_s) complex in the same order.  A system may hold at most
 * 21,845 dipoles.  Duplicate a system to solve it for several right-hand
 * sides. */
typedef struct lum_batch lum_batch;
LUM_API int lum_batch_create(lum_ctx* ctx, int n_systems, const int* sys_dipoles,
                             const double* pos, const double* inv_alpha, const double* k,
                             const double* cell, int use_fcd, lum_batch** out);
/* y_s = A_s x_s for every system (host or device vectors). */
LUM_API int lum_batch_matvec(lum_batch* b, int precision, const double* x, double* y);
LUM_API int lum_batch_matvec_device(lum_batch* b, int precision, const void* x_dev, void* y_dev);
/* GMRES of lum_solve_gmres on every system at once; info has K entries.
 * Returns NOT_CONVERGED if any system did not converge (info says which),
 * DEVICE on a non-finite residual, TIMEOUT if a tensor-core product of a
 * right-hand-side batch gave up a pipeline wait (checked after every restart
 * cycle; the solution is then not written). */
LUM_API int lum_batch_solve(lum_batch* b, const double* rhs, double tol, int max_iter,
                            int restart, int mode, double* x, lum_solve_info* info);
LUM_API int lum_batch_solve_device(lum_batch* b, const void* rhs_dev, void* x_dev, double tol,
                                   int max_iter, int restart, int mode, lum_solve_info* info);
LUM_API int lum_batch_set_stream(lum_batch* b, void* stream);
/* The kernels a cluster batch runs, as "key=value" tokens: the FP32 pair
 * scheme chosen at creation (split work list or a symmetric build) and its
 * work-list sizes.  No counterpart in the reference. */
LUM_API int lum_batch_kernel_config(lum_batch* b, char* buf, size_t len);
/* No counterpart in the reference, which solves one incidence at a time
 * (cda/mod.rs:238-391): a batch of nrhs right-hand sides of one session's
 * operator (incidence directions, polarisations), solved by lum_batch_solve
 * with vectors stored back to back (vector r at 3N*r complex).  Each
 * operator application takes all nrhs vectors at once: for a cached session
 * with FP32 storage, the FP32 steps are one tensor-core product
 * (lum_session_matmul_vectors, TENSOR); otherwise the session's operator
 * runs two vectors at a time.  The FP64 restart residuals use the session's
 * FP64 operator (the on-the-fly FP64 product for a device-assembled FP32
 * matrix).  The batch borrows the session (destroy the batch first) and runs
 * on the session's stream; at most 21,845 dipoles. */
LUM_API int lum_batch_create_rhs(lum_session* s, int nrhs, lum_batch** out);
/* Launch configuration: systems, dipoles, near-list width, CTAs per system
 * cluster, vector elements per thread, pair work-list items and persistent
 * grid per precision. */
LUM_API int lum_batch_info(lum_batch* b, int* n_systems, int* n_dipoles, int* ell_width,
                           int* cluster, int* elems_per_thread, int* items32, int* grid32,
                           int* items64, int* grid64);
LUM_API int lum_batch_destroy(lum_batch* b);

/* ---- adjoint gradients --------------------------------------------------- */
/* No counterpart in the reference (it has no gradient code).  For an
 * on-the-fly session without lattice or substrate: solves A p = E for the
 * plane wave E_i = amplitude * e * exp(i k dhat . r_i) (polarisation e is 3
 * complex = 6 doubles, so circular polarisation is allowed), then the adjoint
 * A mu = conj(E) (A is complex symmetric), and returns
 *   c_ext      = k/amplitude^2 * sum Im(conj(E) . p)   (cda/mod.rs:175-236),
 *   moments    = p (3N complex; may be NULL),
 *   grad_r     = dC_ext/dr (3N doubles, dipole-major),
 *   grad_eps   = (dC_ext/dRe eps_i, dC_ext/dIm eps_i) per dipole (2N doubles;
 *                may be NULL), given dinv_alpha_deps = d(alpha_i^-1)/d eps_i
 *                per dipole (18N doubles like inv_alpha; NULL = zero).
 * The FCD near/far switch is a step: the gradient is that of the branch each
 * pair is on.  info_fwd / info_adj describe the two solves (may be NULL). */
LUM_API int lum_grad_cext(lum_session* s, const double direction[3],
                          const double polarisation[6], double amplitude,
                          const double* dinv_alpha_deps, double tol, int max_iter, int restart,
                          int mode, double* c_ext, double* moments, double* grad_r,
                          double* grad_eps, lum_solve_info* info_fwd, lum_solve_info* info_adj);

/* Several right-hand sides of one session (the nrhs argument of the proposed
 * lum_solve_gmres; the reference solves polarisations one call at a time,
 * cda/mod.rs:304-389).  b and x hold nrhs vectors of 3N complex back to back;
 * info has nrhs entries.  Right-hand sides are solved two at a time in
 * lockstep: each operator application evaluates every pair tensor once for
 * both vectors.  Each vector's GMRES is the single-vector algorithm; a
 * vector that converges first drops out.  The device variant runs on
 * `stream` (NULL = the session stream) and returns without synchronising. */
LUM_API int lum_solve_gmres_multi(lum_session* s, int nrhs, const double* b, double tol,
                                  int max_iter, int restart, int mode, double* x,
                                  lum_solve_info* info);
LUM_API int lum_solve_gmres_multi_device(lum_session* s, int nrhs, const void* b_dev,
                                         void* x_dev, double tol, int max_iter, int restart,
                                         int mode, lum_solve_info* info, void* stream);

/* ---- fields from solved moments (fields.rs) ------------------------------- */
/* The field entry points and lum_harmonic_sources keep one stream and their
 * device buffers with the context (grown on demand, freed by
 * lum_ctx_destroy); calls on one context from several threads run one at a
 * time. */
/* field_at_point (crates/lumina-core/src/fields.rs:18-49) at m observation
 * points obs (3m doubles): E = E_inc + sum_i G(r - r_i) p_i, the point-dipole
 * tensor of greens.rs:34-71, dipoles with |r - r_i|^2 < 1e-20 skipped, FP64.
 * moments: 3N complex (the solved p).  The incident field is
 * IncidentField::at_position (types.rs:60-73) with a real polarisation.
 * field (3m complex) and intensity (|E|^2, m doubles) may each be NULL.
 * n = 0 gives the incident field. */
LUM_API int lum_near_field(lum_ctx* ctx, int n_dipoles, const double* pos, const double* moments,
                           double k, const double direction[3], const double polarisation[3],
                           double amplitude, int n_obs, const double* obs, double* field,
                           double* intensity);
/* compute_near_field_map (fields.rs:52-105, plane_basis :111-139): the
 * nx x ny grid on the plane (centre, normal, half_width, half_height), row
 * iy outer and column ix inner, its |E|^2 and extent [x_min, x_max, y_min,
 * y_max].  positions: 3*nx*ny doubles (may be NULL), intensity: nx*ny. */
LUM_API int lum_near_field_map(lum_ctx* ctx, int n_dipoles, const double* pos,
                               const double* moments, double k, const double direction[3],
                               const double polarisation[3], double amplitude,
                               const double centre[3], const double normal[3], double half_width,
                               double half_height, int nx, int ny, double* positions,
                               double* intensity, double extent[4]);
/* compute_far_field (fields.rs:147-221): n_theta x n_phi directions,
 * theta = pi it / max(n_theta - 1, 1), phi = 2 pi ip / n_phi (it outer);
 * intensity |(I - r r) . F|^2 with F = sum_i p_i exp(-i k r . r_i), FP64.
 * theta, phi and intensity hold n_theta * n_phi doubles each. */
LUM_API int lum_far_field(lum_ctx* ctx, int n_dipoles, const double* pos, const double* moments,
                          double k, int n_theta, int n_phi, double* theta, double* phi,
                          double* intensity);

/* ---- nonlinear sources (nonlinear.rs) -------------------------------------- */
/* compute_shg_sources / compute_thg_sources (crates/lumina-core/src/
 * nonlinear.rs:61-86, :233-258): order 2: p_a = sum chi_abc E_b E_c
 * (Chi2Tensor, 27 complex, index a*9+b*3+c); order 3: p_a = sum chi_abcd
 * E_b E_c E_d (Chi3Tensor, 81 complex).  local_fields and sources are 3N
 * complex; chi holds n_tensors tensors back to back (1: one tensor for every
 * dipole, or N).  FP64 on the device.  The harmonic response solves
 * A(k_h) p = sources with a session at the harmonic wave number
 * (nonlinear.rs:108-240). */
LUM_API int lum_harmonic_sources(lum_ctx* ctx, int order, int n_dipoles, const double* local_fields,
                                 int n_tensors, const double* chi, double* sources);

/* ---- measurement --------------------------------------------------------- */
/* While enabled, every launch of the session's dominant matvec kernel (the
 * dense pair kernel, or the GEMV of a cached session) is bracketed by CUDA
 * events on the session stream.  lum_session_profile resets the record;
 * lum_session_kernel_time synchronises and returns the launches and total
 * milliseconds recorded for one precision (LUM_FP32 / LUM_FP64). */
LUM_API int lum_session_profile(lum_session* s, int enable);
LUM_API int lum_session_kernel_time(lum_session* s, int precision, int* launches,
                                    double* total_ms);
/* Dense-pair on-the-fly geometry facts: near pairs (FCD) and split factor. */
LUM_API int lum_session_stats(lum_session* s, long long* near_pairs, int* ell_width, int* nsplit32,
                      int* nsplit64);
/* Kernel configuration chosen for this session (autotuned FP32 pair-kernel
 * variant, split factors, near-list width, FP32 position mode) as a
 * "key=value ..." string. */
LUM_API int lum_session_kernel_config(lum_session* s, char* buf, size_t len);
/* CUDA-core throughput microbenchmark (FMA chains), the roofline
 * denominator for the compute-bound on-the-fly kernels: FP32 and FP64
 * GFLOP/s measured on the context's device. */
LUM_API int lum_measure_fma_peak(lum_ctx* ctx, double* fp32_gflops, double* fp64_gflops);
/* L2 read microbenchmark (16-byte loads that bypass L1 over a 16 MiB,
 * L2-resident buffer), the roofline denominator for the table gathers of the
 * periodic operator: GB/s on the context's device.  No counterpart in the
 * reference. */
LUM_API int lum_measure_l2_peak(lum_ctx* ctx, double* gbs);
/* The same FMA-chain microbenchmark with packed f32x2 FMAs (the instruction
 * the FP32 pair kernels use): FP32 GFLOP/s.  No counterpart in the
 * reference. */
LUM_API int lum_measure_fma2_peak(lum_ctx* ctx, double* gflops);

/* ---- allocation-free matvec ---------------------------------------------- */
/* No counterpart in the reference.  For callers that cannot let a library
 * allocate device memory (their HBM is owned by another allocator or reserved
 * up front, or allocation is not allowed where they call from):
 * y = alpha^-1 x - sum_{j != i} G(r_i - r_j) x_j, the FP64 point-dipole
 * on-the-fly matvec (use_fcd = 0), from caller-owned device arrays only --
 * pos N*3 doubles, inv_alpha N*9 complex, x and y 3N complex -- on `stream`
 * (NULL = the legacy default stream) of the current device.  Its scratch is a
 * fixed 8 MiB device array inside the library; N above 174,762 is rejected
 * with LUM_ERR_INVALID.  The first call on each device looks up that array's
 * device address, so make it before any stream capture; after a device reset
 * (a new context) the next call looks it up again.  All calls share the
 * array: calls that overlap on the GPU race and must be serialised.  Nothing
 * is allocated or freed. */
LUM_API int lum_matvec_onthefly_noalloc(int n_dipoles, const double* pos_dev,
                                        const double* inv_alpha_dev, double k,
                                        const double* x_dev, double* y_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LUMINA_B200_H */
