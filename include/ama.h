/*
 * amaterasu_b200 C-ABI: a B200 (sm_100a) plane-wave Kohn-Sham engine.
 *
 * Every entry point returns an int status (AMA_OK or an AMA_ERR_* code); the message of
 * the last failure on the calling thread is returned by ama_last_error(). Array
 * arguments are plain pointers: "host" arrays are read before the call returns, "device"
 * arrays are CUDA device pointers that the call uses in stream order on `stream`
 * (a cudaStream_t passed as void*; NULL means the legacy default stream). Complex arrays
 * are interleaved (re, im) pairs of float (AMA_C64) or double (AMA_C128).
 *
 * The entry points replace the numpy routines of the reference Python package
 * (amaterasu 0.1.0a2); each declaration names the reference function it stands in for.
 * One engine per stream; engines share no mutable state.
 */
#ifndef AMA_H_
#define AMA_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define AMA_API __attribute__((visibility("default")))
#else
#define AMA_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
  AMA_OK = 0,
  AMA_ERR_SHAPE = 1,         /* shape/size mismatch (Python: ValueError)            */
  AMA_ERR_CUDA = 2,          /* a CUDA runtime or library call failed               */
  AMA_ERR_NOT_CONVERGED = 3, /* an iteration hit its limit                          */
  AMA_ERR_TIMEOUT = 4,       /* a bounded device wait ran out                       */
  AMA_ERR_NOT_SPD = 5,       /* Cholesky met a non-positive pivot                   */
  AMA_ERR_ARG = 6,           /* invalid argument (null pointer, bad enum)           */
  AMA_ERR_UNSUPPORTED = 7    /* a size or option the engine does not implement      */
};

enum { AMA_C64 = 0, AMA_C128 = 1 };

typedef struct AmaEngine AmaEngine;

typedef struct AmaSystemDesc {
  int32_t n1, n2, n3;        /* FFT grid, C order (axis 2 fastest)                   */
  int32_t nk;                /* number of k-points                                   */
  const int32_t* npw;        /* host [nk]: plane waves per k                          */
  const int32_t* miller;     /* host [sum npw][3]: Miller indices, sphere order, k-major */
  const double* kinetic;     /* host [sum npw]: |k+G|^2/2 in Hartree                  */
  int32_t nproj;             /* projector rows (same for every k), may be 0           */
  const double* projectors;  /* host complex [sum_k nproj*npw_k]: <k+G|beta_i>, k-major,
                                row-major (nproj, npw_k) per k; may be NULL if nproj==0 */
  const double* dij;         /* host [nproj*nproj]: D_ij in Hartree                   */
  int32_t nspin;             /* 1 or 2                                               */
  uint32_t precisions;       /* bit AMA_C64: keep complex64 copies; bit AMA_C128: complex128 */
} AmaSystemDesc;

AMA_API const char* ama_last_error(void);
AMA_API int ama_version(void);

/* Build an engine: index maps, kinetic energies, projector matrices and D.B on the
 * current CUDA device. Replaces the per-geometry tables the reference builds in
 * hamiltonian/system.py:215-379 (wave spheres, fft.py:174-190 indices, kb.py:260-343). */
AMA_API int ama_engine_create(const AmaSystemDesc* desc, AmaEngine** engine);
AMA_API int ama_engine_destroy(AmaEngine* engine);

/* Engine options (no counterpart in the reference):
 *   option 0: nonlocal products of the complex64 path on the tensor cores (value 1, default)
 *             or on the SIMT GEMM (value 0);
 *   option 1: complex64 stage B (x transforms and V) variant: 0 shared-memory slabs,
 *             1 register-resident x columns, 2 register-resident with the spheres' compile-time
 *             x-plane set, 3 register-resident with two threads per column (even x length),
 *             4 shared-memory slabs split in two along z (complex64: x lines of 100 or
 *             more; complex128: 40 or more);
 *             AMA_ERR_UNSUPPORTED when the variant is not compiled for the grid;
 *   option 2: the same for complex128 (variants 0 and 4).
 *   option 3: complex64 stages A and C (scatter + z, y backward; y, z forward + gather)
 *             variant: 0 shared-memory y passes, 1 y transforms in registers with four
 *             threads per column (n2 a multiple of 4 on a compile-time grid);
 *             AMA_ERR_UNSUPPORTED when the variant is not compiled for the grid.
 *   option 4: ama_davidson replays recurring iteration segments as CUDA graphs (value 1,
 *             default) or launches every kernel (value 0); the results are the same.
 * amaterasu_b200.autotune times the variants and keeps the fastest. */
AMA_API int ama_engine_option(AmaEngine* engine, int32_t option, int32_t value);

/* Device-side status of the tensor-core kernels (0 = fine; otherwise the code of the
 * first bounded wait that ran out). Synchronous. No counterpart in the reference. */
AMA_API int ama_tc_status(AmaEngine* engine, int32_t* code);

/* Effective potential V_eff(r) for each spin channel, device FP64 [nspin][n1*n2*n3],
 * natural grid order. Replaces Hamiltonian.__init__ (hamiltonian/operator.py:49-58). */
AMA_API int ama_set_potential(AmaEngine* engine, const double* v, int32_t nspin, void* stream);

/* Pre-size the H.psi workspace for up to `max_bands` bands in flight (sum over the
 * k-points of one call). Optional: ama_hpsi grows it on demand. */
AMA_API int ama_reserve(AmaEngine* engine, int32_t precision, int64_t max_bands);

/* H.psi = T psi + G[V R[psi]] + B^H D B psi for `nbands` bands at each of the k-points
 * k_first .. k_first+k_count-1. psi/hpsi are device arrays holding, back to back, one
 * row-major (nbands, npw_k) block per k-point. Replaces Hamiltonian.apply
 * (hamiltonian/operator.py:60-69) batched over k. */
AMA_API int ama_hpsi(AmaEngine* engine, int32_t precision, int32_t k_first, int32_t k_count,
             int32_t nbands, int32_t spin, const void* psi, void* hpsi, void* stream);

/* Occupation-weighted density: rho[spin][r] += sum_k sum_n weights[k*nbands+n] |u_nk(r)|^2
 * over the bands of k_first..k_first+k_count-1 (device weights, FP64), accumulated in
 * FP64 into the device array rho [n1*n2*n3] (natural order; caller zeroes it and applies
 * 1/Omega). Replaces the inner loop of compute_density (scf/density.py:60-71). */
AMA_API int ama_density_accumulate(AmaEngine* engine, int32_t precision, int32_t k_first,
                           int32_t k_count, int32_t nbands, const void* psi,
                           const double* weights, double* rho, void* stream);

/* <beta_i|psi_n> for one k-point: proj[n][i] = sum_G psi[n][G] conj(B[i][G]).
 * Replaces KBProjectors.project (pseudo/kb.py:216-218). */
AMA_API int ama_project(AmaEngine* engine, int32_t precision, int32_t k, int32_t nbands,
                const void* psi, void* proj, void* stream);

/* Complex GEMM on device arrays, batched with fixed strides:
 *   trans_b == 0: C[b] = alpha * A[b] (m x k) * B[b] (k x n)           + beta * C[b]
 *   trans_b == 1: C[b] = alpha * A[b] (m x k) * conj(B[b] (n x k))^T   + beta * C[b]
 *   trans_b == 2: C[b] = alpha * conj(A[b] (k x m))^T * B[b] (k x n)   + beta * C[b]
 * All matrices row-major with leading dimensions lda/ldb/ldc (elements); alpha and beta
 * are complex (re, im) in double. Replaces the ndarray products of the Davidson
 * subspace steps (scf/eigen/subspace.py:24-76, davidson.py:81-100). */
AMA_API int ama_zgemm(int32_t precision, int32_t trans_b, int32_t m, int32_t n, int32_t k,
              const double* alpha, const void* a, int64_t lda, int64_t stride_a,
              const void* b, int64_t ldb, int64_t stride_b, const double* beta, void* c,
              int64_t ldc, int64_t stride_c, int32_t batch, void* stream);

/* A block of rows inside per-k-point packed storage (for the batched Davidson).
 * ragged = 1: block k starts at rows_per_k * pw_off[k] elements, rows have npw_k elements,
 *             and the operand starts at row row0 of the block;
 * ragged = 0: block k starts at k * kstride elements, rows have ld elements, row row0. */
typedef struct AmaKOperand {
  void* base;
  int64_t rows_per_k;
  int64_t row0;
  int32_t ragged;
  int64_t ld;
  int64_t kstride;
} AmaKOperand;

/* One complex GEMM per k-point in a single launch (forms as ama_zgemm: 0 NN, 1 NC, 2 CN);
 * m, n or k equal to -1 mean the k-point's plane-wave count npw[k] (device int32 [nk]);
 * pw_off (device int64 [nk]) are the prefix sums of npw; max_m/max_n bound the shapes.
 * Replaces the per-k ndarray products of davidson/rayleigh_ritz run over every k. */
AMA_API int ama_kbatch_zgemm(int32_t precision, int32_t form, int32_t nk, int32_t m, int32_t n, int32_t k,
                             const int32_t* npw, const int64_t* pw_off, const AmaKOperand* a,
                             const AmaKOperand* b, const AmaKOperand* c, const double* alpha,
                             const double* beta, int32_t max_m, int32_t max_n, void* stream);

/* The complex64 forms of ama_kbatch_zgemm on the tensor cores (tcgen05, split-TF32 with
 * FP32 chains drained into registers every 2 k-blocks and FP64 reduction of the splits):
 *   form 1 (NC): C = alpha A B^H + beta C with k = -1 (reduction over each k's plane
 *                waves), A and B per-k blocks, C a small matrix per k;
 *   form 0 (NN): C = alpha A B + beta C with n = -1 (output columns = plane waves), A a
 *                small matrix per k, B and C per-k blocks.
 * max_npw bounds npw (host value: the staging arrays are padded to it). Same products as
 * ama_kbatch_zgemm (davidson.py/subspace.py GEMMs); other forms or shapes are
 * AMA_ERR_UNSUPPORTED / AMA_ERR_SHAPE. Stream-ordered; scratch grows on demand. */
AMA_API int ama_kbatch_zgemm_tc(int32_t form, int32_t nk, int32_t m, int32_t n, int32_t k,
                                const int32_t* npw, const int64_t* pw_off, const AmaKOperand* a,
                                const AmaKOperand* b, const AmaKOperand* c, const double* alpha,
                                const double* beta, int32_t max_npw, void* stream);

/* Error flag of the subspace tensor-core kernels (0 = none; otherwise the code of a bounded
 * wait that timed out). Synchronous. */
AMA_API int ama_subspace_tc_status(int32_t* code);

/* Teter-Payne-Allan preconditioning fused with the residual and normalisation:
 *   r = hx - eps*x; t_n = sum_G |x|^2 T_G; out = K(T_G / max(t_n,1e-8)) r / ||.||
 * for the `nrows` rows listed in `rows` (device int32); norms (device FP64 [nbands]) get
 * ||hx - eps x|| for every band. Replaces davidson.py:81-93 and precond.py:27-46. */
AMA_API int ama_residual_precondition(int32_t precision, int32_t nbands, int32_t npw,
                              const void* x, const void* hx, const double* eps,
                              const double* kinetic, double* norms, const int32_t* rows,
                              int32_t nrows, void* out, void* stream);

/* Reciprocal-space filter of a real grid field (FP64): stores a filter f(G) (host array,
 * natural FFT order, one value per grid point) in slot 0..3 of the engine. */
AMA_API int ama_set_grid_filter(AmaEngine* engine, int32_t slot, const double* filter);

/* out(r) = Re sum_G f_slot(G) rho(G) e^{iG.r} with rho(G) = (1/N) sum_r rho(r) e^{-iG.r}
 * (device FP64 arrays [n1*n2*n3], natural order); if energy_slot >= 0, *energy (device
 * double) += sum_G f_energy_slot(G) |rho(G)|^2. With f = 4pi/G^2 on the density sphere this
 * is the Hartree potential and energy (hamiltonian/hartree.py:28-50); with
 * f = G^2/(G^2+q0^2) the Kerker filter (scf/mixing.py:94-105). */
AMA_API int ama_grid_filter(AmaEngine* engine, int32_t slot, int32_t energy_slot,
                            const double* in, double* out, double* energy, void* stream);

/* ama_grid_filter without any allocation, for callers that cannot let the library call
 * cudaMalloc (device memory already reserved by a framework's allocator, or loops that
 * must not take cudaMalloc's device-wide synchronisation). No counterpart in the
 * reference. Same arguments and result as ama_grid_filter; the complex work grid is a
 * fixed device array of 128^3 points (32 MiB, held on every GPU that loads the library),
 * and a larger grid returns AMA_ERR_SHAPE. The array's address is looked up when an
 * engine is created on the device (which also loads the library's device code there, so
 * create the engine before a framework allocator reserves the GPU); that lookup happens
 * before any stream capture the caller makes. The library does not survive a
 * cudaDeviceReset of a device it has used. All calls share the array: calls that overlap
 * on the GPU race. */
AMA_API int ama_grid_filter_noalloc(AmaEngine* engine, int32_t slot, int32_t energy_slot,
                                    const double* in, double* out, double* energy, void* stream);

/* Forward transform of a real grid field to natural FFT order (device FP64 in
 * [n1*n2*n3], device complex128 out [n1*n2*n3]): out[G] = (1/N) sum_r in(r) e^{-iG.r}.
 * Replaces FFTGrid.to_reciprocal on a density (basis/fft.py:228-235). */
AMA_API int ama_grid_fft_forward(AmaEngine* engine, const double* in, void* out, void* stream);

/* Spectral gradient of a real grid field (device FP64 in [N], out [3][N], Cartesian x, y, z):
 * out_a = scale * Re IFFT(i G_a FFT(in)), the Nyquist frequency of every even axis zeroed.
 * cell: host, the 3 x 3 lattice vectors as rows (Bohr). Needs the complex128 tables.
 * Replaces FFTGrid.gradient (basis/fft.py:288-295). */
AMA_API int ama_grid_gradient(AmaEngine* engine, const double* cell, const double* in, double scale,
                              double* out, void* stream);

/* Spectral divergence of a real vector field (device FP64 in [3][N]), accumulated:
 * out = beta * out + alpha * Re IFFT(sum_a i G_a FFT(in_a)) (Nyquist zeroed as above).
 * Replaces FFTGrid.divergence (basis/fft.py:297-304). */
AMA_API int ama_grid_divergence(AmaEngine* engine, const double* cell, const double* in, double alpha,
                                double beta, double* out, void* stream);

/* PBE (functional 0) or PBEsol (1) exchange-correlation of a density (device FP64
 * rho [nspin][N], electrons/Bohr^3; nspin 1 is split n/2, n/2): vxc [nspin][N] the full
 * potential d(n eps)/dn_s - div(2 vsigma_ss grad n_s + vsigma_ud grad n_s'); result (device,
 * 7 doubles): [0] E_xc (Ha), [1..6] the gradient stress sum
 * sum_r [2 vsigma_uu g_u g_u + vsigma_ud (g_u g_d + g_d g_u) + 2 vsigma_dd g_d g_d] dV in the
 * order xx yy zz yz xz xy. Replaces XCFunctional.evaluate_on_grid for a GGA
 * (xc/driver.py:108-165, xc/gga.py:112-254) and the gradient part of the xc stress
 * (properties/stress.py:159-185). */
AMA_API int ama_xc_gga(AmaEngine* engine, int32_t functional, int32_t nspin, const double* cell,
                       const double* rho, double* vxc, double* result, void* stream);

/* ama_residual_precondition for every k-point in one launch: x/hx packed (nbands, npw_k)
 * blocks, eps/norms [nk][nbands], kinetic packed by pw_off; rows [nk][nbands] gives the
 * output row of each band's correction (-1: none) in out, packed (nrows, npw_k) blocks. */
AMA_API int ama_kbatch_residual(int32_t precision, int32_t nk, int32_t nbands, const int32_t* npw,
                                const int64_t* pw_off, const void* x, const void* hx, const double* eps,
                                const double* kinetic, double* norms, const int32_t* rows, int32_t nrows,
                                void* out, void* stream);

/* Block Davidson for the nbands lowest eigenpairs at every k-point of the engine, all
 * k-points in lockstep, with the engine's H.psi (its current potential, spin channel
 * `spin`) as the operator; the reference's algorithm per k-point (scf/eigen/davidson.py:48-111:
 * Rayleigh-Ritz, Teter-Payne-Allan corrections of the bands with residual norm > tolerance,
 * two projections off the basis, 1e-7 rank test, orthonormalisation, collapse at 4 nbands),
 * orchestrated in C++ over the library's kernels. guess and x: device, one row-major
 * (nbands, npw_k) block per k-point back to back, in the precision's complex type (x may be
 * guess). eigenvalues, norms: device FP64 [nk][nbands] (norms may be NULL); iterations: host.
 * tc_min_npw > 0 routes the complex64 plane-wave products to the tensor cores when the
 * largest sphere has at least that many plane waves (0: never). The iterations run on the
 * library's own stream after the work queued on `stream`; the call returns when its results
 * are written. The host synchronises twice per iteration (the active bands; the rank test
 * and the orthonormalisation's admissibility); the launches between two synchronisations
 * depend only on the basis size, the block width and the Newton-Schulz step count, and with
 * engine option 4 on (the default) such a segment is captured as a CUDA graph on its second
 * occurrence and replayed afterwards (segments with eigensolves above order 80 are launched
 * directly). AMA_ERR_ARG for a rank-deficient start. */
AMA_API int ama_davidson(AmaEngine* engine, int32_t precision, int32_t spin, int32_t nbands, const void* guess,
                         double tolerance, int32_t max_iterations, int32_t tc_min_npw, double* eigenvalues,
                         void* x, double* norms, int32_t* iterations, void* stream);

/* ama_davidson's iteration segments on the calling host thread and current device: captured
 * as CUDA graphs, replayed from a graph, launched kernel by kernel (counts since the last
 * reset; reset != 0 zeroes them after reading). No counterpart in the reference. */
AMA_API int ama_davidson_graph_stats(int64_t* captured, int64_t* replayed, int64_t* launched, int32_t reset);

/* Copy nrows rows per k-point between packed per-k blocks (block k at rows_per_k*pw_off[k],
 * rows of npw_k elements, starting at row row0). */
AMA_API int ama_kbatch_copy_rows(int32_t precision, int32_t nk, int32_t nrows, const int32_t* npw,
                                 const int64_t* pw_off, const void* src, int64_t src_rows_per_k,
                                 int64_t src_row0, void* dst, int64_t dst_rows_per_k, int64_t dst_row0,
                                 void* stream);

/* LDA exchange plus Perdew-Zunger 1981 correlation on a spin-resolved density
 * (device FP64, rho [2][npoints]); writes eps_xc [npoints] and v_xc [2][npoints].
 * Replaces lda.exchange + lda.correlation_pz81 (xc/lda.py:122-142,203-262). */
AMA_API int ama_lda_pz(const double* rho, int64_t npoints, double* eps, double* vrho, void* stream);

/* ---- FP64 grid vectors of the SCF loop (mixers, density, energies). Vectors are device
 * arrays of n doubles; `vectors` is a HOST array of nvec device pointers; coefficients are
 * host arrays. Every reduction is deterministic (fixed summation order). */

/* Overlaps of linear combinations of up to 16 vectors: u_a = sum_j coef[a*nvec+j] v_j for
 * a < ncomb, plus u_ncomb = extra when extra != NULL; gram (device, (ncomb+e)^2 doubles,
 * row-major, symmetric) = u_a . u_b. Replaces the residual overlap products of
 * PulayMixer._coefficients and BroydenMixer (scf/mixing.py:173-193,238-258). */
AMA_API int ama_vec_gram(int32_t nvec, const double* const* vectors, int32_t ncomb, const double* coef,
                         const double* extra, int64_t n, double* gram, void* stream);

/* out = sum_j coef[j] v_j (up to 16 vectors). Replaces the history combinations of the
 * mixers (scf/mixing.py:195-201, 258-260). */
AMA_API int ama_vec_lincomb(int32_t nvec, const double* const* vectors, const double* coef, int64_t n,
                            double* out, void* stream);

/* *out = (accumulate ? *out : 0) + scale * R with R = sum a*b (op 0), sum |a - b| (op 1),
 * sum a (op 2) or sum max(a, 0) (op 3); out is a device double. The energy integrals and the
 * density residual of run_scf (scf/driver.py:376-419). */
AMA_API int ama_vec_reduce(int32_t op, int64_t n, const double* a, const double* b, double scale,
                           int32_t accumulate, double* out, void* stream);

/* rho[c] <- max(rho[c] / volume, 0) * (sum rho[c] / sum max(rho[c], 0)) for each of the
 * nchannels channels of n points (in place): the 1/Omega and the charge-preserving floor of
 * compute_density (scf/density.py:71-84, symmetry off). */
AMA_API int ama_density_floor(int32_t nchannels, int64_t n, double volume, double* rho, void* stream);

/* rows[k*nbands + b] = sum_G |psi_bk(G)|^2 T_k(G) over the packed per-k blocks (npw, pw_off
 * device as for ama_kbatch_zgemm, kinetic packed by pw_off). Per-band kinetic energies of
 * _kinetic_energy (scf/driver.py:520-528). */
AMA_API int ama_band_kinetic(int32_t precision, int32_t nk, int32_t nbands, const int32_t* npw,
                             const int64_t* pw_off, const void* psi, const double* kinetic, double* rows,
                             void* stream);

/* rows[i] = Re sum_j conj(a[i][j]) b[i][j] for complex128 row-major (nrows, ncols) arrays:
 * the per-band <beta|psi>^* D <beta|psi> of _nonlocal_energy (scf/driver.py:531-541). */
AMA_API int ama_rowdot(int32_t nrows, int32_t ncols, const void* a, const void* b, double* rows, void* stream);

/* Ewald energy, forces and stress of point charges in a periodic cell (FP64):
 *   out[0] = E (Ha); out[1 + 3a + c] = F_a,c (Ha/Bohr); out[1 + 3 natoms + 3i + j] = sigma_ij
 *   = (1/Omega) dE/d eps_ij (Ha/Bohr^3).
 * positions [natoms][3] Bohr, charges [natoms], shifts [nshift][3] lattice translations
 * covering the real-space cutoff rcut (terms with r > rcut are skipped), gvectors [ng][3]
 * nonzero reciprocal vectors of the reciprocal sum, eta the splitting parameter, volume the
 * cell volume; work holds 13 natoms + 9 ng doubles, 16-byte aligned. All arrays on the device. Replaces
 * hamiltonian/ewald.py:94-228 (ewald). */
AMA_API int ama_ewald(int32_t natoms, const double* positions, const double* charges, const double* shifts,
                      int32_t nshift, const double* gvectors, int32_t ng, double eta, double rcut, double volume,
                      double* work, double* out, void* stream);

/* Structure sums of the set-up (superposed atomic densities and local potentials):
 *   out[g] = scale * sum_a radial[species[a] * ng + g] * exp(-i G_g . tau_a)
 * gcart: device FP64 [ng][3] Cartesian G vectors; positions: [natoms][3] Bohr; species:
 * int32 [natoms] row of `radial` (device FP64 [nspecies][ng]); out: complex128 [ng].
 * Replaces the phase matrix and per-atom sums of hamiltonian/local.py:37-74. */
AMA_API int ama_structure_sum(const double* gcart, int32_t ng, const double* positions, const int32_t* species,
                              int32_t natoms, const double* radial, double scale, double* out, void* stream);

/* Dense FP64 Hermitian eigensolver for `batch` matrices of order n <= 2400 (device,
 * row-major, interleaved complex, overwritten by eigenvectors as columns); eigenvalues
 * ascending. Hand-written: Householder tridiagonalisation in one cooperative launch,
 * multisection bisection, inverse iteration with Gram-Schmidt inside eigenvalue clusters,
 * back-transformation; no vendor solver library and no host synchronisation (a device-side
 * failure is reported by ama_solver_status). Scratch grows on demand per host thread and
 * device. Replaces scipy.linalg.eigh in rayleigh_ritz (scf/eigen/subspace.py:74). */
AMA_API int ama_heev(int32_t n, void* matrices, double* eigenvalues, int32_t batch, void* stream);

/* The lowest nvec eigenpairs of each matrix (as ama_heev: eigenvalues ascending in
 * eigenvalues[b*n + 0 .. nvec), eigenvectors in row-major columns 0 .. nvec-1; the rest of
 * both is undefined). Only nvec eigenvalues are bisected and nvec vectors back-transformed:
 * the Rayleigh-Ritz step needs the nbands lowest of m = up to 5 nbands Ritz pairs
 * (subspace.py:74 computes all of them with scipy.linalg.eigh). */
AMA_API int ama_heev_lowest(int32_t n, int32_t nvec, void* matrices, double* eigenvalues, int32_t batch,
                            void* stream);

/* Sticky device-side status of ama_heev/ama_heev_lowest on the current device and host
 * thread (0 = fine, 1 = a bounded grid-barrier wait ran out, so the results of some call
 * since the last read are invalid); synchronous; clears the word. No counterpart in the
 * reference. */
AMA_API int ama_solver_status(int32_t* code);

/* The same for many small matrices (order n <= 80) at once: one CTA per matrix, cyclic
 * Jacobi in shared memory, FP64. Used for the per-k-point Rayleigh-Ritz problems of the
 * batched Davidson (scf/eigen/subspace.py:74 for every k). */
AMA_API int ama_heev_small(int32_t n, void* matrices, double* eigenvalues, int32_t batch, void* stream);

/* Inverse Cholesky factor of `batch` Hermitian positive-definite FP64 matrices (device,
 * row-major, interleaved complex): on return each holds L^{-1} (lower triangular) with
 * S = L L^H. AMA_ERR_NOT_SPD if a pivot is not positive (synchronous: the caller falls back
 * on it). Hand-written, one CTA per matrix. Replaces the cholesky + solve_triangular pair of
 * orthonormalize (scf/eigen/subspace.py:17-32). */
AMA_API int ama_potrf_inv(int32_t n, void* matrices, int32_t batch, void* stream);

/* ---- learned start density: periodic 3D convolution network (no counterpart in the
 * reference; the start density it replaces is hamiltonian/local.py:77-106).
 * Tensors [batch][channels][d][d][d], 3x3x3 kernels w[co][ci][3][3][3], circular
 * padding 1, stride 1 or 2 (d_out = d_in / stride); BF16 activations and weights
 * (x, w, y of the _bf16 functions), FP32 accumulation, outputs and gradients. */
AMA_API int ama_conv3d_fwd_bf16(const void* x, const void* w, const float* bias, float* y, int32_t batch,
                                int32_t ci, int32_t co, int32_t din, int32_t stride, void* stream);
AMA_API int ama_conv3d_bwd_data_bf16(const float* dy, const void* w, float* dx, int32_t batch, int32_t ci,
                                     int32_t co, int32_t din, int32_t stride, void* stream);
AMA_API int ama_conv3d_bwd_weight_bf16(const float* dy, const void* x, float* dw, float* dbias, int32_t batch,
                                       int32_t ci, int32_t co, int32_t din, int32_t stride, void* stream);
AMA_API int ama_silu_fwd_bf16(const float* x, void* y, int64_t n, void* stream);
AMA_API int ama_silu_bwd(const float* x, const float* dy, float* dx, int64_t n, void* stream);
AMA_API int ama_upsample2_fwd_bf16(const void* x, void* y, int64_t channels, int32_t d, void* stream);
AMA_API int ama_upsample2_bwd(const float* dy, float* dx, int64_t channels, int32_t d, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* AMA_H_ */
