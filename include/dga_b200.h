/*
 * dga_b200.h -- C ABI of the B200 ladder-DGA hot path (libdga_b200.so).
 *
 * Every entry point is extern "C", takes plain device pointers, sizes and a cudaStream_t, enqueues its
 * kernels on that stream without synchronising, allocates nothing (callers pass scratch buffers sized by the
 * *_scratch_bytes queries) and returns 0 on success or a DGA_ERR_* code, with a message available from
 * dga_last_error_string().  Complex arrays are interleaved (re, im) doubles, the memory layout of numpy
 * complex128.  Per-item status words report singular pivots, non-finite results and non-convergence.
 *
 * Layout vocabulary (n = orbitals, n2 = n*n, nv = 2*niv core, nvf = 2*(niv+niv_shell), W = niw+1 bosonic
 * frequencies w >= 0, Q = irreducible q points, Nk = momentum grid points, N = n2*nv compound size):
 *   compound orbital matrix  [(o1,o2),(o4,o3)]: row p = o1*n+o2, column s = o4*n+o3
 *   compound BSE matrix      row (o1,o2,nu) = p*nv+nu, column (o4,o3,nu') = s*nv+nu'
 *
 * Each declaration names the upstream (Julpe/DGAmore, Python) function whose body it replaces.
 */
#ifndef DGA_B200_H
#define DGA_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* dga_stream_t; /* cudaStream_t */

#define DGA_OK 0
#define DGA_ERR_ARG 1
#define DGA_ERR_SCRATCH 2
#define DGA_ERR_LAUNCH 3
#define DGA_ERR_CUDA 4

#define DGA_ITEM_OK 0
#define DGA_ITEM_SINGULAR 1
#define DGA_ITEM_NONFINITE 2
#define DGA_ITEM_NOCONVERGE 4
#define DGA_ITEM_WAIT_TIMEOUT 8 /* a bounded wait on an asynchronous copy or tensor-core tile ran out */

/* Library version (major*10000 + minor*100 + patch) and the last error message of the calling thread. */
int dga_version(void);
const char* dga_last_error_string(void);

/* Streaming multiprocessors of the current device (cached per device); the grid sizes of the streaming kernels
 * and the caller's chunking of the Sigma contraction are multiples of it.  No counterpart in the upstream. */
int dga_device_sm_count(void);

/* Resident CTAs per SM of the block-form mixed BSE kernel (tuning kernel 4) for n2 = n_orb^2 right-hand sides,
 * as the occupancy calculator gives it on the current device (-1 on error).  No counterpart in the upstream. */
int dga_bse_block_ctas_per_sm(int n2);

/* Generic strided complex copy dst[idx . dst_stride] = scale * src[idx . src_stride] over `shape`
 * (up to 8 dims, strides in complex elements).  Layout conversions at the boundary
 * (FourPoint.to_compound_indices / to_full_indices, dgamore/four_point.py:166-293). */
int dga_strided_copy_c128(const void* src, void* dst, int ndim, const long long* shape, const long long* src_stride,
                          const long long* dst_stride, double scale, dga_stream_t stream);

/* dga_sigma_c128 through the irreducible wedge of real space, for kernels without per-k orbital rotations whose
 * grid group holds the inversion (R and -R share a representative): F(R) = sum_q K(q) e^{iqR} is invariant under
 * the group, so it is formed only at the irreducible R as one complex GEMM over the irreducible q against
 * s_star [Q][Q], S[q_irr][r] = sum over the star of q_irr of e^{+i q R_r} (R_r = the point irrk_ind[r]), and the
 * contraction reads F at each R's representative (irrk_inv).  gemm_tile: the GEMM's output tile (rows of kernel
 * planes x columns of irreducible R; 0 = 64 x 64, 1 = 128 x 32), a choice of the autotuner.  Same
 * inputs and output as dga_sigma_c128 otherwise; scratch: dga_sigma_wedge_scratch_bytes. */
size_t dga_sigma_wedge_scratch_bytes(int n_orb, int niv, int niw, int n_q, int nk, int n_chunks);
int dga_sigma_wedge_c128(const void* kern, const void* g_r, int n_orb, int niv, int niw, int n_q, int nx, int ny,
                         int nz, const int* irrk_inv, const void* s_star, const void* tw_inv, double beta,
                         int n_chunks, int gemm_tile, void* out, void* scratch, size_t scratch_bytes,
                         dga_stream_t stream);

/* IBZ -> FBZ expansion of a four-orbital object with the auto-mode orbital rotation (IAmNonLocal._map_to_full_bz,
 * dgamore/n_point_base.py:462-507, through symmetry_reduction.apply_auto_orbital_transform, :791-902):
 *   dst[k](o1,o2,o3,o4; f) = sigma_k^2 sum U_{o1 p} U*_{o2 q} U_{o3 r} U*_{o4 s} [src[irrk_inv[k]](p,q,r,s; f)]^(*conj_k)
 * for k < nk.  A block of `block` elements per point holds orbital index i at orb_strides[i] and the frequency
 * pairs (f1 < f1_count, f2 < f2_count) at f1 f1_stride + f2 f2_stride; us [nk][n][n], sigmas [nk] (may be null),
 * conjs [nk] (bytes, nonzero = conjugate) are the per-k data of the upstream's symmetry discovery
 * (KGrid.specify_auto_symmetries, brillouin_zone.py:365-449).  n_orb <= 4, nk <= 65535. */
int dga_fbz_rotate_c128(const void* src, const int* irrk_inv, int nk, const void* us, const double* sigmas,
                        const unsigned char* conjs, int n_orb, const long long* orb_strides, long long f1_stride,
                        int f1_count, long long f2_stride, int f2_count, long long block, void* dst,
                        dga_stream_t stream);

/* Batched separable DFT of momentum planes; replaces IAmNonLocal.fft / ifft (dgamore/n_point_base.py:509-551).
 * Element (plane p = p_hi*n_lo + p_lo, point R) at p_hi*s_hi + p_lo*s_lo + R*s_r; tw = nx+ny+nz twiddles
 * e^{s 2 pi i m/n} (sign folded in by the caller); output multiplied by `scale`. */
int dga_dft_planes_c128(const void* in, long long in_s_hi, long long in_s_lo, long long in_s_r, void* out,
                        long long out_s_hi, long long out_s_lo, long long out_s_r, int n_lo, int n_planes, int nx,
                        int ny, int nz, const void* tw, double scale, dga_stream_t stream);

/* Bare bubble chi0[q_irr,a,b,c,d,w>=0,nu] = -beta/Nk IFFT_R[G_ad(R,nu) G_cb(-R,nu-w)], filtered at 1e-12;
 * replaces BubbleGenerator.create_generalized_chi0_q_fft_cpu/_gpu/_auto (dgamore/bubble_gen.py:33-144).
 * g_r: [2niv+niw][n][n][Nk] transforms of G(k) for nu in [-niv-niw, niv); q_irr: [n_qirr][3];
 * out addressed by 7 element strides (q, w, nu, a, b, c, d). */
int dga_bubble_c128(const void* g_r, int n_orb, int niv, int niw, int nx, int ny, int nz, const int* q_irr,
                    int n_qirr, const void* tw, double beta, void* out, const long long* out_strides,
                    dga_stream_t stream);

/* chi0^-1 per (q, w, nu_core) and the nu sums (1/beta^2) sum chi0 over the full and core boxes; replaces
 * FourPoint.invert(copy=False) for one nu dimension (dgamore/four_point.py:601-613) and
 * nonlocal_sde.py:824-835.  chi0: [Q][W][nvf][n2][n2] -> chi0_inv [Q][W][nv][n2][n2], sums [Q][W][n2][n2]. */
int dga_chi0_prep_c128(const void* chi0, int n_orb, int niv_core, int niv_shell, int niw_half, int n_q, double beta,
                       void* chi0_inv, void* full_sum, void* core_sum, int* status, dga_stream_t stream);

/* Scratch bytes of dga_bse_solve_sum_c128 / dga_invert_sum_dense_c128 for n_items items of size N. */
size_t dga_bse_scratch_bytes(int N, int n2, int n_items);

/* Ladder BSE in FP64: X[ch][q][w][(o1,o2,nu)][(o4,o3)] = sum_nu' [chi0^-1 + (Gamma_r - U_r - V_r^q)/beta^2]^-1 / beta
 * for each work item (ch, q, w); replaces nonlocal_sde.create_auxiliary_chi_r_q_sum_v1/_v3
 * (dgamore/nonlocal_sde.py:85-156) with FourPoint.invert_and_sum_over_last_vn(_v2) (four_point.py:620-684).
 * gamma_cm: [n_ch][W][N][N] column-major compound Gamma_r; chi0_inv: [Q][W][nv][n2][n2]; uv: [n_ch][Q][n2][n2]
 * (U_r + V_r^q); work: [n_items][3] ints (ch, q, w); out: [n_ch][Q][W][N][n2]; status: [n_items]. */
int dga_bse_solve_sum_c128(int n_orb, int niv, int niw_half, int n_q, int n_ch, double beta, double inv_beta2,
                           const void* gamma_cm, const void* chi0_inv, const void* uv, const int* work, int n_items,
                           void* out, int* status, void* scratch, size_t scratch_bytes, dga_stream_t stream);

/* Mixed-precision ladder BSE (same inputs and outputs as dga_bse_solve_sum_c128): complex64 LU with FP32
 * trailing updates, then FP64 iterative refinement -- residuals r = S - A Y with A formed in FP64 from Gamma_r,
 * chi0^-1 and U_r + V_r^q -- until the correction, or the error left after it estimated from the observed
 * contraction rho = |d_k|/|d_(k-1)| as |d_k| rho/(1-rho), is at most tol max|Y|, or max_iter corrections; items
 * that do not converge are flagged DGA_ITEM_NOCONVERGE.  The launch runs the block-form kernel (kernel 4 of
 * dga_bse_tuning) wherever its solve phase fits shared memory (every size of the benchmark configurations; see
 * dga_bse_default_kernel), else the shared-memory-panel kernel (320 <= N <= about 790) or the 128-thread kernel.
 * Replaces the same upstream functions as dga_bse_solve_sum_c128.  iters: optional per-item number of
 * corrections. */
size_t dga_bse_mixed_scratch_bytes(int N, int n2, int n_items);
int dga_bse_solve_sum_mixed_c128(int n_orb, int niv, int niw_half, int n_q, int n_ch, double beta, double inv_beta2,
                                 const void* gamma_cm, const void* chi0_inv, const void* uv, const int* work,
                                 int n_items, int max_iter, double tol, void* out, int* status, int* iters,
                                 void* scratch, size_t scratch_bytes, dga_stream_t stream);

/* The kernel a single request of n_orb orbitals and niv positive fermionic frequencies takes by default (the
 * kernel numbers of dga_bse_tuning; the FP64 form always 2); -1 for an unsupported size.  A batch launch runs each
 * request with this same kernel, so requests whose defaults differ go to different launches. */
int dga_bse_default_kernel(int n_orb, int niv, int mixed);

/* Loads the code of the mixed form's block-form kernels on the current device now.  CUDA otherwise loads a kernel
 * at its first launch, which for these large kernels takes tens of milliseconds inside that launch; a server calls
 * this once at start-up so that no request pays it.  Returns 0 or DGA_ERR_LAUNCH. */
int dga_bse_preload(void);

/* FP64 re-solve of the items a mixed launch flagged (status & (NOCONVERGE | NONFINITE | WAIT_TIMEOUT)), leaving the others
 * untouched; at most grid_limit CTAs (scratch: grid_limit * (N*N + N*n2) complex128). */
int dga_bse_resolve_fp64_c128(int n_orb, int niv, int niw_half, int n_q, int n_ch, double beta, double inv_beta2,
                              const void* gamma_cm, const void* chi0_inv, const void* uv, const int* work, int n_items,
                              void* out, int* status, int grid_limit, void* scratch, size_t scratch_bytes,
                              dga_stream_t stream);

/* Launch choices of the BSE solvers, the search space of the autotuner (dgamore_b200/autotune.py); no
 * counterpart in the upstream.  kernel: 0 = default (dga_bse_default_kernel), 1 = shared-memory-panel kernel
 * (mixed form only, N up to about 790), 2 = 128-thread kernel, 3 = shared-memory-panel kernel whose trailing
 * tiles run on the tensor cores (tcgen05.mma kind::tf32 with a three-term split for FP32-level products,
 * accumulators in tensor memory; mixed form only), 4 = block-form kernel (pivoting inside 32 x 32 diagonal
 * blocks, every update on the tensor cores, two 256-thread CTAs per SM; mixed form only); ctas_per_sm: CTAs per
 * SM of the 128-thread kernel (0 = all that fit).  The choices change the speed only: every choice computes the
 * same solves (the mixed ones to the refinement tolerance). */
typedef struct {
  int kernel;
  int ctas_per_sm;
  long long wait_limit; /* polls of each bounded wait on a copy or tensor-core tile inside an item (0 = default);
                           an item whose wait runs out is flagged DGA_ITEM_WAIT_TIMEOUT for the FP64 re-solve,
                           and the waits that drain the CTA's copies and tiles at exit always use the default.
                           A negative value is a test hook: each CTA first waits -wait_limit polls on a barrier
                           phase that nothing completes, so that wait runs out and the CTA takes the timeout
                           path (no further copies or tiles, every item of the CTA flagged) */
} dga_bse_tuning;

/* dga_bse_solve_sum_c128 (mixed = 0) or dga_bse_solve_sum_mixed_c128 (mixed = 1) with an explicit tuning;
 * status is required in the mixed form.  Scratch: dga_bse_tuned_scratch_bytes (0 if the tuning cannot run). */
size_t dga_bse_tuned_scratch_bytes(int N, int n2, int n_items, int mixed, const dga_bse_tuning* tuning);
int dga_bse_solve_sum_tuned_c128(int n_orb, int niv, int niw_half, int n_q, int n_ch, double beta, double inv_beta2,
                                 const void* gamma_cm, const void* chi0_inv, const void* uv, const int* work,
                                 int n_items, int mixed, int max_iter, double tol, void* out, int* status, int* iters,
                                 const dga_bse_tuning* tuning, void* scratch, size_t scratch_bytes,
                                 dga_stream_t stream);

/* One request of a heterogeneous BSE batch: the inputs and output of one dga_bse_solve_sum_c128 problem
 * (both channels; layouts as there) with its own frequency box, q set and beta. */
typedef struct {
  const void* gamma_cm; /* [2][W][N][N] column-major compound Gamma_r */
  const void* chi0_inv; /* [Q][W][nv][n2][n2] */
  const void* uv;       /* [2][Q][n2][n2] */
  void* out;            /* [2][Q][W][N][n2] */
  int n_orb, niv, niw_half, n_q;
  double beta, inv_beta2;
} dga_bse_problem;

/* Ladder BSE of several requests in ONE persistent launch (the serving path's continuous batch; the upstream
 * runs one create_auxiliary_chi_r_q_sum call per request, dgamore/nonlocal_sde.py:85-156).  Requests may differ
 * in niv, niw, Q, beta, inputs and n_orb (1..4), but every request must take the same default kernel
 * (dga_bse_default_kernel).  The 128-thread kernels (the FP64 form) and the mixed form's block kernel for 1 to 3
 * orbitals choose the right-hand-side count per item, so their requests share a launch whatever their orbital
 * counts; the shared-memory-panel kernels and the 4-orbital block kernel take one n_orb per launch.
 * probs_host: the descriptors on the host (launch
 * geometry); probs_dev: the same array copied to device memory; work: [n_items][4] ints (request, ch, q, w);
 * mode 0 runs the FP64 LU of dga_bse_solve_sum_c128, mode 1 the FP32 LU + FP64 refinement of
 * dga_bse_solve_sum_mixed_c128 (max_iter, tol), mode 2 the FP64 re-solve of the items a mode-1 launch flagged;
 * each item's result is bitwise the single-request result.  The launch uses at most scratch_bytes / slot CTAs
 * (a smaller scratch caps its footprint); dga_bse_batch_scratch_bytes gives the size for a full grid. */
size_t dga_bse_batch_scratch_bytes(const dga_bse_problem* probs_host, int n_prob, int n_items, int mode);
int dga_bse_solve_sum_batch_c128(const dga_bse_problem* probs_host, const void* probs_dev, int n_prob,
                                 const int* work, int n_items, int mode, int max_iter, double tol, int* status,
                                 int* iters, void* scratch, size_t scratch_bytes, dga_stream_t stream);

/* Allocation-free variant of dga_bse_solve_sum_c128 (no counterpart in the upstream, which has no device
 * code): for callers that cannot call cudaMalloc -- a host that binds only this C ABI and has no device
 * allocator, or a steady-state loop that must not trigger cudaMalloc's device-wide synchronisation.  The
 * working matrices live in a fixed DGA_BSE_NOALLOC_SCRATCH_BYTES (64 MiB) array inside the library, held by
 * every GPU that loads the library until exit; compound sizes N whose N*N + N*n2 complex slot does not fit
 * (N above about 2040) are rejected with DGA_ERR_SCRATCH.  The first call on a device looks up the array's
 * device address (it can load the module): make it before any stream capture.  Calls share the array, so
 * calls that overlap on the GPU race; calls ordered on one stream are safe.  Nothing needs clearing between
 * calls (every item rewrites its slot before reading it).  The looked-up address is kept per device for the life
 * of the process: after cudaDeviceReset (or after the primary context is released and created again) it is stale,
 * so do not use this entry point across a device reset. */
#define DGA_BSE_NOALLOC_SCRATCH_BYTES (64ull << 20)
int dga_bse_solve_sum_noalloc_c128(int n_orb, int niv, int niw_half, int n_q, int n_ch, double beta,
                                   double inv_beta2, const void* gamma_cm, const void* chi0_inv, const void* uv,
                                   const int* work, int n_items, void* out, int* status, dga_stream_t stream);

/* Generic FourPoint.invert_and_sum_over_last_vn (dgamore/four_point.py:620-642) on an explicit matrix in the
 * FourPoint layout [q][o1][o2][o3][o4][w][nu][nu']; out: [Q][W][N][n2]. */
int dga_invert_sum_dense_c128(int n_orb, int niv, int niw_half, int n_q, double beta, const void* mat, const int* work,
                              int n_items, void* out, int* status, void* scratch, size_t scratch_bytes,
                              dga_stream_t stream);

/* Physical susceptibility with the shell correction; replaces
 * nonlocal_sde.create_generalized_chi_q_with_shell_correction (dgamore/nonlocal_sde.py:167-182) with the nu sum
 * of nonlocal_sde.py:298.  X from dga_bse_solve_sum_c128; out: [n_ch][Q][W][n2][n2]. */
int dga_chi_phys_c128(const void* X, const void* uv, const void* full_sum, const void* core_sum, int n_orb,
                      int niv_core, int niw_half, int n_q, int n_ch, double beta, void* out, int* status,
                      dga_stream_t stream);

/* Hartree and Fock terms; replaces nonlocal_sde.get_hartree_fock (dgamore/nonlocal_sde.py:31-69) on the full,
 * ordered q list of one rank.  u: [n][n][n][n] local U; v_q: [Nq][n][n][n][n] V(q) over the full grid in
 * row-major (qx, qy, qz) order (Nq = Nk = nx*ny*nz); occ: [n][n] (config.sys.occ); occ_k: [Nk][n][n]
 * (config.sys.occ_k).  hartree: [n][n] = 2 sum_cd (U+V_(q=0))_abcd occ_dc; fock: [Nk][n][n] =
 * -1/Nq sum_q sum_cd (U+V_q)_abcd occ_k(k+q)_dc.  sigma (optional, [Nk][n][n][nv2]): hartree + fock is added
 * to every frequency, as calculate_self_energy_q does before returning (nonlocal_sde.py:884). */
int dga_hartree_fock_c128(const void* u, const void* v_q, const void* occ, const void* occ_k, int n_orb, int nx,
                          int ny, int nz, void* hartree, void* fock, void* sigma, int nv2, dga_stream_t stream);

/* Self-consistency glue (dgamore_b200/selfconsistency.py holds the host side).  sigma, g: [Nk][n][n][2 niv]
 * complex128 (compressed k, nu = (2m+1) pi/beta for m = -niv .. niv-1); ek: [Nk][n][n] complex128; n_orb 1..4.
 * dga_g_full_c128: G(k,nu) = [i nu + mu - e_k - Sigma(k,nu)]^-1, as GreensFunction.get_g_full
 *   (dgamore/greens_function.py:110-124).
 * dga_fill_sums_c128: s_out[k] = sum_nu Re G(k,nu) and t_out[k] = sum_nu Re [i nu + mu - e_k - s0]^-1 ([Nk][n][n]
 *   float64; s0: [n][n] float64, the self-energy's zeroth tail moment), the frequency sums behind get_total_fill
 *   and get_fill_nonlocal (greens_function.py:20-52, 212-240).
 * dga_sigma_kmean_c128: out[n][n][nvs] = mean over k of sigma[k][.][.][v0 .. v0+nvs), the k-average the tail-moment
 *   fit reads (SelfEnergy.fit_smom, dgamore/self_energy.py:51-75); nv = 2 niv. */
int dga_g_full_c128(const void* sigma, const void* ek, int n_orb, int nk, int niv, double mu, double beta, void* g,
                    dga_stream_t stream);
int dga_fill_sums_c128(const void* sigma, const void* ek, const double* s0, int n_orb, int nk, int niv, double mu,
                       double beta, double* s_out, double* t_out, dga_stream_t stream);
int dga_sigma_kmean_c128(const void* sigma, int n_orb, int nk, int nv, int v0, int nvs, void* out,
                         dga_stream_t stream);

/* Single-band lambda correction (FP64 Newton with delta halving); replaces lambda_correction.find_lambda and
 * perform_single_lambda_correction (dgamore/lambda_correction.py:28-73).  chi: [n_ch][Q][W]; weights: [Q]
 * multiplicities (irrk_count); target: [n_ch] complex; outputs lambda [n_ch], iterations, corrected chi. */
int dga_lambda_c128(const void* chi, int n_q, int niw_half, int n_ch, const long long* weights, const void* target,
                    double beta, double nk_tot, double delta, double eps, int maxiter, double* lambda_out,
                    int* iters_out, int* status, void* chi_out, dga_stream_t stream);

/* Three-leg vertex and SDE kernel: gamma_r = beta chi0^-1 X (nonlocal_sde.create_vrg_r_q, :159-164) and
 * K = -K_dc + K_dens + 3 K_magn with K_r = U_r (gamma - gamma U_r chi_r [- 2/3 1]) (calculate_kernel_r_q,
 * :201-215, summed as in :820-853).  K: [Q][W][nv][n2][n2]; gamma_out optional [2][Q][W][nv][n2][n2]. */
int dga_kernel_assembly_c128(const void* chi0_inv, const void* X, const void* uv, const void* chi_phys,
                             const void* k_dc, int n_orb, int niv_core, int niw_half, int n_q, double beta, void* K,
                             void* gamma_out, dga_stream_t stream);

/* Double-counting kernel; replaces nonlocal_sde.calculate_sigma_dc_kernel (dgamore/nonlocal_sde.py:185-198).
 * chi0: [Q][W][nvf][n2][n2]; u_perm: compound U_adcb / beta^2 [n2][n2]; fdc: [W][Nf][Nf] row-major compound
 * F_dc = 2 F_magn,loc permuted cbad; k_dc: [Q][W][nv][n2][n2]. */
size_t dga_dc_scratch_bytes(int n_orb, int niv_full, int niw_half, int n_q);
int dga_dc_kernel_c128(const void* chi0, const void* u_perm, const void* fdc, int n_orb, int niv_core, int niv_shell,
                       int niw_half, int n_q, void* k_dc, void* scratch, size_t scratch_bytes, dga_stream_t stream);

/* Schwinger-Dyson contraction through real space plus the inverse transform and the full-nu completion;
 * replaces nonlocal_sde.calculate_sigma_from_kernel_fft_cpu/_gpu/_auto (dgamore/nonlocal_sde.py:544-674) and the
 * caller's ifft().to_full_niv_range() (:876-879).  kern: [Q][W][nv][n2][n2]; g_r: [niv+2niw][n][n][Nk];
 * irrk_inv: [Nk]; out: [Nk][n][n][2niv]. */
size_t dga_sigma_scratch_bytes(int n_orb, int niv, int nk, int n_chunks);
int dga_sigma_c128(const void* kern, const void* g_r, int n_orb, int niv, int niw, int n_q, int nx, int ny, int nz,
                   const int* irrk_inv, const void* tw_inv, double beta, int n_chunks, void* out, void* scratch,
                   size_t scratch_bytes, dga_stream_t stream);

/* The real-space half of dga_sigma_c128: Sigma(R, nu >= 0) = -1/(2 beta Nk) sum_w sum_ad G_ad(R, nu - w)
 * K_aijd(-R, w, nu), the result of nonlocal_sde.calculate_sigma_from_kernel_fft_cpu/_gpu/_auto
 * (dgamore/nonlocal_sde.py:544-652) before the caller's ifft().to_full_niv_range(); out: [niv][n2][Nk] (planes
 * contiguous in R).  Arguments and scratch as dga_sigma_c128. */
int dga_sigma_rspace_c128(const void* kern, const void* g_r, int n_orb, int niv, int niw, int n_q, int nx, int ny,
                          int nz, const int* irrk_inv, const void* tw_inv, double beta, int n_chunks, void* out,
                          void* scratch, size_t scratch_bytes, dga_stream_t stream);

/* dga_dft_planes_c128 with the input point of output R read from gather[R]: the IBZ -> FBZ expansion
 * (IAmNonLocal._map_to_full_bz, dgamore/n_point_base.py:489-494) folded into the transform's load. */
int dga_dft_planes_gather_c128(const void* in, long long in_s_hi, long long in_s_lo, long long in_s_r, void* out,
                               long long out_s_hi, long long out_s_lo, long long out_s_r, int n_lo, int n_planes,
                               int nx, int ny, int nz, const void* tw, double scale, const int* gather,
                               dga_stream_t stream);

/* Eliashberg full vertex F_r(q, w) of both channels in the pp frequency box (P = niv_pp, Mb = n2*2P) for the
 * work items (ch, q, w < w_pp); replaces eliashberg_solver.create_full_vertex_q_r(_v2)
 * (dgamore/eliashberg_solver.py:78-298) up to the frequency transform.  Inputs as dga_bse_solve_sum_c128 plus
 * g3 = gamma_r [2][Q][W][nv][n2][n2] and chi_phys [2][Q][W][n2][n2] (lambda-corrected); out [2][Q][w_pp][Mb][Mb],
 * row (p=(a,b), nu), column (s=(d,c), nu'). */
size_t dga_eli_vertex_scratch_bytes(int n_orb, int niv, int niv_pp, int n_items);
int dga_eli_full_vertex_c128(int n_orb, int niv, int niw_half, int n_q, int niv_pp, int w_pp, double beta,
                             double inv_beta2, const void* gamma_cm, const void* chi0_inv, const void* uv,
                             const void* g3, const void* chi_phys, const int* work, int n_items, void* out,
                             int* status, void* scratch, size_t scratch_bytes, dga_stream_t stream);

/* The Eliashberg full vertex fused into the FP64 BSE: dga_bse_solve_sum_c128 (same inputs, X into out) whose items
 * with w < w_pp also solve the unit vectors of the pp box (niv_pp) with the item's own LU factors and write
 * out_pp [2][Q][w_pp][Mb][Mb] = beta^2 (delta c0 - c0 chi* c0), the chi* part of the vertex of
 * create_full_vertex_q_r(_v2) (dgamore/eliashberg_solver.py:78-298), without a second factorisation.
 * dga_eli_ladder_term_c128 adds the ladder term (U_r - U_r chi_r U_r) gamma_r gamma_r once the pass has the
 * lambda-corrected chi_r and the three-leg vertex, giving the out of dga_eli_full_vertex_c128. */
size_t dga_bse_eli_scratch_bytes(int N, int n2, int n_items);
int dga_bse_solve_sum_eli_c128(int n_orb, int niv, int niw_half, int n_q, int n_ch, double beta, double inv_beta2,
                               const void* gamma_cm, const void* chi0_inv, const void* uv, const int* work,
                               int n_items, int niv_pp, int w_pp, void* out, void* out_pp, int* status, void* scratch,
                               size_t scratch_bytes, dga_stream_t stream);
int dga_eli_ladder_term_c128(const void* uv, const void* g3, const void* chi_phys, int n_orb, int niv, int niw_half,
                             int n_q, int niv_pp, int w_pp, void* f, dga_stream_t stream);

/* PH -> PP (w = 0) transform, singlet/triplet combination and gap-equation layout; replaces
 * _transform_vertex_frequencies_w0 and the Gamma_sing/trip sums (dgamore/eliashberg_solver.py:44-75, 620-628).
 * fph: [2][Q][w_pp][Mb][Mb] from dga_eli_full_vertex_c128; out [2 (sing, trip)][Q][Mb][Mb] with
 * Mat[(a,b,nu)][(c,d,nu')] = Gamma[a,c,b,d](nu,nu'). */
int dga_eli_pairing_vertex_c128(const void* fph, int n_orb, int niv_pp, int n_q, int w_pp, void* out,
                                dga_stream_t stream);

/* chi0pp[Nk][2P][(a,b)][(c,d)] = G_ad(k,nu) conj(G_cb(k,nu)); replaces
 * BubbleGenerator.create_generalized_chi0_q_pp_w0 (dgamore/bubble_gen.py:268-279). */
int dga_eli_chi0pp_c128(const void* g_k, int n_orb, int niv_g, int niv_pp, int nk, void* out, dga_stream_t stream);

/* One application of the linearised gap equation, the matvec of solve_eliashberg_lanczos
 * (dgamore/eliashberg_solver.py:420-428): mat [Nk][M][M] = sign * FFT_q of the pairing vertex (full BZ),
 * chi0pp from dga_eli_chi0pp_c128, gap / gap_out [Nk][n2][2P]; sign = +1 singlet, -1 triplet. */
size_t dga_eli_matvec_scratch_bytes(int n_orb, int niv_pp, int nk);
int dga_eli_matvec_c128(const void* mat, const void* chi0pp, const void* gap, int n_orb, int niv_pp, int nx, int ny,
                        int nz, const void* tw_fwd, const void* tw_inv, double beta, double sign, void* gap_out,
                        void* scratch, size_t scratch_bytes, dga_stream_t stream);

/* dga_eli_matvec_c128 with Gamma(R) stored in complex64 (mat_c64 [Nk][M][M], made by dga_narrow_c128_to_c64):
 * half the bytes of the operator's dominant stream, every product and sum in FP64 and the vectors complex128,
 * so the Krylov normalisation and Rayleigh quotients stay FP64 (the power-iteration form of
 * solve_eliashberg_lanczos, dgamore/eliashberg_solver.py:420-428, with its operator in complex64 storage). */
int dga_eli_matvec_c64mat_c128(const void* mat_c64, const void* chi0pp, const void* gap, int n_orb, int niv_pp,
                               int nx, int ny, int nz, const void* tw_fwd, const void* tw_inv, double beta,
                               double sign, void* gap_out, void* scratch, size_t scratch_bytes, dga_stream_t stream);

/* dst[e] = complex64(src[e]) for e < n (round to nearest); no counterpart in the upstream. */
int dga_narrow_c128_to_c64(const void* src, void* dst, long long n, dga_stream_t stream);

/* ---- dense batched LU (the full inverses of the local Schwinger-Dyson equation) ---- */

/* LU with partial pivoting (LAPACK's pivot order, the zgetrf behind numpy.linalg.inv in LocalFourPoint.invert,
 * dgamore/local_four_point.py:298-310) of n_mat column-major N x N matrices a + m*mat_stride, in place (N <= 8192);
 * piv [n_mat][N]; status [n_mat]: DGA_ITEM_SINGULAR on an exact zero pivot. */
int dga_lu_batched_c128(void* a, int N, int n_mat, long long mat_stride, int* piv, int* status, dga_stream_t stream);

/* X_m = A_m^-1 B_m with the factors of dga_lu_batched_c128 for n_rhs right-hand sides B_m(r, k) =
 * b[m*b_stride_m + r*b_stride_r + k*b_stride_k] (b null: the identity, n_rhs <= N, giving the inverse), written
 * column-major (leading dimension N) to out + m*out_stride in blocks of 16 columns: out holds ceil(n_rhs/16)*16
 * columns, those past n_rhs solved for zero right-hand sides.  A non-finite element of X_m ORs DGA_ITEM_NONFINITE
 * into status[m]. */
int dga_lu_solve_batched_c128(const void* lu, const int* piv, int N, int n_mat, long long lu_stride, const void* b,
                              long long b_stride_m, long long b_stride_r, long long b_stride_k, int n_rhs, void* out,
                              long long out_stride, int* status, dga_stream_t stream);

/* ---- local Schwinger-Dyson equation (dgamore/local_sde.py:17-217), W = niw_core + 1 frequencies w >= 0 ----
 * Compound orbital index p = (a,b), s = (d,c); N = n^2 * 2 niv_core; matrices of both channels ordered
 * m = ch*W + w (ch 0 = density, 1 = magnetic); uv [2][n2][n2] = U_dens, U_magn (interaction.py:43-65). */

/* chi0[w][nu][p][s] = -beta G_ad(nu) G_cb(nu - w) over the box of 2*niv_box frequencies, entries with both parts
 * below 1e-12 set to zero; replaces BubbleGenerator.create_generalized_chi0 (dgamore/bubble_gen.py:20-30) in the
 * half w range.  g: [n][n][2 niv_g], niv_g >= niv_box + niw_half. */
int dga_local_bubble_c128(const void* g, int n_orb, int niv_g, int niw_half, int niv_box, double beta, void* chi0,
                          dga_stream_t stream);

/* chi_cm[w] (column-major compound N x N) = beta G2[a,b,c,d,w0+w,nu,nu'] - 2 beta G_ab(nu) G_cd(nu') at w = 0 if
 * dens; replaces create_generalized_chi (dgamore/local_sde.py:17-29).  g2: [n][n][n][n][n_wg][2niv][2niv] with
 * w = 0 at index w0 (w0 = niw for the full range, 0 for the half range). */
int dga_local_chi_c128(const void* g2, int n_orb, int niv, int niw_half, int w0, int n_wg, const void* g, int niv_g,
                       double beta, int dens, void* chi_cm, dga_stream_t stream);

/* ucorr[ch][w] = U_r - U_r [1 + (full_sum - core_sum) U_r]^-1 (n2 x n2; full/core sums [W][n2][n2] of
 * dga_chi0_prep_c128 with one q): the shell correction of create_gamma_r_with_shell_correction
 * (dgamore/local_sde.py:49-51) in closed form.  status [2][W]: DGA_ITEM_SINGULAR if the bracket is singular. */
int dga_local_ucorr_c128(const void* uv, const void* full_sum, const void* core_sum, int n_orb, int niw_half,
                         void* ucorr, int* status, dga_stream_t stream);

/* gamma_cm[m] = beta^2 chi_inv[m] - delta_{nu nu'} beta^2 chi0_inv[w][nu] + ucorr[m] (column-major compound, the
 * layout dga_bse_solve_sum_c128 reads); chi_inv column-major at m*inv_stride; chi0_inv [W][nv][n2][n2].  Replaces
 * create_gamma_r_with_shell_correction (dgamore/local_sde.py:40-51). */
int dga_local_gamma_c128(const void* chi_inv, long long inv_stride, const void* chi0_inv, const void* ucorr,
                         int n_orb, int niv, int niw_half, double beta, void* gamma_cm, dga_stream_t stream);

/* Operands of F = Gamma_u [1 + chi0 Gamma_u / beta^2]^-1 over the full box (create_full_vertex_from_gamma,
 * dgamore/local_sde.py:75-82): gamma_u (Gamma_r in the core box, U_r outside it, pad_with_u) and mt = the
 * transpose of 1 + chi0 Gamma_u / beta^2, both column-major [2W][Nf][Nf], Nf = n^2 * 2(niv_core + niv_shell);
 * chi0 [W][nvf][n2][n2] from dga_local_bubble_c128 over the full box.  F follows as the solve mt X = gamma_u^T
 * (X = F^T) of dga_lu_solve_batched_c128. */
int dga_local_fvertex_operands_c128(const void* gamma_cm, const void* uv, const void* chi0, int n_orb, int niv_core,
                                    int niv_shell, int niw_half, double beta, void* mt, void* gamma_u,
                                    dga_stream_t stream);

/* Local self-energy from the three-leg vertices vrg [2][W][nv][n2][n2] and susceptibilities chi_phys
 * [2][W][n2][n2] (get_loc_self_energy_vrg, dgamore/local_sde.py:150-172): sigma [n][n][2niv] = Hartree term
 * U_dens occ + the SDE sum over the full w range; u [n][n][n][n] (plain U), g [n][n][2niv_g], occ [n][n];
 * inner: scratch [W][nv][n2][n2]. */
int dga_local_sigma_c128(const void* vrg, const void* chi_phys, const void* uv, const void* u, const void* g,
                         const void* occ, int n_orb, int niv, int niw_half, int niv_g, double beta, void* inner,
                         void* sigma, dga_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* DGA_B200_H */
