/*
 * qsb200.h -- C ABI of the B200 (sm_100a) NEGF solver: QUICHOTTE's self-consistent
 * loop on the GPU (library libqsb200.so).
 *
 * The reference calls these steps from Fortran module procedures; each entry point below
 * names the reference interface it replaces (file:line, paths relative to the reference
 * project). A Fortran caller binds them with ISO_C_BINDING (an interface block of
 * bind(C) procedures with value/reference arguments as declared here); the argument
 * layout is the one the reference already uses:
 *   - matrices column-major, complex(dp) = two doubles (re, im);
 *   - packed SCF vectors in the layout of pack_gf (common/linear_algebra.f90:155-191)
 *     or pack_nil (src/scf.f90:226-240);
 *   - state indices 1-based where the reference stores indices (atom_first).
 * All host pointers are plain host memory; the library owns every device allocation
 * (made in qs_create, released in qs_destroy).
 *
 * Status convention: 0 = success; > 0 = a numerical condition the reference stops on
 * (e.g. a singular Dyson matrix: 1 + the 0-based energy index); < 0 = CUDA error or
 * HBM admission failure. The library never aborts the process. qs_last_error() gives
 * the message of the last failure on a handle.
 */
#ifndef QSB200_H
#define QSB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { QS_PREC_FP64 = 0, QS_PREC_MIXED = 1 };

/* Everything the reference's module globals hold when setup_storage runs
 * (src/green_functions.f90:43-67, src/scf.f90:38-43, src/parameters.f90). */
typedef struct qs_problem {
    int Norb, N_sites, N_atoms, order, n_omega;
    const double *H;       /* Norb*Norb complex, column-major                      */
    const double *GammaL;  /* Norb*Norb complex                                    */
    const double *GammaR;  /* Norb*Norb complex                                    */
    const double *U_site;  /* Norb (U on the spin-up index of a site)              */
    const double *omega;   /* n_omega energies                                     */
    const int *atom_norb;  /* N_atoms                                              */
    const int *atom_first; /* N_atoms, 1-based                                     */
    double mu, beta, delta;
    double alpha_mix, tolf, tolf_order1;
    int nhist, maxscf, single_history;
    int precision; /* QS_PREC_FP64 or QS_PREC_MIXED */
    int device;    /* CUDA device ordinal                                          */
} qs_problem;

typedef struct qs_scf_step {
    int step;
    double fmax, rms;
    int nh;
} qs_scf_step;

typedef struct qs_scf_result {
    int converged;  /* as solve_scf's `converged` (src/scf.f90:142-150)        */
    int n_iter;
    double fmax;
    int aborted;    /* SCF runaway inside broyden_solve                         */
    int runaway, unphysical, i_worst; /* final_sanity (src/scf.f90:260-275)     */
    double n_worst, w_worst;
    int n_resets;   /* Broyden history resets (ill-conditioned Gram matrix)     */
    qs_scf_step *log; /* caller buffer for the scf_V_<V>.dat lines, or NULL     */
    int log_cap, n_log;
    double seconds; /* device time of the solve                                 */
    int n_mixed;    /* QS_PREC_MIXED: leading steps whose residual used the FP32
                     * self-energies; the later steps, convergence included, are FP64 */
} qs_scf_result;

typedef struct qs_handle qs_handle;

/* setup_storage + scf_setup_sizes + sigma2_init (src/green_functions.f90:90-190,
 * src/scf.f90:61-68, src/self_energies.f90:91-106): active subspace, device storage. */
int qs_create(const qs_problem *p, qs_handle **h);
/* sigma2_finalize (src/self_energies.f90:108-113) and every other release. */
void qs_destroy(qs_handle *h);
const char *qs_last_error(const qs_handle *h);

/* solve_scf(Volt, fresh_start, converged) (src/scf.f90:78-151): converge at Volt, then
 * the final sweep. fresh_start = 0 continues from the last converged input. */
int qs_solve_scf(qs_handle *h, double Volt, int fresh_start, qs_scf_result *res);

/* Current(Volt, J_up, J_down) (src/observables.f90:22-39), from the last final sweep. */
int qs_current(qs_handle *h, double Volt, double *J_up, double *J_down);

/* Arrays the final sweep leaves for the host observables (src/scf.f90:136-139):
 * G_less_obs (Norb*Norb complex), dosd (Norb*n_omega), trU, trD (n_omega). Any
 * pointer may be NULL. */
int qs_get_observables(qs_handle *h, double *G_less_obs, double *dosd, double *trU, double *trD);

/* Sizes: n_vec (src/green_functions.f90:397-405), nA, Nf. */
int64_t qs_vector_length(const qs_handle *h);
int qs_active_states(const qs_handle *h);
int qs_fft_length(const qs_handle *h);

/* ---- finer entry points (one reference routine each; host arrays in and out) ---- */

/* sweep(M_INIT2) + pack_gf (src/scf.f90:116-122) at order 2, or the non-interacting
 * G^<(t=0) + pack_nil (src/scf.f90:103-110) at order 1: the fresh-start SCF vector. */
int qs_initial_vector(qs_handle *h, double Volt, double *x);

/* scf_residual2 / scf_residual1 (src/scf.f90:158-224): F = pack(G_out[x]) - x. On a
 * QS_PREC_MIXED handle the order-2 residual is evaluated as in the FP32 phase of its solves
 * (FP32 self-energies; Keldysh products on the tensor cores in 3xTF32 for 32 <= nA <= 128). */
int qs_residual(qs_handle *h, double Volt, const double *x, double *F, int *abort_flag);

/* unpack_gf + equal_time_lesser + sigma_first_order + sigma2_compute(.true.)
 * (src/self_energies.f90:45-72,135-219): Sigma2^r, Sigma2^< as (nA,nA,n_omega) complex
 * column-major, and Sigma1 (Norb*Norb complex); any output may be NULL. On a QS_PREC_MIXED
 * handle Sigma2 is formed as in the FP32 phase of its solves (FP32 transforms). */
int qs_self_energies(qs_handle *h, const double *x, double *SigR2, double *SigL2, double *Sig1);

/* invert_complex (common/linear_algebra.f90:58-88) over a batch: A holds `batch`
 * N x N complex column-major matrices, replaced by their inverses. info[b] = 0, or k+1
 * if pivot k of matrix b is zero (the reference's ZGETRF INFO > 0). */
int qs_invert_batched(int N, int batch, double *A, int *info, int precision);

/* ---- set-up (host arrays; each call allocates and frees its own device buffers and runs
 * on CUDA device `device`, or on the calling thread's current device if device < 0) ---- */

/* hermitian_eigensystem (common/linear_algebra.f90:32-56, LAPACK zheev) over a batch: A holds
 * `batch` N x N Hermitian complex column-major matrices (only their Hermitian part is used;
 * the diagonal's imaginary part is ignored) and is replaced by the eigenvectors, one per
 * column, in the order of E (`batch` x N eigenvalues, ascending). Parallel two-sided Jacobi on
 * the device. info[b] = 0, or 1 if matrix b did not converge or holds non-finite entries
 * (the reference's ZHEEV INFO > 0, where it stops). 1 <= N <= 2048, batch <= 65535. Returns 0,
 * 1 if some info[b] != 0, -1 for bad arguments, or a CUDA error (< 0). */
int qs_hermitian_eigensystem(int N, int batch, double *A, double *E, int *info, int device);

/* The same eigenvalues without the eigenvectors (zheev with JOBZ = 'N'), as the energy grid
 * needs them (src/quichotte.f90:81-83): A is not modified. For N <= 160 one thread block per
 * matrix, with the matrix in shared memory, reduces it to a real tridiagonal matrix by
 * Householder reflectors and finds the eigenvalues by Sturm-count multisection (one launch
 * for the batch; info[b] = 1 only for non-finite entries); larger N takes the path of
 * qs_hermitian_eigensystem. Same info, limits and returns. */
int qs_hermitian_eigenvalues(int N, int batch, const double *A, double *E, int *info, int device);

/* The dense linear algebra of build_hamiltonian_from_dftb_hs (src/hamiltonian.f90:625-689):
 * S (N x N real symmetric overlap) and H0 (N x N real, eV) as the reference holds them after
 * symmetrisation, Lam (2N x 2N complex, the p-shell SOC matrix, spin fastest);
 *   S^-1/2 = U diag(s^-1/2) U^T (for N > 160 from the eigenpairs of S; for N <= 160 the same
 *            matrix function by the coupled Newton-Schulz iteration, the step count fixed by
 *            the eigenvalues of S),
 *   Hao = H0 (x) I2 + (soc_dual ? (Sx2 Lam + Lam Sx2)/2 : Lam),   Sx2 = S (x) I2,
 *   H = (Sm2 Hao Sm2 + its conjugate transpose)/2,                 Sm2 = S^-1/2 (x) I2,
 * into H (2N x 2N complex). evmin receives the smallest eigenvalue of S. Returns 0, 1 if S is
 * not positive definite (evmin <= 1e-8: the reference stops there) or its eigenproblem did not
 * converge, -1 for bad arguments, or a CUDA error (< 0). 1 <= N <= 2048. */
int qs_dftb_lowdin(int N, const double *S, const double *H0, const double *Lam, int soc_dual, double *H,
                   double *evmin, int device);

/* pack_gf / unpack_gf (common/linear_algebra.f90:155-233) for nb x nb x Nw arrays. */
int qs_pack_gf(int nb, int Nw, const double *Gr, const double *Gl, double *out);
int qs_unpack_gf(int nb, int Nw, const double *in, double *Gr, double *Gl);

/* broyden_solve (common/broyden_mixing.f90:51-184) with a residual evaluated on the
 * host: residual(ctx, n, x, F, &abort) gets host arrays. The Broyden state lives on
 * the device. */
typedef void (*qs_residual_fn)(void *ctx, int64_t n, const double *x, double *F, int *abort_flag);
int qs_broyden_solve_host(qs_residual_fn residual, void *ctx, double *x, int64_t n, double alpha_mix,
                          int nhist, int maxscf, double tolf, int single_history, int *converged,
                          int *n_iter, double *fmax, qs_scf_step *log, int log_cap);

/* ---- inversion without allocation (no counterpart in the reference) ----
 * The batched inversion of qs_invert_batched for callers that cannot allocate GPU memory
 * (their device memory belongs to an enclosing application's pool or arena, or their
 * loop cannot take the synchronisation of cudaMalloc/cudaFree). A and info are DEVICE
 * pointers the caller owns: A holds `batch` N x N complex column-major matrices and is
 * replaced by their inverses; info[b] = 0, or k+1 for a zero pivot at step k. The work
 * runs asynchronously on `stream` (a cudaStream_t, NULL = legacy default stream); read info
 * after synchronising. The library allocates nothing: its workspace is a fixed 16 MiB
 * device array that every GPU loading the library holds until exit. Each call looks up
 * that array's address (cudaGetSymbolAddress) on the calling thread's current device; the
 * first call on a device may load the module there, so make it before any stream capture. All calls share the array, so
 * calls that overlap on the GPU (other streams or threads) race: serialise them. Limits:
 * 1 <= N <= 512 (else QS_ERR_NOALLOC_LIMIT, with a message on stderr). Returns 0 or a
 * CUDA error (< 0). */
enum { QS_ERR_NOALLOC_LIMIT = -1001 };
int qs_invert_batched_noalloc(int N, int batch, double *A, int *info, void *stream);

/* ---- memory (setup_storage's memory estimate, src/green_functions.f90:90-190) ---- */

/* Device memory (GiB) a solve of this problem keeps from qs_create to qs_destroy: the
 * allocations of qs_create, computed on the host without a device. */
int qs_estimate_bytes(const qs_problem *p, double *gib);
/* Device memory (GiB) the handle has allocated. */
double qs_device_bytes(const qs_handle *h);

/* ---- serving (no counterpart in the reference, whose program solves the voltages of one
 * model one after another, src/quichotte.f90:125-143) ----
 * A request is one IV point: a problem (model + energy grid, arrays copied at submit) and
 * a voltage, solved from a fresh start as qs_create + qs_solve_scf + qs_current. Requests
 * are admitted in arrival order as soon as a worker is free and the estimated device
 * memory of the solve fits into the budget left by the solves in flight; admitted solves
 * keep their state on the device and run concurrently on their own streams and threads
 * (continuous batching). A request that exceeds the whole budget is refused at submit
 * (QS_ERR_TOO_LARGE). Times are seconds on the server's clock (qs_server_clock). */
enum { QS_ERR_TOO_LARGE = -1002 };
typedef struct qs_server qs_server;
typedef struct qs_server_config {
    int device;
    int max_inflight;      /* solves on the device at once, 1..64                    */
    double hbm_budget_gib; /* admission budget; <= 0: 90% of the free HBM at creation */
} qs_server_config;
typedef struct qs_request_result {
    int64_t id;
    int status;            /* 0, or the qs_create / qs_solve_scf status               */
    int converged, n_iter, n_mixed;
    double fmax, J_up, J_down;
    double solve_s;        /* device time of the solve                                */
    double t_arrival, t_start, t_done; /* submit, admission, completion              */
    double device_gib;     /* admitted memory (estimate + headroom)                  */
    char error[160];       /* qs_last_error of a failed request, else empty           */
} qs_request_result;
int qs_server_create(const qs_server_config *cfg, qs_server **s);
int qs_server_submit(qs_server *s, const qs_problem *p, double V, int64_t id);
/* Copies up to cap finished results into out, waiting up to timeout_s for the first. */
int qs_server_poll(qs_server *s, qs_request_result *out, int cap, double timeout_s);
int qs_server_pending(qs_server *s); /* submitted and not yet returned by poll */
double qs_server_clock(const qs_server *s);
double qs_server_budget_gib(const qs_server *s);
/* Waits for the solves in flight; queued requests that were never admitted are dropped. */
void qs_server_destroy(qs_server *s);

/* ---- autotuner (no counterpart in the reference) ----
 * Kernel variants whose relative speed depends on the size (kind 0: Dyson, blocked tensor-
 * core (variant 1: in shared memory, one block per SM, or in the global workspace above the
 * shared-memory limit; variant 3: in the global workspace, two blocks per SM) or unblocked
 * Gauss-Jordan (2); kind 1: Keldysh, tensor-core or CUDA-core GEMMs; kinds 2
 * and 3: the tile width 4 or 2 of the persistent Sigma2 kernels A and C, +2^20 in the key
 * for the FP32 ones; kind 4: the Keldysh step of a mixed solve's FP32 phase, variant 3 the
 * 3xTF32 kernel on the fifth-generation tensor cores, 1 / 2 the FP64 ones) are timed on the
 * first launch at a new size and the fastest is kept for the process.
 * qs_autotune(1) tunes (default), qs_autotune(0) uses the size heuristics only, 2 / 3 force
 * the first (kind 4: the 3xTF32 kernel; else the tensor-core / blocked variant) / last
 * applicable variant, 4 the second of three (kind 0: variant 3; kind 4: the FP64 tensor-core
 * kernel), qs_autotune(-1) forgets the recorded choices. qs_tuned_choice returns
 * the recorded variant (1, 2 or 3) or -1; a decision
 * is keyed by size = order + 1024 * floor(log2(n_omega)) (order N for Dyson, nA for Keldysh). */
int qs_autotune(int mode);
int qs_tuned_choice(int kind, int size);

/* ---- instrumentation (no counterpart in the reference, whose only timer is the
 * wall clock of src/quichotte.f90:50-58) ---- */

/* Number of kernels this library has launched in the process so far (the kernels of a
 * replayed CUDA graph included). */
int64_t qs_kernel_launches(void);

/* SCF residuals of this handle replayed from a CUDA graph: the FP64 residual's launches
 * (G^<(t=0), Sigma2, Dyson, Keldysh, the sanity sums) are captured once per (x, F, V) buffer
 * pair and replayed by the Broyden loop (not while per-launch profiling is on). */
int64_t qs_graph_replays(const qs_handle *h);

/* Per-kernel-family device time measured with CUDA events on the solver's stream.
 * enable = 1 starts recording, 0 stops, -1 only reads and resets. Fills ms[f] and
 * launches[f] for f < nfam (families: 0 Dyson, 1 Keldysh, 2-4 Sigma2 FFT kernels A/B/C,
 * 5 final-sweep outputs, 6 Broyden, 7 reductions, 8 other). Returns the family count. */
int qs_profile(qs_handle *h, int enable, double *ms, int64_t *launches, int nfam);

#ifdef __cplusplus
}
#endif
#endif
