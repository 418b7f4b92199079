// qs_common.cuh -- shared definitions of the B200 NEGF solver.
//
// Device data layout (HBM), with nA active states, n energies, Nf padded FFT length:
//   X, F, Fold, xold   SCF vectors, energy-major: block w (3 nA^2 doubles) holds
//                      [ G^r  nA^2 complex, column-major, (re,im) interleaved
//                      | G^< strict upper triangle, column by column, complex
//                      | Im G^<_ii, nA doubles ].
//                      This is a fixed permutation of the reference's pack_gf block
//                      (common/linear_algebra.f90:155-191), so every Broyden quantity
//                      (norms, dots, updates) is the reference's up to summation order.
//   SigR, SigL         Sigma2^r, Sigma2^< as n blocks of nA x nA complex, column-major
//                      (the reference's SigR2(nA,nA,n_omega)).
//   Y, V               FFT intermediates, sequence-major: sequence s holds Nf complex
//                      values ordered [l1][m2] of the four-step split Nf = N1*N2.
//   gRd, gLd           diagonals (n x nA complex) for the sanity check.
//   onsL, dosd, atomL, trU, trD   final-sweep arrays, energy-major (reference layout).
#pragma once
#include <functional>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "qsb200.h"

namespace qs {

template <typename T>
struct __align__(2 * sizeof(T)) cplx {
    T x, y;
};
using zc = cplx<double>;
using cc = cplx<float>;

template <typename T> __host__ __device__ __forceinline__ cplx<T> mk(T a, T b) { return cplx<T>{a, b}; }
template <typename T> __host__ __device__ __forceinline__ cplx<T> operator+(cplx<T> a, cplx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T> __host__ __device__ __forceinline__ cplx<T> operator-(cplx<T> a, cplx<T> b) { return {a.x - b.x, a.y - b.y}; }
template <typename T> __host__ __device__ __forceinline__ cplx<T> operator-(cplx<T> a) { return {-a.x, -a.y}; }
template <typename T> __host__ __device__ __forceinline__ cplx<T> operator*(cplx<T> a, cplx<T> b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T> __host__ __device__ __forceinline__ cplx<T> operator*(T s, cplx<T> a) { return {s * a.x, s * a.y}; }
template <typename T> __host__ __device__ __forceinline__ cplx<T> conj(cplx<T> a) { return {a.x, -a.y}; }
// a += b*c (complex fused multiply-add)
template <typename T> __host__ __device__ __forceinline__ void cfma(cplx<T> &a, cplx<T> b, cplx<T> c) {
    a.x = fma(b.x, c.x, a.x);
    a.x = fma(-b.y, c.y, a.x);
    a.y = fma(b.x, c.y, a.y);
    a.y = fma(b.y, c.x, a.y);
}
// a += b*conj(c)
template <typename T> __host__ __device__ __forceinline__ void cfma_conj(cplx<T> &a, cplx<T> b, cplx<T> c) {
    a.x = fma(b.x, c.x, a.x);
    a.x = fma(b.y, c.y, a.x);
    a.y = fma(-b.x, c.y, a.y);
    a.y = fma(b.y, c.x, a.y);
}
template <typename T> __host__ __device__ __forceinline__ T cabs1(cplx<T> a) { return fabs(a.x) + fabs(a.y); }
// 1/a by Smith's method (no overflow for |a| near the range limits)
template <typename T> __device__ __forceinline__ cplx<T> crecip(cplx<T> a) {
    if (fabs(a.x) >= fabs(a.y)) {
        T r = a.y / a.x, d = a.x + a.y * r;
        return {T(1) / d, -r / d};
    } else {
        T r = a.x / a.y, d = a.y + a.x * r;
        return {r / d, T(-1) / d};
    }
}
template <typename D, typename S> __host__ __device__ __forceinline__ cplx<D> cvt(cplx<S> a) { return {(D)a.x, (D)a.y}; }

// FP64 tensor-core MMA, D = A B + D with A 16x16 (row), B 16x8 (col), f64 accumulate.
// Fragments (g = lane/4, t = lane%4): a_i = A(g + 8(i&1), t + 4(i>>1)), i < 8;
// b_i = B(t + 4i, g), i < 4; c_i = C(g + 8(i>>1), 2t + (i&1)), i < 4.
// (not volatile: the compiler may schedule independent MMAs between dependent ones)
__device__ __forceinline__ void dmma16816(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
    asm(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
        "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]), "d"(b[1]),
          "d"(b[2]), "d"(b[3]));
}
// complex 16x8 tile update C += A B from split real/imaginary fragments (4 real MMAs)
__device__ __forceinline__ void zmma16816(double (&cr)[4], double (&ci)[4], const double (&ar)[8], const double (&ai)[8],
                                          const double (&br)[4], const double (&bi)[4]) {
    double nai[8];
#pragma unroll
    for (int k = 0; k < 8; k++) nai[k] = -ai[k];
    dmma16816(cr, ar, br);
    dmma16816(cr, nai, bi);
    dmma16816(ci, ar, bi);
    dmma16816(ci, ai, br);
}

constexpr double PI = 3.14159265358979323846;
constexpr int SMEM_MAX = 232448;  // max dynamic shared memory per block on sm_100 (227 KB)

// The Gauss-Jordan kernel keeps the N x N complex matrix in shared memory when it fits
// next to its ~1.3 KB of static shared memory (N <= 120 in FP64).
inline bool dyson_fits_smem(int N) { return (size_t)N * N * 16 + 1536 <= (size_t)SMEM_MAX; }

// FFT plan of one length L that divides Nf (radices applied in order).
struct FftLen {
    int L;
    int nrad;
    unsigned code;  // radix of pass p in bits 4p..4p+3
    int rad[8];     // the same radices (host side)
};

// Stockham plan for Nf = N1 * N2 and the twiddle table W[k] = exp(-2 pi i k / Nf).
struct FftPlan {
    int Nf, N1, N2;
    FftLen p1, p2;
};

// ---------------------------------------------------------------------------------
// The solver handle (one per qs_create).
// ---------------------------------------------------------------------------------
struct DeviceBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

}  // namespace qs

namespace qs {
// kernel families timed by the optional profiler (qs_profile)
enum KernelFamily { K_DYSON = 0, K_KELDYSH, K_SIG2A, K_SIG2B, K_SIG2C, K_FINAL, K_BROYDEN, K_REDUCE, K_OTHER, K_NFAM };
}  // namespace qs

struct qs_handle {
    // optional per-launch CUDA-event timing on the solver stream
    bool prof_on = false;
    std::vector<cudaEvent_t> prof_ev;           // pool, 2 per timed launch
    std::vector<int> prof_fam;                  // family of launch i (events 2i, 2i+1)
    double prof_ms[qs::K_NFAM] = {0};
    int64_t prof_count[qs::K_NFAM] = {0};
    // problem (host copies)
    int Norb = 0, N_sites = 0, N_atoms = 0, order = 0, n = 0, device = 0, precision = 0;
    double mu = 0, beta = 0, delta = 0, alpha_mix = 0.5, tolf = 1e-6, tolf_order1 = 1e-8;
    int nhist = 16, maxscf = 300;
    double mixed_switch = 1e-4;  // QS_PREC_MIXED: FP32 max|F| below which the residual turns FP64
    bool single = true;
    std::vector<double> H, GammaL, GammaR, U_site, omega;  // complex arrays as double pairs
    std::vector<int> atom_norb, atom_first;
    // active subspace (setup_storage), 0-based indices
    int nA = 0, nS = 0, nCL = 0, nAs = 0, n_int_sites = 0;
    std::vector<int> act, pos, sup, cl, asite;
    std::vector<char> site_int, site_act;
    bool has_atomL = false;
    std::vector<int> atom_off;
    int64_t n_vec = 0, nblk = 0;
    // device model arrays
    qs::zc *d_Hemb = nullptr, *d_Sig1 = nullptr, *d_GamLs = nullptr, *d_GamRs = nullptr, *d_GamLcl = nullptr;
    int *d_pos = nullptr;
    int *d_kd_cidx = nullptr;  // contact states of GamLs / GamRs (the lead terms of SL)
    int kd_nc = -1;
    int *d_act = nullptr, *d_sup = nullptr, *d_cl = nullptr, *d_atom_first = nullptr, *d_atom_norb = nullptr,
        *d_atom_off = nullptr, *d_site_int = nullptr;
    double *d_omega = nullptr, *d_U = nullptr;
    // SCF vectors and Broyden history (order 2: n_vec doubles; order 1: tiny)
    double *d_x = nullptr, *d_F = nullptr, *d_Fold = nullptr, *d_xold = nullptr;
    void *d_hdF = nullptr, *d_hU = nullptr;  // nhist columns, float (single history) or double
    // second-order self-energies and the FFT
    qs::FftPlan fft{};
    qs::zc *d_tw = nullptr;  // Nf twiddles
    qs::zc *d_SigR = nullptr, *d_SigL = nullptr;
    qs::zc *d_Y = nullptr, *d_V = nullptr;
    size_t nY = 0, nV = 0;
    int2 *d_ydesc = nullptr;  // per Y sequence: offsets of (re, im) in a DL block (-1 = zero)
    double *sig2_Upair = nullptr;  // U_I U_J hbar^2 (delta/2pi)^2 / Nf per site pair
    int2 *sig2_pairs = nullptr;    // interacting site pairs I <= J
    int sig2_npairs = 0, sig2_SA = 1, sig2_GA = 1, sig2_GC = 1;
    // sweep scratch
    qs::zc *d_G = nullptr;  // Dyson output (G_AA for all energies, or full G for a chunk)
    size_t G_chunk = 0;     // energies per chunk in full-G mode
    qs::zc *d_T = nullptr;  // per-CTA GEMM scratch
    size_t T_slots = 0, T_bytes = 0;
    qs::zc *d_Gws = nullptr;  // Gauss-Jordan workspace when N x N does not fit in shared memory
    size_t ws_slots = 0;
    qs::zc *d_gRd = nullptr, *d_gLd = nullptr, *d_onsL = nullptr, *d_atomL = nullptr;
    double *d_dosd = nullptr, *d_trU = nullptr, *d_trD = nullptr;
    qs::zc *d_Glt0 = nullptr;  // G^<(t=0) on-site blocks, 4 per site
    double *d_red = nullptr;   // reduction scratch
    size_t red_len = 0;
    int *d_info = nullptr;     // first singular energy (+1), 0 if none
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // host state
    std::vector<double> G_less_t0, G_less_obs, Sig1;  // Norb*Norb complex
    double J_up = 0, J_down = 0;
    bool have_x = false, final_done = false;
    std::vector<double> x1_host;  // order-1 SCF vector
    std::string err;
    size_t bytes_allocated = 0;
    std::vector<void *> allocs;
    // CUDA graphs of the FP64 residual's launches, one per (x, F, V) the Broyden loop uses
    // (x and F alternate between two buffers each): replayed instead of re-launching
    struct ResidualGraph {
        const double *x = nullptr;
        double *F = nullptr;
        double V = 0.0;
        cudaGraphExec_t exec = nullptr;
        int64_t launches = 0;  // kernels in the graph (added to the launch count per replay)
    };
    ResidualGraph graphs[2];
    int graph_next = 0;
    bool graphs_off = false;   // a capture failed: eager launches from then on
    int64_t graph_replays = 0;
};

namespace qs {

// error handling: every CUDA call inside the library goes through this
#define QS_CUDA(h, call)                                                                        \
    do {                                                                                        \
        cudaError_t _e = (call);                                                                \
        if (_e != cudaSuccess) {                                                                \
            (h)->err = std::string(#call) + ": " + cudaGetErrorString(_e);                      \
            return -(int)_e;                                                                     \
        }                                                                                       \
    } while (0)

int dalloc(qs_handle *h, void **p, size_t bytes);
// The dynamic shared-memory cap of a kernel is a process-wide attribute: it is always set
// to the device maximum (a cap, not a reservation), so that handles that size the same
// kernel differently, on other threads, never lower it under each other's launches.
inline cudaError_t smem_cap(const void *kernel) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(SMEM_MAX - fa.sharedSizeBytes));
}

// every kernel launch of the library is counted (qs_kernel_launches)
void count_launch();
void count_launches(int64_t k);
// bracket a launch with events when profiling is on: idx = prof_begin(...); launch; prof_end(h, idx)
int prof_begin(qs_handle *h, int fam, bool count = true);
void prof_end(qs_handle *h, int idx);

__device__ __forceinline__ double fermi_d(double w, double V, double mu, double beta) {
    // src/green_functions.f90:74-84 (hbar = 1)
    double arg = (w - mu + V) * beta;
    return 1.0 / (exp(fmin(arg, 700.0)) + 1.0);
}

// arguments of the Keldysh kernels (sweep modes M_INIT2 / M_SCF2)
struct KeldyshArgs {
    int nA, n;
    int64_t nblk;
    const zc *G;     // G_AA per energy (nA^2 complex)
    const zc *SigL;  // Sigma2^< per energy, or nullptr
    const zc *GamLs, *GamRs;
    const double *omega;
    double V, mu, beta;
    double *out;        // DL blocks (SCF vector)
    const double *xsub; // subtracted (F = out - x), or nullptr
    zc *gRd, *gLd;      // diagonals, or nullptr
    zc *Tws;            // per-block scratch, nA^2 complex
    int *err;           // set to 1 if a bounded tensor-core wait gave up (tcgen05 kernel)
    const int *cidx;    // the contact states: rows/columns where GamLs or GamRs is non-zero
    int nc;             // their number (-1: not known)
};
// the FP32-phase Keldysh step of a QS_PREC_MIXED solve on the fifth-generation tensor cores
// (keldysh_tf32.cu): 32 <= nA <= 128; returns -1 for other sizes
int launch_keldysh_tf32(qs_handle *h, const KeldyshArgs &k);
bool keldysh_tf32_fits(int nA);

// launchers (implemented in the .cu files)
int sigma2_setup(qs_handle *h);
// fp32: FFTs, 2x2 algebra and spectra in FP32 (QS_PREC_MIXED handles), Sigma written in FP64
int sigma2_compute(qs_handle *h, const double *d_x, bool fp32 = false);
// autotuner (autotune.cu): kinds of decisions and the variants they choose between
// TUNE_KELDYSH32: the Keldysh step of a mixed solve's FP32 phase, where the 3xTF32 tensor-core
// kernel (keldysh_tf32.cu) competes with the two FP64 ones
enum TuneKind { TUNE_DYSON = 0, TUNE_KELDYSH = 1, TUNE_SIG2_A = 2, TUNE_SIG2_C = 3, TUNE_KELDYSH32 = 4 };
// DYSON_BLOCKED2: the blocked Gauss-Jordan with its matrix in the global workspace, two
// 8-warp blocks per SM
enum { DYSON_BLOCKED = 1, DYSON_UNBLOCKED = 2, DYSON_BLOCKED2 = 3, KELDYSH_TC = 1, KELDYSH_CUDA = 2, KELDYSH_TF32 = 3 };
// the size key of a decision: the matrix order and the octave of the grid length (how many
// energies each SM gets changes which variant wins)
inline int tune_key(int order, int n) {
    int lg = 0;
    while ((2 << lg) <= n) lg++;
    return order + 1024 * lg;
}
int tune_get(int kind, int size);
bool tune_enabled();
void tune_put(int kind, int size, int choice);
// launch(cand[c]) for the recorded choice of (kind, size); the first time, every candidate
// is launched and timed and the fastest recorded. fallback: the choice without tuning.
int tune_launch(qs_handle *h, int kind, int size, const int *cand, int ncand, int fallback,
                const std::function<int(int)> &launch);
// max |v_i| over a device vector (uses the Broyden reduction scratch)
int vec_maxabs(qs_handle *h, const double *d_v, int64_t n, double &mx);
int equal_time_lesser_sigma1(qs_handle *h, const double *d_x);
enum SweepMode { M_INIT2 = 1, M_SCF2 = 2, M_SCF1 = 3, M_FINAL = 4 };
// fp32: the FP32 phase of a QS_PREC_MIXED solve (M_SCF2 only: tensor-core Keldysh products)
int sweep(qs_handle *h, int mode, double V, bool use_sigma, double *d_out, const double *d_x, bool fp32 = false);
int sum_over_energies(qs_handle *h, const zc *d_A, int64_t ld, int ncols, int64_t nrows, zc *d_out);
int sum_over_energies_real(qs_handle *h, const double *d_A, int64_t ld, int ncols, int64_t nrows, double *d_out);
int invert_batched_dev(cudaStream_t st, int N, int batch, zc *d_A, int *d_info, zc *d_ws, int ws_slots);
int invert_batched_ws(cudaStream_t st, int N, int batch, zc *d_A, int *d_min_info, int *d_info_each, zc *d_ws,
                      int ws_slots);
int convert_ref_to_dl(cudaStream_t st, int nA, int64_t Nw, const double *ref, double *dl);
int convert_dl_to_ref(cudaStream_t st, int nA, int64_t Nw, const double *dl, double *ref);

// check_diag_sanity (common/scf_checks.f90:59-91) from the per-state sums over energies:
// sumL[i] = sum_w G^<_ii(w), sumRim[i] = sum_w Im G^r_ii(w); state_index maps i to the
// reported (0-based) state label, or nullptr for i itself
struct SanityOut {
    bool runaway = false, unphysical = false;
    int i_worst = 1;
    double n_worst = 0.5, w_worst = 1.0;
};
SanityOut check_diag_sanity(int nb, const std::vector<zc> &sumL, const std::vector<double> &sumRim, double delta,
                            const int *state_index);
void release_all(qs_handle *h);

// Broyden (common/broyden_mixing.f90) on device vectors; the residual is a host callback
// that fills F (device) from x (device) and may set abort.
struct BroydenResidual {
    virtual int operator()(const double *d_x, double *d_F, bool &abort) = 0;
    // true if the residual just evaluated used another precision than the one before: the
    // (dF, u) pair of this step would mix two different residual functions and is not
    // stored, and the history built on the other function is dropped
    virtual bool precision_changed() const { return false; }
    virtual ~BroydenResidual() = default;
};
struct BroydenOut {
    bool converged = false;
    int n_iter = 0, n_resets = 0;
    double fmax = 0;
    bool aborted = false;
    std::vector<qs_scf_step> log;
};
// column stride (elements) of the Broyden history: n rounded up to a multiple of 4, so that
// every column starts on a 16-byte boundary for the kernels' 4-wide vector accesses
inline int64_t broyden_ld(int64_t n) { return (n + 3) & ~(int64_t)3; }
int broyden_solve_dev(qs_handle *h, BroydenResidual &res, double *&d_x, double *&d_F, double *&d_Fold,
                      double *&d_xold, void *d_hdF, void *d_hU, int64_t n, double alpha_mix, int nhist, int maxscf,
                      double tolf, bool sp, BroydenOut &out);

}  // namespace qs
