// oracle.cpp -- CPU oracle for QUICHOTTE's self-consistent NEGF loop.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker of the B200 solver: the tests,
// __graft_entry__.smoke() and the cpu_baseline leg of bench.py call it; nothing in the
// shipped library links or calls it.
//
// It is a line-by-line FP64 restatement of the reference's hot path, with OpenMP where
// the reference has OpenMP, LAPACK (zgetrf/zgetri/dposv) and BLAS dnrm2 from the
// OpenBLAS that ships inside the numpy wheel (the reference links OpenBLAS), and a
// project-written mixed-radix Stockham FFT in place of FFTW3 (same sign and scaling
// conventions: forward e^{-2 pi i jk/N}, backward e^{+2 pi i jk/N}, both unnormalised).
//
// Every routine cites the reference routine it follows (paths relative to the reference
// project). Parity is pinned by the reference's own 10 physics golden cases
// (tests/cases/*/reference), compared at its runner's tolerance (tests/run_tests.f90:14).
//
// Exported as qso_* with the signatures of include/qsb200.h.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../include/qsb200.h"

using cplx = std::complex<double>;
static const cplx IM(0.0, 1.0);
static const double PI = 3.14159265358979323846;
static const double HBAR = 1.0;  // common/constants.f90:19

// ------------------------------------------------------------------------------------
// LAPACK / BLAS from the numpy wheel's OpenBLAS (ILP64, symbol suffix 64_)
// ------------------------------------------------------------------------------------
extern "C" {
void scipy_zgetrf_64_(const int64_t *m, const int64_t *n, cplx *a, const int64_t *lda, int64_t *ipiv, int64_t *info);
void scipy_zgetri_64_(const int64_t *n, cplx *a, const int64_t *lda, const int64_t *ipiv, cplx *work,
                      const int64_t *lwork, int64_t *info);
void scipy_dposv_64_(const char *uplo, const int64_t *n, const int64_t *nrhs, double *a, const int64_t *lda,
                     double *b, const int64_t *ldb, int64_t *info, size_t uplo_len);
double scipy_dnrm2_64_(const int64_t *n, const double *x, const int64_t *incx);
void scipy_openblas_set_num_threads64_(int n);
}

static double dnrm2(int64_t n, const double *x) {
    const int64_t one = 1;
    return scipy_dnrm2_64_(&n, x, &one);
}

// invert_complex (common/linear_algebra.f90:58-88): zgetrf + zgetri with a workspace
// query; returns INFO (the reference stops on INFO /= 0).
static int64_t invert_complex(int N, cplx *A) {
    int64_t n = N, info = 0, lwork = -1;
    std::vector<int64_t> ipiv(N);
    scipy_zgetrf_64_(&n, &n, A, &n, ipiv.data(), &info);
    if (info != 0) return info;
    cplx wq;
    scipy_zgetri_64_(&n, A, &n, ipiv.data(), &wq, &lwork, &info);
    lwork = (int64_t)wq.real();
    std::vector<cplx> work(std::max<int64_t>(lwork, 1));
    scipy_zgetri_64_(&n, A, &n, ipiv.data(), work.data(), &lwork, &info);
    return info;
}

// ------------------------------------------------------------------------------------
// Mixed-radix (2,3,4,5,7,8) Stockham FFT, FFTW conventions (the reference plans
// dfftw_plan_dft_1d FORWARD/BACKWARD, src/self_energies.f90:102-103).
// ------------------------------------------------------------------------------------
struct FFTPlan {
    int n = 0;
    std::vector<int> radix;
    std::vector<cplx> tw;  // tw[k] = exp(-2 pi i k / n)
    // power-of-two lengths: radix-4 Stockham stages (one radix-2 stage first when log2 n
    // is odd), stage s with span L holding the twiddles w^(j*n/(4L)), j < L, contiguously
    bool pow2 = false;
    std::vector<int> p2_span;             // L of each radix-4 stage
    std::vector<std::vector<cplx>> p2_tw;  // per stage: [w1, w2, w3] for j = 0..L-1
    void init(int nn) {
        n = nn;
        radix.clear();
        int m = n;
        for (int r : {8, 4, 2, 3, 5, 7})
            while (m % r == 0) { radix.push_back(r); m /= r; }
        tw.resize(n);
        for (int k = 0; k < n; k++) {
            long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)n;
            tw[k] = cplx((double)cosl(a), (double)sinl(a));
        }
        pow2 = n >= 4 && (n & (n - 1)) == 0;
        p2_span.clear();
        p2_tw.clear();
        if (pow2) {
            int L = ((__builtin_ctz(n) & 1) ? 2 : 1);
            for (; L < n; L *= 4) {
                std::vector<cplx> t(3 * (size_t)L);
                const int step = n / (4 * L);
                for (int j = 0; j < L; j++)
                    for (int q = 1; q <= 3; q++) t[3 * (size_t)j + q - 1] = tw[(size_t)q * j * step];
                p2_span.push_back(L);
                p2_tw.push_back(std::move(t));
            }
        }
    }
    // power-of-two transform: Stockham autosort, out of place between x and work
    void exec_pow2(cplx *x, cplx *work, int sign) const {
        cplx *a = x, *b = work;
        int L = 1;
        if (__builtin_ctz(n) & 1) {  // radix-2 stage: b[2j + {0,1}] from a[j], a[j + n/2]
            const int h = n / 2;
            for (int j = 0; j < h; j++) {
                cplx u = a[j], v = a[j + h];
                b[2 * j] = u + v;
                b[2 * j + 1] = u - v;
            }
            std::swap(a, b);
            L = 2;
        }
        // stage with span L: input a viewed as [4][n/4] blocks of sub-transforms of length L
        // (element (r, k*L + j)), output b as sub-transforms of length 4L (k*4L + q*L + j)
        for (size_t s = 0; s < p2_span.size(); s++) {
            L = p2_span[s];
            const cplx *t = p2_tw[s].data();
            const int m4 = n / 4, K = m4 / L;
            for (int k = 0; k < K; k++)
                for (int j = 0; j < L; j++) {
                    cplx w1 = t[3 * j], w2 = t[3 * j + 1], w3 = t[3 * j + 2];
                    if (sign > 0) { w1 = std::conj(w1); w2 = std::conj(w2); w3 = std::conj(w3); }
                    const int i0 = k * L + j;
                    cplx v0 = a[i0], v1 = a[i0 + m4] * w1, v2 = a[i0 + 2 * m4] * w2, v3 = a[i0 + 3 * m4] * w3;
                    cplx s02 = v0 + v2, d02 = v0 - v2, s13 = v1 + v3, d13 = v1 - v3;
                    // multiply d13 by -i (forward) or +i (backward)
                    cplx rd13 = sign < 0 ? cplx(d13.imag(), -d13.real()) : cplx(-d13.imag(), d13.real());
                    cplx *o = b + (size_t)k * 4 * L + j;
                    o[0] = s02 + s13;
                    o[L] = d02 + rd13;
                    o[2 * L] = s02 - s13;
                    o[3 * L] = d02 - rd13;
                }
            std::swap(a, b);
        }
        if (a != x) std::memcpy(x, a, sizeof(cplx) * n);
    }
    cplx w(long k, int sign) const {  // exp(sign * 2 pi i k / n)
        long kk = ((k % n) + n) % n;
        return sign < 0 ? tw[kk] : std::conj(tw[kk]);
    }
    // in-place transform of x (length n); work has length n
    void exec(cplx *x, cplx *work, int sign) const {
        if (pow2) {
            exec_pow2(x, work, sign);
            return;
        }
        cplx *a = x, *b = work;
        int Ns = 1;
        cplx v[8], o[8];
        for (int R : radix) {
            int nR = n / R;
            long step = n / R;  // r*k/(Ns*R) in units of 1/n: r*k*(n/(Ns*R))
            for (int j = 0; j < nR; j++) {
                int k = j % Ns;
                long tws = (long)k * (n / (Ns * R));
                for (int r = 0; r < R; r++) v[r] = a[j + r * nR] * (r ? w(r * tws, sign) : cplx(1.0));
                for (int q = 0; q < R; q++) {
                    cplx s = v[0];
                    for (int r = 1; r < R; r++) s += v[r] * w((long)r * q * (n / R), sign);
                    o[q] = s;
                }
                int idxD = (j / Ns) * Ns * R + k;
                for (int r = 0; r < R; r++) b[idxD + r * Ns] = o[r];
            }
            (void)step;
            std::swap(a, b);
            Ns *= R;
        }
        if (a != x) std::memcpy(x, a, sizeof(cplx) * n);
    }
};

// ------------------------------------------------------------------------------------
// Solver state: the module globals of GreenFunctions, SelfEnergies and SCF
// ------------------------------------------------------------------------------------
struct qso_state {
    // problem
    int Norb = 0, N_sites = 0, N_atoms = 0, order = 0, n = 0;
    std::vector<cplx> H, GammaL, GammaR;
    std::vector<double> U_site, omega;
    std::vector<int> atom_norb, atom_first;
    double mu = 0, beta = 0, delta = 0;
    double alpha_mix = 0.5, tolf = 1e-6, tolf_order1 = 1e-8;
    int nhist = 16, maxscf = 300;
    bool single_history = true;
    // setup_storage
    int nA = 0, nS = 0, nCL = 0, nAs = 0, n_int_sites = 0;
    std::vector<int> act, pos, sup, cl, asite;  // 1-based values, as in the reference
    std::vector<char> site_int, site_act;
    std::vector<cplx> Hemb, Sig1, GamL_s, GamR_s, GamL_cl, G_less_t0, G_less_obs;
    std::vector<cplx> Gr_in, GL_in;  // (nA, nA, n)
    std::vector<cplx> gRd, gLd;      // (nA, n)
    std::vector<cplx> onsL;          // (4 N_sites, n)
    std::vector<double> dosd;        // (Norb, n)
    std::vector<cplx> atomL;         // (atom_off(N_atoms+1), n)
    std::vector<int> atom_off;
    bool has_atomL = false;
    std::vector<double> trU, trD;
    int n_full = 0, n_strict_upper = 0, n_upper = 0, nblk = 0;
    int64_t n_vec = 0;
    // SelfEnergies
    int Nf = 0;
    FFTPlan plan;
    std::vector<cplx> Fr, FL, SigR2, SigL2;
    bool sigma2_ready = false;
    // SCF
    bool use_sigma = false;
    double V_scf = 0;
    int scf_iter = 0;
    std::vector<double> x_keep;  // converged input of the last voltage (continuation)
    bool have_x = false;
    std::string err;
    int64_t singular = 0;

    cplx &H_(int i, int j) { return H[(i - 1) + (size_t)(j - 1) * Norb]; }
};

static inline cplx &at2(std::vector<cplx> &A, int ld, int i, int j) { return A[(i - 1) + (size_t)(j - 1) * ld]; }
static inline cplx &at3(std::vector<cplx> &A, int ld, int i, int j, int k) {
    return A[(i - 1) + (size_t)(j - 1) * ld + (size_t)(k - 1) * ld * ld];
}

// fermi (src/green_functions.f90:74-84)
static double fermi(const qso_state &s, double w, double V) {
    double arg = (w - s.mu + V / HBAR) * s.beta;
    return 1.0 / (std::exp(std::min(HBAR * arg, 700.0)) + 1.0);
}

// setup_storage (src/green_functions.f90:90-190) + scf_setup_sizes (src/scf.f90:61-68)
static void setup_storage(qso_state &s) {
    const int No = s.Norb;
    s.site_int.assign(s.N_sites + 1, 0);
    s.site_act.assign(s.N_sites + 1, 0);
    s.pos.assign(No + 1, 0);
    std::vector<char> conL(No + 1, 0), conR(No + 1, 0);
    for (int st = 1; st <= s.N_sites; st++) s.site_int[st] = (s.order >= 1 && s.U_site[2 * st - 2] != 0.0);
    s.n_int_sites = 0;
    for (int st = 1; st <= s.N_sites; st++) s.n_int_sites += s.site_int[st];
    for (int st = 1; st <= s.N_sites; st++) s.site_act[st] = s.site_int[st];
    for (int i = 1; i <= No; i++) {
        bool l = false, r = false;
        for (int j = 1; j <= No; j++) {
            l = l || at2(s.GammaL, No, i, j) != 0.0 || at2(s.GammaL, No, j, i) != 0.0;
            r = r || at2(s.GammaR, No, i, j) != 0.0 || at2(s.GammaR, No, j, i) != 0.0;
        }
        conL[i] = l;
        conR[i] = r;
        if (l || r) s.site_act[(i + 1) / 2] = 1;
    }
    s.act.clear();
    for (int i = 1; i <= No; i++)
        if (s.site_act[(i + 1) / 2]) { s.act.push_back(i); s.pos[i] = (int)s.act.size(); }
    s.nA = (int)s.act.size();
    s.asite.clear();
    for (int st = 1; st <= s.N_sites; st++)
        if (s.site_act[st]) s.asite.push_back(st);
    s.nAs = (int)s.asite.size();
    s.cl.clear();
    for (int i = 1; i <= No; i++)
        if (conL[i]) s.cl.push_back(i);
    s.nCL = (int)s.cl.size();
    s.sup.clear();
    if (s.order == 2) s.sup = s.act;
    else
        for (int i = 1; i <= No; i++)
            if (conL[i] || conR[i]) s.sup.push_back(i);
    s.nS = (int)s.sup.size();
    s.GamL_s.assign((size_t)s.nS * s.nS, 0.0);
    s.GamR_s.assign((size_t)s.nS * s.nS, 0.0);
    s.GamL_cl.assign((size_t)s.nCL * s.nCL, 0.0);
    for (int b = 1; b <= s.nS; b++)
        for (int a = 1; a <= s.nS; a++) {
            at2(s.GamL_s, s.nS, a, b) = at2(s.GammaL, No, s.sup[a - 1], s.sup[b - 1]);
            at2(s.GamR_s, s.nS, a, b) = at2(s.GammaR, No, s.sup[a - 1], s.sup[b - 1]);
        }
    for (int b = 1; b <= s.nCL; b++)
        for (int a = 1; a <= s.nCL; a++) at2(s.GamL_cl, s.nCL, a, b) = at2(s.GammaL, No, s.cl[a - 1], s.cl[b - 1]);
    s.Hemb.assign((size_t)No * No, 0.0);
    s.Sig1.assign((size_t)No * No, 0.0);
    s.G_less_t0.assign((size_t)No * No, 0.0);
    s.G_less_obs.assign((size_t)No * No, 0.0);
    s.onsL.assign((size_t)4 * s.N_sites * s.n, 0.0);
    s.dosd.assign((size_t)No * s.n, 0.0);
    s.trU.assign(s.n, 0.0);
    s.trD.assign(s.n, 0.0);
    int mx = 0;
    for (int v : s.atom_norb) mx = std::max(mx, v);
    s.has_atomL = mx > 1;
    if (s.has_atomL) {
        s.atom_off.assign(s.N_atoms + 1, 0);
        for (int i = 1; i <= s.N_atoms; i++) s.atom_off[i] = s.atom_off[i - 1] + (2 * s.atom_norb[i - 1]) * (2 * s.atom_norb[i - 1]);
        s.atomL.assign((size_t)s.atom_off[s.N_atoms] * s.n, 0.0);
    }
    if (s.order >= 1) {
        s.gRd.assign((size_t)s.nA * s.n, 0.0);
        s.gLd.assign((size_t)s.nA * s.n, 0.0);
    }
    s.n_vec = 0;
    if (s.order == 1) s.n_vec = 8 * s.n_int_sites;
    else if (s.order == 2) {
        int64_t nfull = (int64_t)s.nA * s.nA, nsu = (nfull - s.nA) / 2;
        s.n_vec = (2 * nfull + nsu + nsu + s.nA) * s.n;
        s.Gr_in.assign((size_t)nfull * s.n, 0.0);
        s.GL_in.assign((size_t)nfull * s.n, 0.0);
    }
    s.n_full = s.nA * s.nA;
    s.n_strict_upper = (s.n_full - s.nA) / 2;
    s.n_upper = s.n_strict_upper + s.nA;
    s.nblk = 2 * s.n_full + s.n_strict_upper + s.n_upper;
}

// equal_time_lesser (src/green_functions.f90:192-213)
static void equal_time_lesser(qso_state &s) {
    double pp = s.delta / (2.0 * PI);
    std::fill(s.G_less_t0.begin(), s.G_less_t0.end(), 0.0);
    for (int is = 1; is <= s.nAs; is++)
        for (int a = 2 * s.asite[is - 1] - 1; a <= 2 * s.asite[is - 1]; a++)
            for (int b = 2 * s.asite[is - 1] - 1; b <= 2 * s.asite[is - 1]; b++) {
                cplx acc = 0.0;
                for (int k1 = 1; k1 <= s.n; k1++) acc += at3(s.GL_in, s.nA, s.pos[a], s.pos[b], k1);
                at2(s.G_less_t0, s.Norb, a, b) = acc * pp;
            }
}

// gather_onsite (src/green_functions.f90:215-238)
static void gather_onsite(qso_state &s, const std::vector<char> &mask, std::vector<cplx> &G) {
    double pp = s.delta / (2.0 * PI);
    for (int st = 1; st <= s.N_sites; st++) {
        if (!mask[st]) continue;
        for (int b = 1; b <= 2; b++)
            for (int a = 1; a <= 2; a++) {
                int k = 4 * (st - 1) + 2 * (b - 1) + a;
                cplx acc = 0.0;
                for (int iw = 1; iw <= s.n; iw++) acc += s.onsL[(k - 1) + (size_t)(iw - 1) * 4 * s.N_sites];
                at2(G, s.Norb, 2 * st - 2 + a, 2 * st - 2 + b) = acc * pp;
            }
    }
}

// gather_atoms (src/green_functions.f90:240-257)
static void gather_atoms(qso_state &s, std::vector<cplx> &G) {
    if (!s.has_atomL) return;
    double pp = s.delta / (2.0 * PI);
    size_t ld = s.atom_off[s.N_atoms];
    for (int at = 1; at <= s.N_atoms; at++) {
        int m = 2 * s.atom_norb[at - 1], lo = 2 * s.atom_first[at - 1] - 2;
        for (int b = 1; b <= m; b++)
            for (int a = 1; a <= m; a++) {
                cplx acc = 0.0;
                size_t row = s.atom_off[at - 1] + (b - 1) * m + a - 1;
                for (int iw = 0; iw < s.n; iw++) acc += s.atomL[row + iw * ld];
                at2(G, s.Norb, lo + a, lo + b) = acc * pp;
            }
    }
}

// sigma_first_order (src/self_energies.f90:45-72)
static void sigma_first_order(qso_state &s) {
    std::fill(s.Sig1.begin(), s.Sig1.end(), 0.0);
    for (int i = 1; i <= s.Norb; i += 2) {
        cplx hartree = at2(s.G_less_t0, s.Norb, i, i) + at2(s.G_less_t0, s.Norb, i + 1, i + 1);
        for (int a = 0; a <= 1; a++)
            for (int b = 0; b <= 1; b++) {
                if (a == b)
                    at2(s.Sig1, s.Norb, i + a, i + b) = IM * HBAR * s.U_site[i - 1] * (at2(s.G_less_t0, s.Norb, i + a, i + b) - hartree);
                else
                    at2(s.Sig1, s.Norb, i + a, i + b) = IM * HBAR * s.U_site[i - 1] * at2(s.G_less_t0, s.Norb, i + a, i + b);
            }
    }
}

// good_fft_size (src/self_energies.f90:75-89)
static int good_fft_size(int nmin) {
    int n = nmin;
    for (;;) {
        int m = n;
        while (m % 2 == 0) m /= 2;
        while (m % 3 == 0) m /= 3;
        while (m % 5 == 0) m /= 5;
        while (m % 7 == 0) m /= 7;
        if (m == 1) return n;
        n++;
    }
}

// sigma2_init (src/self_energies.f90:91-106)
static void sigma2_init(qso_state &s) {
    s.Nf = good_fft_size(2 * s.n - 1);
    s.Fr.assign((size_t)s.Nf * s.nA * s.nA, 0.0);
    s.FL.assign((size_t)s.Nf * s.nA * s.nA, 0.0);
    s.SigR2.assign((size_t)s.nA * s.nA * s.n, 0.0);
    s.SigL2.assign((size_t)s.nA * s.nA * s.n, 0.0);
    s.plan.init(s.Nf);
    s.sigma2_ready = true;
}

// adj2 (src/self_energies.f90:222-228)
struct M2 { cplx a[2][2]; };
static inline M2 adj2(const M2 &M) {
    M2 A;
    A.a[0][0] = M.a[1][1];
    A.a[0][1] = -M.a[0][1];
    A.a[1][0] = -M.a[1][0];
    A.a[1][1] = M.a[0][0];
    return A;
}
static inline M2 mm(const M2 &X, const M2 &Y) {
    M2 Z;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) Z.a[i][j] = X.a[i][0] * Y.a[0][j] + X.a[i][1] * Y.a[1][j];
    return Z;
}
static inline M2 dag(const M2 &X) {
    M2 Z;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) Z.a[i][j] = std::conj(X.a[j][i]);
    return Z;
}

// sigma2_compute (src/self_energies.f90:135-219)
static void sigma2_compute(qso_state &s, bool do_lesser) {
    const int nA = s.nA, Nf = s.Nf, n = s.n;
    double pp = s.delta / (2.0 * PI);
    // 1. forward FFT of every active element of G^r and G^< (load_fft, lines 116-130)
#pragma omp parallel
    {
        std::vector<cplx> work(Nf);
#pragma omp for collapse(2) schedule(static)
        for (int jj = 1; jj <= nA; jj++)
            for (int ii = 1; ii <= nA; ii++) {
                cplx *dr = &s.Fr[(size_t)Nf * ((ii - 1) + (size_t)(jj - 1) * nA)];
                cplx *dl = &s.FL[(size_t)Nf * ((ii - 1) + (size_t)(jj - 1) * nA)];
                for (int iw = 1; iw <= n; iw++) {
                    dr[iw - 1] = at3(s.Gr_in, nA, ii, jj, iw);
                    dl[iw - 1] = at3(s.GL_in, nA, ii, jj, iw);
                }
                for (int k = n; k < Nf; k++) dr[k] = dl[k] = 0.0;
                s.plan.exec(dr, work.data(), -1);
                s.plan.exec(dl, work.data(), -1);
            }
    }
    auto Fr = [&](int l, int i, int j) { return s.Fr[(size_t)(l - 1) + (size_t)Nf * ((i - 1) + (size_t)(j - 1) * nA)]; };
    auto FL = [&](int l, int i, int j) { return s.FL[(size_t)(l - 1) + (size_t)Nf * ((i - 1) + (size_t)(j - 1) * nA)]; };
    // 2. per pair of active sites: 2x2 algebra at every l, then inverse FFT
#pragma omp parallel
    {
        std::vector<cplx> bufR((size_t)Nf * 4), bufL((size_t)Nf * 4), work(Nf);
#pragma omp for collapse(2) schedule(dynamic)
        for (int ja = 1; ja <= s.nAs; ja++)
            for (int ia = 1; ia <= s.nAs; ia++) {
                int io = s.pos[2 * s.asite[ia - 1] - 1], jo = s.pos[2 * s.asite[ja - 1] - 1];
                double Uprod = s.U_site[s.act[io - 1] - 1] * s.U_site[s.act[jo - 1] - 1];
                if (Uprod == 0.0) {
                    for (int iw = 1; iw <= n; iw++)
                        for (int a = 0; a < 2; a++)
                            for (int b = 0; b < 2; b++) {
                                at3(s.SigR2, nA, io + a, jo + b, iw) = 0.0;
                                at3(s.SigL2, nA, io + a, jo + b, iw) = 0.0;
                            }
                    continue;
                }
                for (int l = 1; l <= Nf; l++) {
                    int lm = (Nf - (l - 1)) % Nf + 1;
                    M2 r_ij, L_ij, r_ji, L_ji;
                    for (int a = 0; a < 2; a++)
                        for (int b = 0; b < 2; b++) {
                            r_ij.a[a][b] = Fr(l, io + a, jo + b);
                            L_ij.a[a][b] = FL(l, io + a, jo + b);
                            r_ji.a[a][b] = Fr(lm, jo + a, io + b);
                            L_ji.a[a][b] = FL(lm, jo + a, io + b);
                        }
                    M2 a_ij = dag(r_ji), a_ji = dag(r_ij), G_ij, G_ji;
                    for (int a = 0; a < 2; a++)
                        for (int b = 0; b < 2; b++) {
                            G_ij.a[a][b] = L_ij.a[a][b] + r_ij.a[a][b] - a_ij.a[a][b];
                            G_ji.a[a][b] = L_ji.a[a][b] + r_ji.a[a][b] - a_ji.a[a][b];
                        }
                    M2 chi1 = mm(L_ji, G_ij);
                    M2 t1 = mm(L_ji, r_ij), t2 = mm(a_ji, L_ij), chi2;
                    for (int a = 0; a < 2; a++)
                        for (int b = 0; b < 2; b++) chi2.a[a][b] = t1.a[a][b] + t2.a[a][b];
                    M2 u1 = mm(r_ij, adj2(chi1)), u2 = mm(L_ij, adj2(chi2));
                    for (int a = 0; a < 2; a++)
                        for (int b = 0; b < 2; b++) bufR[(size_t)(l - 1) + (size_t)Nf * (a + 2 * b)] = u1.a[a][b] + u2.a[a][b];
                    if (do_lesser) {
                        M2 chiL = mm(G_ji, L_ij);
                        M2 sL = mm(L_ij, adj2(chiL));
                        for (int a = 0; a < 2; a++)
                            for (int b = 0; b < 2; b++) bufL[(size_t)(l - 1) + (size_t)Nf * (a + 2 * b)] = sL.a[a][b];
                    }
                }
                cplx c = Uprod * HBAR * HBAR * pp * pp / (double)Nf;
                for (int sp1 = 1; sp1 <= 2; sp1++)
                    for (int sp = 1; sp <= 2; sp++) {
                        cplx *bR = &bufR[(size_t)Nf * ((sp - 1) + 2 * (sp1 - 1))];
                        s.plan.exec(bR, work.data(), +1);
                        for (int iw = 1; iw <= n; iw++) at3(s.SigR2, nA, io + sp - 1, jo + sp1 - 1, iw) = c * bR[iw - 1];
                        if (do_lesser) {
                            cplx *bL = &bufL[(size_t)Nf * ((sp - 1) + 2 * (sp1 - 1))];
                            s.plan.exec(bL, work.data(), +1);
                            for (int iw = 1; iw <= n; iw++) at3(s.SigL2, nA, io + sp - 1, jo + sp1 - 1, iw) = c * bL[iw - 1];
                        }
                    }
            }
    }
}

// pack_gf (common/linear_algebra.f90:155-191), one energy block or Nw of them
static void pack_gf(const cplx *In1, const cplx *In2, double *out, int n_full, int n_strict_upper, int nb, int Nw) {
    int nblock = 2 * n_full + n_strict_upper + (n_strict_upper + nb);
    for (int iw = 1; iw <= Nw; iw++) {
        size_t off = (size_t)(iw - 1) * nblock;
        const cplx *A = In1 + (size_t)(iw - 1) * nb * nb, *B = In2 + (size_t)(iw - 1) * nb * nb;
        int n = 0;
        for (int i = 1; i <= nb; i++)
            for (int j = 1; j <= nb; j++) {
                n++;
                out[off + n - 1] = A[(i - 1) + (size_t)(j - 1) * nb].real();
                out[off + n + n_full - 1] = A[(i - 1) + (size_t)(j - 1) * nb].imag();
            }
        n = 2 * n_full + n_strict_upper;
        int n1 = 2 * n_full;
        for (int i = 1; i <= nb; i++)
            for (int j = i; j <= nb; j++) {
                n++;
                if (i != j) { n1++; out[off + n1 - 1] = B[(i - 1) + (size_t)(j - 1) * nb].real(); }
                out[off + n - 1] = B[(i - 1) + (size_t)(j - 1) * nb].imag();
            }
    }
}

// unpack_gf (common/linear_algebra.f90:193-233)
static void unpack_gf(cplx *O1, cplx *O2, const double *in, int n_full, int n_strict_upper, int nb, int Nw) {
    int nblock = 2 * n_full + n_strict_upper + (n_strict_upper + nb);
    for (int iw = 1; iw <= Nw; iw++) {
        size_t off = (size_t)(iw - 1) * nblock;
        cplx *A = O1 + (size_t)(iw - 1) * nb * nb, *B = O2 + (size_t)(iw - 1) * nb * nb;
        int n = 0;
        for (int i = 1; i <= nb; i++)
            for (int j = 1; j <= nb; j++) {
                n++;
                A[(i - 1) + (size_t)(j - 1) * nb] = cplx(in[off + n - 1], in[off + n + n_full - 1]);
            }
        n = 2 * n_full + n_strict_upper;
        int n1 = 2 * n_full;
        for (int i = 1; i <= nb; i++)
            for (int j = i; j <= nb; j++) {
                n++;
                double re = 0.0;
                if (i != j) { n1++; re = in[off + n1 - 1]; }
                B[(i - 1) + (size_t)(j - 1) * nb] = cplx(re, in[off + n - 1]);
                B[(j - 1) + (size_t)(i - 1) * nb] = -std::conj(B[(i - 1) + (size_t)(j - 1) * nb]);
            }
    }
}

enum { M_INIT2 = 1, M_SCF2 = 2, M_SCF1 = 3, M_FINAL = 4 };

// G_at_energy (src/scf.f90:305-415)
static void G_at_energy(qso_state &s, int iw, double Volt, int mode, double *F) {
    const int No = s.Norb, nA = s.nA, nS = s.nS;
    double w = s.omega[iw - 1];
    std::vector<cplx> w1(s.Hemb);
    if (s.use_sigma) {
        for (int b = 1; b <= nA; b++)
            for (int a = 1; a <= nA; a++) {
                cplx sg = at2(s.Sig1, No, s.act[a - 1], s.act[b - 1]);
                if (s.order == 2) sg += at3(s.SigR2, nA, a, b, iw);
                at2(w1, No, s.act[a - 1], s.act[b - 1]) -= sg;
            }
    }
    for (int i = 1; i <= No; i++) at2(w1, No, i, i) += HBAR * w;
    int64_t info = invert_complex(No, w1.data());
    if (info != 0) {
#pragma omp critical
        s.singular = iw;
    }
    auto W = [&](int i, int j) { return w1[(i - 1) + (size_t)(j - 1) * No]; };

    double fL = fermi(s, w, Volt), fR = fermi(s, w, 0.0);
    std::vector<cplx> SL((size_t)nS * nS);
    for (size_t k = 0; k < SL.size(); k++) SL[k] = IM * (fL * s.GamL_s[k] + fR * s.GamR_s[k]) / HBAR;
    if (s.use_sigma && s.order == 2)
        for (int b = 1; b <= nS; b++)
            for (int a = 1; a <= nS; a++) at2(SL, nS, a, b) += at3(s.SigL2, nA, a, b, iw);

    if (mode == M_INIT2 || mode == M_SCF2) {
        // sup = act: grA = w1(act,act); T = grA SL; glA = T grA^dagger
        std::vector<cplx> grA((size_t)nA * nA), T((size_t)nA * nA, 0.0), glA((size_t)nA * nA, 0.0);
        for (int b = 1; b <= nA; b++)
            for (int a = 1; a <= nA; a++) grA[(a - 1) + (size_t)(b - 1) * nA] = W(s.act[a - 1], s.act[b - 1]);
        for (int j = 0; j < nA; j++)
            for (int k = 0; k < nA; k++) {
                cplx b = SL[k + (size_t)j * nA];
                for (int i = 0; i < nA; i++) T[i + (size_t)j * nA] += grA[i + (size_t)k * nA] * b;
            }
        for (int j = 0; j < nA; j++)
            for (int k = 0; k < nA; k++) {
                cplx b = std::conj(grA[j + (size_t)k * nA]);
                for (int i = 0; i < nA; i++) glA[i + (size_t)j * nA] += T[i + (size_t)k * nA] * b;
            }
        if (mode == M_INIT2) {
            std::copy(grA.begin(), grA.end(), s.Gr_in.begin() + (size_t)(iw - 1) * nA * nA);
            std::copy(glA.begin(), glA.end(), s.GL_in.begin() + (size_t)(iw - 1) * nA * nA);
        } else {
            size_t off = (size_t)(iw - 1) * s.nblk;
            pack_gf(grA.data(), glA.data(), F + off, s.n_full, s.n_strict_upper, nA, 1);
            for (int k = 1; k <= nA; k++) {
                s.gRd[(k - 1) + (size_t)(iw - 1) * nA] = grA[(k - 1) + (size_t)(k - 1) * nA];
                s.gLd[(k - 1) + (size_t)(iw - 1) * nA] = glA[(k - 1) + (size_t)(k - 1) * nA];
            }
        }
    } else if (mode == M_SCF1) {
        // T = w1(act, sup) SL
        std::vector<cplx> T((size_t)nA * nS, 0.0);
        for (int j = 1; j <= nS; j++)
            for (int k = 1; k <= nS; k++) {
                cplx b = at2(SL, nS, k, j);
                for (int i = 1; i <= nA; i++) T[(i - 1) + (size_t)(j - 1) * nA] += W(s.act[i - 1], s.sup[k - 1]) * b;
            }
        for (int k = 1; k <= nA; k++) {
            s.gRd[(k - 1) + (size_t)(iw - 1) * nA] = W(s.act[k - 1], s.act[k - 1]);
            cplx acc = 0.0;
            for (int q = 1; q <= nS; q++) acc += T[(k - 1) + (size_t)(q - 1) * nA] * std::conj(W(s.act[k - 1], s.sup[q - 1]));
            s.gLd[(k - 1) + (size_t)(iw - 1) * nA] = acc;
        }
        for (int st = 1; st <= s.N_sites; st++) {
            if (!s.site_int[st]) continue;
            int lo = 2 * st - 1, p1 = s.pos[lo];
            for (int b = 0; b < 2; b++)
                for (int a = 0; a < 2; a++) {
                    cplx acc = 0.0;
                    for (int q = 1; q <= nS; q++)
                        acc += T[(p1 + a - 1) + (size_t)(q - 1) * nA] * std::conj(W(lo + b, s.sup[q - 1]));
                    s.onsL[(size_t)(4 * (st - 1) + a + 2 * b) + (size_t)(iw - 1) * 4 * s.N_sites] = acc;
                }
        }
    } else {  // M_FINAL
        std::vector<cplx> T((size_t)No * nS, 0.0);
        for (int j = 1; j <= nS; j++)
            for (int k = 1; k <= nS; k++) {
                cplx b = at2(SL, nS, k, j);
                if (b == 0.0) continue;
                for (int i = 1; i <= No; i++) T[(i - 1) + (size_t)(j - 1) * No] += W(i, s.sup[k - 1]) * b;
            }
        for (int i = 1; i <= No; i++) s.dosd[(i - 1) + (size_t)(iw - 1) * No] = W(i, i).imag();
        auto blk = [&](int ra, int rb) {  // sum_q T(ra,q) conj(w1(rb, sup(q)))
            cplx acc = 0.0;
            for (int q = 1; q <= nS; q++) acc += T[(ra - 1) + (size_t)(q - 1) * No] * std::conj(W(rb, s.sup[q - 1]));
            return acc;
        };
        for (int st = 1; st <= s.N_sites; st++) {
            int lo = 2 * st - 1;
            for (int b = 0; b < 2; b++)
                for (int a = 0; a < 2; a++)
                    s.onsL[(size_t)(4 * (st - 1) + a + 2 * b) + (size_t)(iw - 1) * 4 * s.N_sites] = blk(lo + a, lo + b);
        }
        if (s.has_atomL) {
            size_t ld = s.atom_off[s.N_atoms];
            for (int at = 1; at <= s.N_atoms; at++) {
                int lo = 2 * s.atom_first[at - 1] - 1, m = 2 * s.atom_norb[at - 1];
                for (int b = 0; b < m; b++)
                    for (int a = 0; a < m; a++)
                        s.atomL[(size_t)(s.atom_off[at - 1] + a + b * m) + (size_t)(iw - 1) * ld] = blk(lo + a, lo + b);
            }
        }
        // current integrand through the left lead (src/scf.f90:390-409)
        const int nCL = s.nCL;
        std::vector<cplx> GLc((size_t)nCL * nCL), X((size_t)nCL * nCL);
        for (int a = 1; a <= nCL; a++)
            for (int k = 1; k <= nCL; k++) GLc[(k - 1) + (size_t)(a - 1) * nCL] = blk(s.cl[k - 1], s.cl[a - 1]);
        for (int a = 1; a <= nCL; a++)
            for (int k = 1; k <= nCL; k++) {
                cplx g = GLc[(k - 1) + (size_t)(a - 1) * nCL];
                X[(k - 1) + (size_t)(a - 1) * nCL] =
                    (fL - 1.0) * g - fL * (g + W(s.cl[k - 1], s.cl[a - 1]) - std::conj(W(s.cl[a - 1], s.cl[k - 1])));
            }
        cplx tu = 0.0, td = 0.0;
        for (int a = 1; a <= nCL; a++) {
            cplx mc = 0.0;  // Mc(a,a) = i sum_k GamL_cl(a,k) X(k,a)
            for (int k = 1; k <= nCL; k++) mc += at2(s.GamL_cl, nCL, a, k) * X[(k - 1) + (size_t)(a - 1) * nCL];
            mc *= IM;
            if (s.cl[a - 1] % 2 == 1) tu += mc;
            else td += mc;
        }
        s.trU[iw - 1] = tu.real() / (2.0 * PI);
        s.trD[iw - 1] = td.real() / (2.0 * PI);
    }
}

// sweep (src/scf.f90:280-290)
static void sweep(qso_state &s, int mode, double *F) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int iw = 1; iw <= s.n; iw++) G_at_energy(s, iw, s.V_scf, mode, F);
}

// check_diag_sanity (common/scf_checks.f90:59-91)
static void check_diag_sanity(const cplx *Grd, const cplx *GLd, int nb, int nw, double delta, bool &runaway,
                              bool &unphysical, int &i_worst, double &n_worst, double &w_worst, const int *state_index) {
    runaway = false;
    unphysical = false;
    i_worst = 1;
    n_worst = 0.5;
    w_worst = 1.0;
    for (int i = 1; i <= nb; i++) {
        int lab = state_index ? state_index[i - 1] : i;
        cplx sl = 0.0;
        double si = 0.0;
        for (int w = 0; w < nw; w++) {
            sl += GLd[(i - 1) + (size_t)w * nb];
            si += Grd[(i - 1) + (size_t)w * nb].imag();
        }
        double nocc = (-IM * HBAR * (delta / (2.0 * PI)) * sl).real();
        double wsum = -HBAR * (delta / PI) * si;
        if (!std::isfinite(nocc) || !std::isfinite(wsum)) {  // runaway only: the return skips the last line
            runaway = true;
            i_worst = lab;
            n_worst = nocc;
            w_worst = wsum;
            return;
        }
        if (nocc < -1.0 || nocc > 2.0) runaway = true;
        if (nocc < -0.05 || nocc > 1.05 || wsum < 0.5) unphysical = true;
        if (std::fabs(nocc - 0.5) > std::fabs(n_worst - 0.5) || (wsum < w_worst && std::fabs(n_worst - 0.5) <= 0.55)) {
            i_worst = lab;
            n_worst = nocc;
            w_worst = wsum;
        }
    }
    if (runaway) unphysical = true;
}

// pack_nil / unpack_nil (src/scf.f90:226-255)
static void pack_nil(qso_state &s, const std::vector<cplx> &G, double *x) {
    int k = 0;
    for (int st = 1; st <= s.N_sites; st++) {
        if (!s.site_int[st]) continue;
        for (int b = 2 * st - 1; b <= 2 * st; b++)
            for (int a = 2 * st - 1; a <= 2 * st; a++) {
                cplx g = G[(a - 1) + (size_t)(b - 1) * s.Norb];
                x[k] = g.real();
                x[k + 1] = g.imag();
                k += 2;
            }
    }
}
static void unpack_nil(qso_state &s, const double *x, std::vector<cplx> &G) {
    std::fill(G.begin(), G.end(), 0.0);
    int k = 0;
    for (int st = 1; st <= s.N_sites; st++) {
        if (!s.site_int[st]) continue;
        for (int b = 2 * st - 1; b <= 2 * st; b++)
            for (int a = 2 * st - 1; a <= 2 * st; a++) {
                G[(a - 1) + (size_t)(b - 1) * s.Norb] = cplx(x[k], x[k + 1]);
                k += 2;
            }
    }
}

// scf_residual2 (src/scf.f90:158-188)
static void scf_residual2(qso_state &s, int64_t n, const double *x, double *F, bool &abort) {
    s.scf_iter++;
    unpack_gf(s.Gr_in.data(), s.GL_in.data(), x, s.n_full, s.n_strict_upper, s.nA, s.n);
    equal_time_lesser(s);
    sigma_first_order(s);
    sigma2_compute(s, true);
    s.use_sigma = true;
    sweep(s, M_SCF2, F);
    bool unphys;
    int iw;
    double nw, ww;
    check_diag_sanity(s.gRd.data(), s.gLd.data(), s.nA, s.n, s.delta, abort, unphys, iw, nw, ww, s.act.data());
    if (abort) {
        std::fill(F, F + n, 0.0);
        return;
    }
#pragma omp parallel for
    for (int64_t i = 0; i < n; i++) F[i] -= x[i];
}

// scf_residual1 (src/scf.f90:194-224)
static void scf_residual1(qso_state &s, int64_t n, const double *x, double *F, bool &abort) {
    s.scf_iter++;
    unpack_nil(s, x, s.G_less_t0);
    sigma_first_order(s);
    s.use_sigma = true;
    sweep(s, M_SCF1, F);
    bool unphys;
    int iw;
    double nw, ww;
    check_diag_sanity(s.gRd.data(), s.gLd.data(), s.nA, s.n, s.delta, abort, unphys, iw, nw, ww, s.act.data());
    if (abort) {
        std::fill(F, F + n, 0.0);
        return;
    }
    std::vector<cplx> Gout((size_t)s.Norb * s.Norb, 0.0);
    gather_onsite(s, s.site_int, Gout);
    pack_nil(s, Gout, F);
    for (int64_t i = 0; i < n; i++) F[i] -= x[i];
}

// wall-clock time (s, steady clock) at the start of every Broyden iteration, recorded while
// qso_solve_scf_timed runs (CPU-baseline timing only)
static std::vector<double> *g_step_times = nullptr;

// broyden_solve (common/broyden_mixing.f90:51-184), with its dot_ss / dot_sd (186-215)
template <class Residual>
static void broyden_solve(Residual residual, double *x, int64_t n, double alpha_mix, int nhist, int maxscf, double tolf,
                          bool sp, bool &converged, int &n_iter, double &fmax, std::vector<qs_scf_step> &log,
                          int &n_resets) {
    const double w0 = 0.01;
    int lda = std::max(nhist, 1);
    std::vector<double> F(n), Fold(n), xold(n), a((size_t)lda * lda), cvec(lda), gram((size_t)lda * lda);
    std::vector<double> dF, U;
    std::vector<float> dFs, Us;
    if (sp) {
        dFs.assign((size_t)n * lda, 0.f);
        Us.assign((size_t)n * lda, 0.f);
    } else {
        dF.assign((size_t)n * nhist, 0.0);
        U.assign((size_t)n * nhist, 0.0);
    }
    converged = false;
    int nstored = 0, nh = 0;
    fmax = HUGE_VAL;
    n_resets = 0;
    for (int its = 1; its <= maxscf; its++) {
        n_iter = its;
        if (g_step_times)
            g_step_times->push_back(
                std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count());
        bool abort = false;
        residual(n, x, F.data(), abort);
        if (abort) break;
        fmax = 0.0;
        for (int64_t i = 0; i < n; i++) fmax = std::max(fmax, std::fabs(F[i]));
        double rms = dnrm2(n, F.data()) / std::sqrt((double)n);
        log.push_back({its, fmax, rms, std::min(nstored, nhist)});
        if (fmax < tolf) {
            converged = true;
            break;
        }
        if (its > 1 && nhist > 0) {
            int slot = nstored % nhist;  // 0-based
            if (sp) {
                for (int64_t i = 0; i < n; i++) Fold[i] = F[i] - Fold[i];
                double fnorm = dnrm2(n, Fold.data());
                if (fnorm > 0.0) {
                    double rf = 1.0 / fnorm;
                    float *dcol = &dFs[(size_t)n * slot], *ucol = &Us[(size_t)n * slot];
#pragma omp parallel for
                    for (int64_t i = 0; i < n; i++) {
                        dcol[i] = (float)(Fold[i] * rf);
                        ucol[i] = (float)(alpha_mix * Fold[i] * rf + (x[i] - xold[i]) * rf);
                    }
                    nstored++;
                    nh = std::min(nstored, nhist);
                    for (int k = 0; k < nh; k++) {
                        const float *u = &dFs[(size_t)n * k];
                        double acc = 0.0;
#pragma omp parallel for reduction(+ : acc)
                        for (int64_t i = 0; i < n; i++) acc += (double)u[i] * (double)dcol[i];
                        cvec[k] = acc;
                    }
                    for (int k = 0; k < nh; k++) {
                        gram[k + (size_t)slot * lda] = cvec[k];
                        gram[slot + (size_t)k * lda] = cvec[k];
                    }
                }
            } else {
                double *dcol = &dF[(size_t)n * slot], *ucol = &U[(size_t)n * slot];
                for (int64_t i = 0; i < n; i++) dcol[i] = F[i] - Fold[i];
                double fnorm = dnrm2(n, dcol);
                if (fnorm > 0.0) {
                    for (int64_t i = 0; i < n; i++) dcol[i] = dcol[i] / fnorm;
                    for (int64_t i = 0; i < n; i++) ucol[i] = alpha_mix * dcol[i] + (x[i] - xold[i]) / fnorm;
                    nstored++;
                    nh = std::min(nstored, nhist);
                    for (int k = 0; k < nh; k++) {
                        const double *u = &dF[(size_t)n * k];
                        double acc = 0.0;
                        for (int64_t i = 0; i < n; i++) acc += u[i] * dcol[i];
                        cvec[k] = acc;
                    }
                    for (int k = 0; k < nh; k++) {
                        gram[k + (size_t)slot * lda] = cvec[k];
                        gram[slot + (size_t)k * lda] = cvec[k];
                    }
                }
            }
        }
        nh = std::min(nstored, nhist);
        std::copy(x, x + n, xold.begin());
        std::copy(F.begin(), F.end(), Fold.begin());
        if (nh > 0) {
            for (int j = 0; j < nh; j++)
                for (int i = 0; i < nh; i++) a[i + (size_t)j * lda] = gram[i + (size_t)j * lda];
            for (int i = 0; i < nh; i++) a[i + (size_t)i * lda] += w0 * w0;
            for (int k = 0; k < nh; k++) {
                double acc = 0.0;
                if (sp) {
                    const float *u = &dFs[(size_t)n * k];
#pragma omp parallel for reduction(+ : acc)
                    for (int64_t i = 0; i < n; i++) acc += (double)u[i] * F[i];
                } else {
                    const double *u = &dF[(size_t)n * k];
                    for (int64_t i = 0; i < n; i++) acc += u[i] * F[i];
                }
                cvec[k] = acc;
            }
            int64_t nn = nh, one = 1, ld = lda, info = 0;
            scipy_dposv_64_("U", &nn, &one, a.data(), &ld, cvec.data(), &ld, &info, 1);
            if (info != 0) {
                nstored = 0;
                nh = 0;
                n_resets++;
            }
        }
        if (sp) {
#pragma omp parallel for
            for (int64_t i = 0; i < n; i++) {
                double xi = x[i] + alpha_mix * F[i];
                for (int k = 0; k < nh; k++) xi -= (double)Us[(size_t)n * k + i] * cvec[k];
                x[i] = xi;
            }
        } else {
            for (int64_t i = 0; i < n; i++) x[i] += alpha_mix * F[i];
            if (nh > 0)
                for (int k = 0; k < nh; k++) {
                    const double *u = &U[(size_t)n * k];
                    for (int64_t i = 0; i < n; i++) x[i] -= u[i] * cvec[k];
                }
        }
    }
}

// final_sanity (src/scf.f90:260-275)
static void final_sanity(qso_state &s, bool &runaway, bool &unphysical, int &i_worst, double &n_worst, double &w_worst) {
    std::vector<cplx> grd((size_t)s.Norb * s.n), gld((size_t)s.Norb * s.n);
    for (int iw = 0; iw < s.n; iw++)
        for (int i = 1; i <= s.Norb; i++) {
            int st = (i + 1) / 2, a = i - 2 * (st - 1);
            grd[(i - 1) + (size_t)iw * s.Norb] = cplx(0.0, s.dosd[(i - 1) + (size_t)iw * s.Norb]);
            gld[(i - 1) + (size_t)iw * s.Norb] = s.onsL[(size_t)(4 * (st - 1) + 2 * (a - 1) + a - 1) + (size_t)iw * 4 * s.N_sites];
        }
    check_diag_sanity(grd.data(), gld.data(), s.Norb, s.n, s.delta, runaway, unphysical, i_worst, n_worst, w_worst, nullptr);
}

static void hemb(qso_state &s) {
    // Hemb = -H + (i/2 hbar)(GammaL + GammaR)   (src/scf.f90:92)
    for (size_t k = 0; k < s.H.size(); k++) s.Hemb[k] = -s.H[k] + 0.5 * (IM / HBAR) * (s.GammaL[k] + s.GammaR[k]);
}

// ------------------------------------------------------------------------------------
// C ABI (same signatures as include/qsb200.h, prefix qso_)
// ------------------------------------------------------------------------------------
extern "C" {

int qso_create(const qs_problem *p, qso_state **out) {
    scipy_openblas_set_num_threads64_(1);  // one LAPACK thread per OpenMP thread, as the reference runs
    auto *s = new qso_state();
    s->Norb = p->Norb;
    s->N_sites = p->N_sites;
    s->N_atoms = p->N_atoms;
    s->order = p->order;
    s->n = p->n_omega;
    size_t nn = (size_t)p->Norb * p->Norb;
    s->H.assign((const cplx *)p->H, (const cplx *)p->H + nn);
    s->GammaL.assign((const cplx *)p->GammaL, (const cplx *)p->GammaL + nn);
    s->GammaR.assign((const cplx *)p->GammaR, (const cplx *)p->GammaR + nn);
    s->U_site.assign(p->U_site, p->U_site + p->Norb);
    s->omega.assign(p->omega, p->omega + p->n_omega);
    s->atom_norb.assign(p->atom_norb, p->atom_norb + p->N_atoms);
    s->atom_first.assign(p->atom_first, p->atom_first + p->N_atoms);
    s->mu = p->mu;
    s->beta = p->beta;
    s->delta = p->delta;
    s->alpha_mix = p->alpha_mix;
    s->tolf = p->tolf;
    s->tolf_order1 = p->tolf_order1;
    s->nhist = p->nhist;
    s->maxscf = p->maxscf;
    s->single_history = p->single_history != 0;
    setup_storage(*s);
    *out = s;
    return 0;
}

void qso_destroy(qso_state *s) { delete s; }
const char *qso_last_error(const qso_state *s) { return s ? s->err.c_str() : "no handle"; }
int64_t qso_vector_length(const qso_state *s) { return s->n_vec; }
int qso_active_states(const qso_state *s) { return s->nA; }
int qso_fft_length(const qso_state *s) { return good_fft_size(2 * s->n - 1); }

static int check_singular(qso_state *s) {
    if (s->singular) {
        s->err = "ERROR: ZGETRF failed (singular matrix?) at energy " + std::to_string(s->singular);
        int e = (int)s->singular;
        s->singular = 0;
        return e;
    }
    return 0;
}

// solve_scf (src/scf.f90:78-151)
int qso_solve_scf(qso_state *s, double Volt, int fresh_start, qs_scf_result *res) {
    auto t0 = std::chrono::steady_clock::now();
    hemb(*s);
    s->V_scf = Volt;
    s->scf_iter = 0;
    bool converged = true;
    int n_iter = 0, n_resets = 0;
    double fmax = 0.0;
    std::vector<qs_scf_step> log;
    bool aborted = false;
    if (s->order == 1) {
        if (fresh_start || !s->have_x) {
            std::fill(s->G_less_t0.begin(), s->G_less_t0.end(), 0.0);
            s->use_sigma = false;
            sweep(*s, M_SCF1, nullptr);
            gather_onsite(*s, s->site_int, s->G_less_t0);
        }
        std::vector<double> x(s->n_vec);
        pack_nil(*s, s->G_less_t0, x.data());
        broyden_solve([&](int64_t n, const double *xx, double *F, bool &ab) { scf_residual1(*s, n, xx, F, ab); aborted = aborted || ab; },
                      x.data(), s->n_vec, s->alpha_mix, s->nhist, s->maxscf, s->tolf_order1, s->single_history, converged,
                      n_iter, fmax, log, n_resets);
    } else if (s->order == 2) {
        if (!s->sigma2_ready) sigma2_init(*s);
        std::vector<double> x(s->n_vec);
        if (fresh_start || !s->have_x) {
            s->use_sigma = false;
            sweep(*s, M_INIT2, nullptr);
        }
        pack_gf(s->Gr_in.data(), s->GL_in.data(), x.data(), s->n_full, s->n_strict_upper, s->nA, s->n);
        broyden_solve([&](int64_t n, const double *xx, double *F, bool &ab) { scf_residual2(*s, n, xx, F, ab); aborted = aborted || ab; },
                      x.data(), s->n_vec, s->alpha_mix, s->nhist, s->maxscf, s->tolf, s->single_history, converged, n_iter,
                      fmax, log, n_resets);
        s->have_x = true;
    } else {
        log.push_back({1, 0.0, 0.0, 0});
        n_iter = 1;
    }
    if (s->order == 1) s->have_x = true;
    if (int e = check_singular(s)) return e;
    // final sweep with the converged self-energies (Sig1, SigR2, SigL2 of the last input)
    s->use_sigma = (s->order >= 1);
    sweep(*s, M_FINAL, nullptr);
    if (int e = check_singular(s)) return e;
    std::fill(s->G_less_obs.begin(), s->G_less_obs.end(), 0.0);
    std::vector<char> all(s->N_sites + 1, 1);
    gather_onsite(*s, all, s->G_less_obs);
    gather_atoms(*s, s->G_less_obs);
    bool runaway, unphysical;
    int i_worst;
    double n_worst, w_worst;
    final_sanity(*s, runaway, unphysical, i_worst, n_worst, w_worst);
    if (converged && unphysical) converged = false;
    res->converged = converged;
    res->n_iter = n_iter;
    res->fmax = fmax;
    res->aborted = aborted;
    res->runaway = runaway;
    res->unphysical = unphysical;
    res->i_worst = i_worst;
    res->n_worst = n_worst;
    res->w_worst = w_worst;
    res->n_resets = n_resets;
    res->n_log = 0;
    for (auto &e : log)
        if (res->log && res->n_log < res->log_cap) res->log[res->n_log++] = e;
    res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return 0;
}

// Current (src/observables.f90:22-39)
int qso_current(qso_state *s, double, double *J_up, double *J_down) {
    double ju = 0.0, jd = 0.0;
    for (int iw = 0; iw < s->n; iw++) {
        ju += s->trU[iw];
        jd += s->trD[iw];
    }
    *J_up = ju * (s->delta / HBAR);
    *J_down = jd * (s->delta / HBAR);
    return 0;
}

int qso_get_observables(qso_state *s, double *G_less_obs, double *dosd, double *trU, double *trD) {
    if (G_less_obs) std::memcpy(G_less_obs, s->G_less_obs.data(), sizeof(cplx) * s->G_less_obs.size());
    if (dosd) std::memcpy(dosd, s->dosd.data(), sizeof(double) * s->dosd.size());
    if (trU) std::memcpy(trU, s->trU.data(), sizeof(double) * s->n);
    if (trD) std::memcpy(trD, s->trD.data(), sizeof(double) * s->n);
    return 0;
}

int qso_initial_vector(qso_state *s, double Volt, double *x) {
    hemb(*s);
    s->V_scf = Volt;
    if (s->order == 2) {
        if (!s->sigma2_ready) sigma2_init(*s);
        s->use_sigma = false;
        sweep(*s, M_INIT2, nullptr);
        pack_gf(s->Gr_in.data(), s->GL_in.data(), x, s->n_full, s->n_strict_upper, s->nA, s->n);
    } else if (s->order == 1) {
        std::fill(s->G_less_t0.begin(), s->G_less_t0.end(), 0.0);
        s->use_sigma = false;
        sweep(*s, M_SCF1, nullptr);
        gather_onsite(*s, s->site_int, s->G_less_t0);
        pack_nil(*s, s->G_less_t0, x);
    }
    return check_singular(s);
}

int qso_residual(qso_state *s, double Volt, const double *x, double *F, int *abort_flag) {
    hemb(*s);
    s->V_scf = Volt;
    bool ab = false;
    if (s->order == 2) {
        if (!s->sigma2_ready) sigma2_init(*s);
        scf_residual2(*s, s->n_vec, x, F, ab);
    } else if (s->order == 1) {
        scf_residual1(*s, s->n_vec, x, F, ab);
    }
    *abort_flag = ab;
    return check_singular(s);
}

int qso_self_energies(qso_state *s, const double *x, double *SigR2, double *SigL2, double *Sig1) {
    if (s->order != 2) return -1;
    if (!s->sigma2_ready) sigma2_init(*s);
    unpack_gf(s->Gr_in.data(), s->GL_in.data(), x, s->n_full, s->n_strict_upper, s->nA, s->n);
    equal_time_lesser(*s);
    sigma_first_order(*s);
    sigma2_compute(*s, true);
    if (SigR2) std::memcpy(SigR2, s->SigR2.data(), sizeof(cplx) * s->SigR2.size());
    if (SigL2) std::memcpy(SigL2, s->SigL2.data(), sizeof(cplx) * s->SigL2.size());
    if (Sig1) std::memcpy(Sig1, s->Sig1.data(), sizeof(cplx) * s->Sig1.size());
    return 0;
}

int qso_invert_batched(int N, int batch, double *A, int *info, int) {
    int bad = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : bad)
    for (int b = 0; b < batch; b++) {
        int64_t e = invert_complex(N, (cplx *)A + (size_t)b * N * N);
        info[b] = (int)e;
        bad += e != 0;
    }
    return bad ? 1 : 0;
}

int qso_pack_gf(int nb, int Nw, const double *Gr, const double *Gl, double *out) {
    int nf = nb * nb, nsu = (nf - nb) / 2;
    pack_gf((const cplx *)Gr, (const cplx *)Gl, out, nf, nsu, nb, Nw);
    return 0;
}
int qso_unpack_gf(int nb, int Nw, const double *in, double *Gr, double *Gl) {
    int nf = nb * nb, nsu = (nf - nb) / 2;
    unpack_gf((cplx *)Gr, (cplx *)Gl, in, nf, nsu, nb, Nw);
    return 0;
}

int qso_broyden_solve_host(qs_residual_fn residual, void *ctx, double *x, int64_t n, double alpha_mix, int nhist,
                           int maxscf, double tolf, int single_history, int *converged, int *n_iter, double *fmax,
                           qs_scf_step *log, int log_cap) {
    bool conv = false;
    int it = 0, resets = 0;
    double fm = 0;
    std::vector<qs_scf_step> lg;
    broyden_solve(
        [&](int64_t nn, const double *xx, double *F, bool &ab) {
            int a = 0;
            residual(ctx, nn, xx, F, &a);
            ab = a != 0;
        },
        x, n, alpha_mix, nhist, maxscf, tolf, single_history != 0, conv, it, fm, lg, resets);
    *converged = conv;
    *n_iter = it;
    *fmax = fm;
    for (int i = 0; i < (int)lg.size() && i < log_cap; i++) log[i] = lg[i];
    return 0;
}

// standalone FFT in the reference's convention (for the FFT pin against numpy)
int qso_fft(int n, double *data, int sign) {
    FFTPlan p;
    p.init(n);
    std::vector<cplx> w(n);
    p.exec((cplx *)data, w.data(), sign);
    return 0;
}
int qso_good_fft_size(int nmin) { return good_fft_size(nmin); }

// Timing helper of the CPU baseline (not a reference routine): qso_solve_scf with the wall
// time of every SCF iteration (residual + Broyden update) in step_seconds[0 .. n-1]; returns
// the number of iterations recorded (at most cap) or a negative status.
int qso_solve_scf_timed(qso_state *s, double Volt, int fresh_start, qs_scf_result *res, double *step_seconds,
                        int cap) {
    std::vector<double> t;
    g_step_times = &t;
    int rc = qso_solve_scf(s, Volt, fresh_start, res);
    g_step_times = nullptr;
    if (rc) return rc < 0 ? rc : -rc;
    t.push_back(std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count());
    int k = 0;
    for (; k + 1 < (int)t.size() && k < cap; k++) step_seconds[k] = t[k + 1] - t[k];
    // the last interval also holds the final sweep: drop it
    return std::max(0, k - 1);
}

// Timing helper of the CPU baseline (not a reference routine): seconds of one broyden_solve
// iteration without its residual, on a vector of n elements with a full history of nhist
// columns (single or double precision). The residual is a cheap contraction whose own time
// is measured and subtracted; the iterations after the history has filled are averaged. The
// residual moves its fixed point every call, so every step stores a history pair.
double qso_broyden_seconds_per_step(int64_t n, int nhist, int single) {
    using clk = std::chrono::steady_clock;
    const int steps = nhist + 4;
    std::vector<double> x(n, 0.0);
    std::vector<clk::time_point> t_call;
    std::vector<double> t_res;
    auto res = [&](int64_t nn, const double *xx, double *F, bool &ab) {
        auto t0 = clk::now();
        const double ph = 0.1 * (double)t_call.size();  // a moving target: F never vanishes
        t_call.push_back(t0);
#pragma omp parallel for
        for (int64_t i = 0; i < nn; i++) F[i] = 0.5 * (std::sin(1e-3 * (double)(i % 1000) + ph) - xx[i]);
        ab = false;
        t_res.push_back(std::chrono::duration<double>(clk::now() - t0).count());
    };
    bool conv;
    int it, resets;
    double fmax;
    std::vector<qs_scf_step> log;
    broyden_solve(res, x.data(), n, 0.5, nhist, steps, 0.0, single != 0, conv, it, fmax, log, resets);
    // interval between residual calls k and k+1 = residual k + the Broyden update of step k
    double s = 0.0;
    int cnt = 0;
    for (int k = nhist + 1; k + 1 < (int)t_call.size(); k++) {
        s += std::chrono::duration<double>(t_call[k + 1] - t_call[k]).count() - t_res[k];
        cnt++;
    }
    return cnt ? s / cnt : 0.0;
}

}  // extern "C"

// =====================================================================================
// SANCHO (SANCHO/src): the spinless chain to third order in U. TEST INFRASTRUCTURE, as the
// rest of this file: the checker of the B200 SANCHO solver (include/qsa200.h), exported as
// qsao_*. Paths below are relative to the reference project's SANCHO/ directory; the common/
// routines (pack_gf, invert_complex, broyden_solve) are the ones restated above.
// =====================================================================================
#include "../include/qsa200.h"

struct qsao_state {
    int Na = 0, n = 0, order = 0;
    std::vector<cplx> H, GammaL, GammaR;
    std::vector<double> U, omega;
    double mu = 0, beta = 0, delta = 0, alpha_mix = 0.3, tolf = 1e-6;
    int nhist = 8, maxscf = 200;
    // G_in, G_out: (Na, Na, n), element (a, b, k) at a + b Na + k Na^2
    std::vector<cplx> Gr, Ga, GL, GG, Or, Oa, OL, OG;
    std::vector<cplx> Glt0;  // G^<_ii(t=0)
    // self-energies (Na, Na, n); bubbles chi(m, a, b), m = -(n-1)..n-1, and phi(q, a, b), q = 2..2n
    std::vector<cplx> S2R, S2L, S2G, S3R, S3L, S3G;
    std::vector<cplx> chiG, chiL, chiR, chiA, phiG, phiL, phiR, phiA;
    int64_t n_vec = 0;
    int n_full = 0, n_strict_upper = 0;
    double V_scf = 0;
    int scf_iter = 0;
    int64_t singular = 0;
    std::string err;
    size_t ix(int a, int b, int k) const { return (size_t)a + (size_t)b * Na + (size_t)k * Na * Na; }
};

// fermi (src/green_functions.f90:46-53): no cap on the exponent here
static double sa_fermi(const qsao_state &s, double w, double V) {
    double arg = (w - s.mu + V / HBAR) * s.beta;
    return 1.0 / (std::exp(HBAR * arg) + 1.0);
}

// G^a = (G^r)^dagger per energy
static void sa_adjoint(const qsao_state &s, const std::vector<cplx> &R, std::vector<cplx> &A) {
    for (int k = 0; k < s.n; k++)
        for (int b = 0; b < s.Na; b++)
            for (int a = 0; a < s.Na; a++) A[s.ix(a, b, k)] = std::conj(R[s.ix(b, a, k)]);
}

// noninteracting_gr_ga + noninteracting_gl_gg (src/green_functions.f90:55-96)
static void sa_noninteracting(qsao_state &s, double Volt) {
    const int Na = s.Na;
    for (int k = 0; k < s.n; k++) {
        std::vector<cplx> w1((size_t)Na * Na);
        for (size_t q = 0; q < w1.size(); q++) w1[q] = -s.H[q] + 0.5 * (IM / HBAR) * (s.GammaL[q] + s.GammaR[q]);
        for (int i = 0; i < Na; i++) w1[i + (size_t)i * Na] += HBAR * s.omega[k];
        if (invert_complex(Na, w1.data()) != 0 && !s.singular) s.singular = k + 1;
        for (int b = 0; b < Na; b++)
            for (int a = 0; a < Na; a++) {
                s.Gr[s.ix(a, b, k)] = w1[a + (size_t)b * Na];
                s.Ga[s.ix(a, b, k)] = std::conj(w1[b + (size_t)a * Na]);
            }
        const double fL = sa_fermi(s, s.omega[k], Volt), fR = sa_fermi(s, s.omega[k], 0.0);
        std::vector<cplx> SL((size_t)Na * Na), T((size_t)Na * Na, 0.0);
        for (size_t q = 0; q < SL.size(); q++) SL[q] = IM * (fL * s.GammaL[q] + fR * s.GammaR[q]) / HBAR;
        for (int b = 0; b < Na; b++)
            for (int c = 0; c < Na; c++)
                for (int a = 0; a < Na; a++) T[a + (size_t)b * Na] += s.Gr[s.ix(a, c, k)] * SL[c + (size_t)b * Na];
        for (int b = 0; b < Na; b++)
            for (int a = 0; a < Na; a++) {
                cplx acc = 0.0;
                for (int c = 0; c < Na; c++) acc += T[a + (size_t)c * Na] * s.Ga[s.ix(c, b, k)];
                s.GL[s.ix(a, b, k)] = acc;
                s.GG[s.ix(a, b, k)] = acc + s.Gr[s.ix(a, b, k)] - s.Ga[s.ix(a, b, k)];
            }
    }
}

// complete_input_gf (src/green_functions.f90:164-173)
static void sa_complete_input(qsao_state &s) {
    sa_adjoint(s, s.Gr, s.Ga);
    for (size_t q = 0; q < s.Gr.size(); q++) s.GG[q] = s.GL[q] + s.Gr[q] - s.Ga[q];
}

// equal_time_lesser (src/green_functions.f90:98-114)
static void sa_equal_time_lesser(qsao_state &s) {
    const double pp = s.delta / (2.0 * PI);
    for (int i = 0; i < s.Na; i++) {
        cplx acc = 0.0;
        for (int k = 0; k < s.n; k++) acc += s.GL[s.ix(i, i, k)];
        s.Glt0[i] = acc * pp;
    }
}

// compute_bubbles (src/self_energies.f90:49-115): chi at nu = m delta (k2 = k1 - m on the
// grid), phi at Omega = 2 w_init + q delta (k2 = q - k1 on the grid); 0-based k here
static void sa_bubbles(qsao_state &s, int ord) {
    const int Na = s.Na, Nw = s.n, Nm = 2 * Nw - 1;
    const double pp = s.delta / (2.0 * PI);
    auto cx = [&](int m, int a, int b) { return (size_t)(m + Nw - 1) + (size_t)Nm * (a + (size_t)b * Na); };
    s.chiG.assign((size_t)Nm * Na * Na, 0.0);
    s.chiL = s.chiR = s.chiA = s.chiG;
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int b = 0; b < Na; b++)
        for (int a = 0; a < Na; a++)
            for (int m = -(Nw - 1); m <= Nw - 1; m++) {
                cplx s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
                for (int k1 = std::max(0, m); k1 <= std::min(Nw - 1, Nw - 1 + m); k1++) {
                    const int k2 = k1 - m;
                    s1 += s.GG[s.ix(a, b, k1)] * s.GL[s.ix(b, a, k2)];
                    s2 += s.GL[s.ix(a, b, k1)] * s.GG[s.ix(b, a, k2)];
                    s3 += s.Gr[s.ix(a, b, k1)] * s.GL[s.ix(b, a, k2)] + s.GL[s.ix(a, b, k1)] * s.Ga[s.ix(b, a, k2)];
                    s4 += s.Ga[s.ix(a, b, k1)] * s.GL[s.ix(b, a, k2)] + s.GL[s.ix(a, b, k1)] * s.Gr[s.ix(b, a, k2)];
                }
                s.chiG[cx(m, a, b)] = s1 * pp;
                s.chiL[cx(m, a, b)] = s2 * pp;
                s.chiR[cx(m, a, b)] = s3 * pp;
                s.chiA[cx(m, a, b)] = s4 * pp;
            }
    if (ord < 3) return;
    const int Nq = 2 * Nw - 1;  // q = 2..2 Nw (1-based energies): q0 = q - 2 = k1 + k2 (0-based), 0..2Nw-2
    s.phiG.assign((size_t)Nq * Na * Na, 0.0);
    s.phiL = s.phiR = s.phiA = s.phiG;
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int b = 0; b < Na; b++)
        for (int a = 0; a < Na; a++)
            for (int q0 = 0; q0 < Nq; q0++) {
                cplx s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0;
                for (int k1 = std::max(0, q0 - (Nw - 1)); k1 <= std::min(Nw - 1, q0); k1++) {
                    const int k2 = q0 - k1;
                    s1 += s.GG[s.ix(a, b, k1)] * s.GG[s.ix(a, b, k2)];
                    s2 += s.GL[s.ix(a, b, k1)] * s.GL[s.ix(a, b, k2)];
                    s3 += s.Gr[s.ix(a, b, k1)] * s.GG[s.ix(a, b, k2)] + s.GL[s.ix(a, b, k1)] * s.Gr[s.ix(a, b, k2)];
                    s4 += s.Ga[s.ix(a, b, k1)] * s.GG[s.ix(a, b, k2)] + s.GL[s.ix(a, b, k1)] * s.Ga[s.ix(a, b, k2)];
                }
                const size_t o = (size_t)q0 + (size_t)Nq * (a + (size_t)b * Na);
                s.phiG[o] = s1 * pp;
                s.phiL[o] = s2 * pp;
                s.phiR[o] = s3 * pp;
                s.phiA[o] = s4 * pp;
            }
}

// second_order_sigma (src/self_energies.f90:117-147)
static void sa_sigma2(qsao_state &s) {
    const int Na = s.Na, Nw = s.n, Nm = 2 * Nw - 1;
    const double pp = s.delta / (2.0 * PI);
    const cplx c2 = -(IM * HBAR) * (IM * HBAR);
    auto cx = [&](int m, int a, int b) { return (size_t)(m + Nw - 1) + (size_t)Nm * (a + (size_t)b * Na); };
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int j = 0; j < Na; j++)
        for (int i = 0; i < Na; i++)
            for (int iw = 0; iw < Nw; iw++) {
                cplx aR = 0.0, aL = 0.0, aG = 0.0;
                for (int m = std::max(iw - (Nw - 1), -(Nw - 1)); m <= std::min(iw, Nw - 1); m++) {
                    const int kk = iw - m;
                    aL += s.GL[s.ix(i, j, kk)] * s.chiL[cx(m, i, j)];
                    aG += s.GG[s.ix(i, j, kk)] * s.chiG[cx(m, i, j)];
                    aR += s.Gr[s.ix(i, j, kk)] * s.chiG[cx(m, i, j)] + s.GL[s.ix(i, j, kk)] * s.chiR[cx(m, i, j)];
                }
                const cplx f = c2 * s.U[i] * s.U[j] * pp;
                s.S2R[s.ix(i, j, iw)] = f * aR;
                s.S2L[s.ix(i, j, iw)] = f * aL;
                s.S2G[s.ix(i, j, iw)] = f * aG;
            }
}

// third_order_sigma (src/self_energies.f90:149-207)
static void sa_sigma3(qsao_state &s) {
    const int Na = s.Na, Nw = s.n, Nm = 2 * Nw - 1, Nq = 2 * Nw - 1;
    const double pp = s.delta / (2.0 * PI);
    const cplx c3 = -(IM * HBAR) * (IM * HBAR) * (IM * HBAR);
    auto cx = [&](int m, int a, int b) { return (size_t)(m + Nw - 1) + (size_t)Nm * (a + (size_t)b * Na); };
    auto px = [&](int q0, int a, int b) { return (size_t)q0 + (size_t)Nq * (a + (size_t)b * Na); };
    std::vector<cplx> SG((size_t)Nm * Na * Na, 0.0), SL(SG), SR(SG), PG((size_t)Nq * Na * Na, 0.0), PL(PG), PR(PG);
    // 2. D and E: products in frequency summed over the internal site k with U_k
#pragma omp parallel for collapse(2)
    for (int j = 0; j < Na; j++)
        for (int i = 0; i < Na; i++)
            for (int k = 0; k < Na; k++) {
                const double u = s.U[k];
                for (int m = 0; m < Nm; m++) {
                    const int mm = m - (Nw - 1);
                    SG[cx(mm, i, j)] += u * (s.chiR[cx(mm, i, k)] * s.chiG[cx(mm, k, j)] + s.chiG[cx(mm, i, k)] * s.chiA[cx(mm, k, j)]);
                    SL[cx(mm, i, j)] += u * (s.chiR[cx(mm, i, k)] * s.chiL[cx(mm, k, j)] + s.chiL[cx(mm, i, k)] * s.chiA[cx(mm, k, j)]);
                    SR[cx(mm, i, j)] += u * s.chiR[cx(mm, i, k)] * s.chiR[cx(mm, k, j)];
                }
                for (int q0 = 0; q0 < Nq; q0++) {
                    PG[px(q0, i, j)] += u * (s.phiR[px(q0, i, k)] * s.phiG[px(q0, k, j)] + s.phiG[px(q0, i, k)] * s.phiA[px(q0, k, j)]);
                    PL[px(q0, i, j)] += u * (s.phiR[px(q0, i, k)] * s.phiL[px(q0, k, j)] + s.phiL[px(q0, i, k)] * s.phiA[px(q0, k, j)]);
                    PR[px(q0, i, j)] += u * s.phiR[px(q0, i, k)] * s.phiR[px(q0, k, j)];
                }
            }
    // 3. convolution with the remaining GF: particle-hole G_ij(w - nu), particle-particle
    // G_ji(Omega - w) with q0 = iw + kk (0-based)
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int j = 0; j < Na; j++)
        for (int i = 0; i < Na; i++)
            for (int iw = 0; iw < Nw; iw++) {
                cplx aR = 0.0, aL = 0.0, aG = 0.0;
                for (int m = std::max(iw - (Nw - 1), -(Nw - 1)); m <= std::min(iw, Nw - 1); m++) {
                    const int kk = iw - m;
                    aL += s.GL[s.ix(i, j, kk)] * SL[cx(m, i, j)];
                    aG += s.GG[s.ix(i, j, kk)] * SG[cx(m, i, j)];
                    aR += s.Gr[s.ix(i, j, kk)] * SG[cx(m, i, j)] + s.GL[s.ix(i, j, kk)] * SR[cx(m, i, j)];
                }
                for (int kk = 0; kk < Nw; kk++) {
                    const int q0 = iw + kk;
                    aL += s.GG[s.ix(j, i, kk)] * PL[px(q0, i, j)];
                    aG += s.GL[s.ix(j, i, kk)] * PG[px(q0, i, j)];
                    aR += s.Ga[s.ix(j, i, kk)] * PG[px(q0, i, j)] + s.GG[s.ix(j, i, kk)] * PR[px(q0, i, j)];
                }
                const cplx f = c3 * s.U[i] * s.U[j] * pp;
                s.S3R[s.ix(i, j, iw)] = f * aR;
                s.S3L[s.ix(i, j, iw)] = f * aL;
                s.S3G[s.ix(i, j, iw)] = f * aG;
            }
}

// build_self_energies (src/self_energies.f90:40-47)
static void sa_self_energies(qsao_state &s) {
    if (s.order >= 2) {
        sa_bubbles(s, s.order);
        sa_sigma2(s);
    }
    if (s.order == 3) sa_sigma3(s);
}

// interacting_gf (src/scf.f90:147-195) at every energy
static void sa_interacting_sweep(qsao_state &s, double Volt) {
    const int Na = s.Na;
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < s.n; k++) {
        std::vector<cplx> SR((size_t)Na * Na, 0.0), SL((size_t)Na * Na, 0.0), w1((size_t)Na * Na);
        if (s.order == 1) {
            for (int i = 0; i < Na; i++) SR[i + (size_t)i * Na] -= IM * HBAR * s.U[i] * s.Glt0[i];
        } else if (s.order >= 2) {
            for (int b = 0; b < Na; b++)
                for (int a = 0; a < Na; a++) {
                    SR[a + (size_t)b * Na] = s.S2R[s.ix(a, b, k)];
                    SL[a + (size_t)b * Na] = s.S2L[s.ix(a, b, k)];
                }
            for (int j = 0; j < Na; j++) SR[j + (size_t)j * Na] -= IM * HBAR * s.U[j] * s.Glt0[j];
            if (s.order == 3)
                for (int b = 0; b < Na; b++)
                    for (int a = 0; a < Na; a++) {
                        SR[a + (size_t)b * Na] += s.S3R[s.ix(a, b, k)];
                        SL[a + (size_t)b * Na] += s.S3L[s.ix(a, b, k)];
                    }
        }
        const double w = s.omega[k];
        for (size_t q = 0; q < w1.size(); q++) w1[q] = -s.H[q] + 0.5 * (IM / HBAR) * (s.GammaL[q] + s.GammaR[q]) - SR[q];
        for (int i = 0; i < Na; i++) w1[i + (size_t)i * Na] += HBAR * w;
        if (invert_complex(Na, w1.data()) != 0) {
#pragma omp critical
            if (!s.singular) s.singular = k + 1;
        }
        const double fL = sa_fermi(s, w, Volt), fR = sa_fermi(s, w, 0.0);
        for (size_t q = 0; q < SL.size(); q++) SL[q] = IM * (fL * s.GammaL[q] + fR * s.GammaR[q]) / HBAR + SL[q];
        std::vector<cplx> T((size_t)Na * Na, 0.0);
        for (int b = 0; b < Na; b++)
            for (int c = 0; c < Na; c++)
                for (int a = 0; a < Na; a++) T[a + (size_t)b * Na] += w1[a + (size_t)c * Na] * SL[c + (size_t)b * Na];
        for (int b = 0; b < Na; b++)
            for (int a = 0; a < Na; a++) {
                cplx acc = 0.0;
                for (int c = 0; c < Na; c++) acc += T[a + (size_t)c * Na] * std::conj(w1[b + (size_t)c * Na]);
                const cplx gr = w1[a + (size_t)b * Na], ga = std::conj(w1[b + (size_t)a * Na]);
                s.Or[s.ix(a, b, k)] = gr;
                s.Oa[s.ix(a, b, k)] = ga;
                s.OL[s.ix(a, b, k)] = acc;
                s.OG[s.ix(a, b, k)] = acc + gr - ga;
            }
    }
}

// check_gf_sanity (common/scf_checks.f90) on the diagonals of a (Na, Na, n) pair
static void sa_sanity(const qsao_state &s, const std::vector<cplx> &R, const std::vector<cplx> &L, bool &runaway,
                      bool &unphysical, int &i_worst, double &n_worst, double &w_worst) {
    std::vector<cplx> rd((size_t)s.Na * s.n), ld((size_t)s.Na * s.n);
    for (int k = 0; k < s.n; k++)
        for (int i = 0; i < s.Na; i++) {
            rd[i + (size_t)k * s.Na] = R[s.ix(i, i, k)];
            ld[i + (size_t)k * s.Na] = L[s.ix(i, i, k)];
        }
    check_diag_sanity(rd.data(), ld.data(), s.Na, s.n, s.delta, runaway, unphysical, i_worst, n_worst, w_worst,
                      nullptr);
}

// scf_residual (src/scf.f90:102-136)
static void sa_residual(qsao_state &s, int64_t n, const double *x, double *F, bool &abort) {
    s.scf_iter++;
    unpack_gf(s.Gr.data(), s.GL.data(), x, s.n_full, s.n_strict_upper, s.Na, s.n);
    sa_complete_input(s);
    sa_equal_time_lesser(s);
    sa_self_energies(s);
    sa_interacting_sweep(s, s.V_scf);
    bool unphys;
    int iw;
    double nw, ww;
    sa_sanity(s, s.Or, s.OL, abort, unphys, iw, nw, ww);
    if (abort) {
        std::fill(F, F + n, 0.0);
        return;
    }
    pack_gf(s.Or.data(), s.OL.data(), F, s.n_full, s.n_strict_upper, s.Na, s.n);
    for (int64_t i = 0; i < n; i++) F[i] -= x[i];
}

extern "C" {

int qsao_create(const qsa_problem *p, qsao_state **out) {
    scipy_openblas_set_num_threads64_(1);
    auto *s = new qsao_state();
    s->Na = p->N_sites;
    s->n = p->n_omega;
    s->order = p->order;
    const size_t nn = (size_t)s->Na * s->Na;
    s->H.assign((const cplx *)p->H, (const cplx *)p->H + nn);
    s->GammaL.assign((const cplx *)p->GammaL, (const cplx *)p->GammaL + nn);
    s->GammaR.assign((const cplx *)p->GammaR, (const cplx *)p->GammaR + nn);
    s->U.assign(p->U_site, p->U_site + s->Na);
    s->omega.assign(p->omega, p->omega + s->n);
    s->mu = p->mu;
    s->beta = p->beta;
    s->delta = p->delta;
    s->alpha_mix = p->alpha_mix;
    s->tolf = p->tolf;
    s->nhist = p->nhist;
    s->maxscf = p->maxscf;
    const size_t tot = nn * s->n;
    for (auto *v : {&s->Gr, &s->Ga, &s->GL, &s->GG, &s->Or, &s->Oa, &s->OL, &s->OG, &s->S2R, &s->S2L, &s->S2G, &s->S3R,
                    &s->S3L, &s->S3G})
        v->assign(tot, 0.0);
    s->Glt0.assign(s->Na, 0.0);
    // src/sancho.f90:106-109
    s->n_full = (int)nn;
    s->n_strict_upper = (s->n_full - s->Na) / 2;
    s->n_vec = (int64_t)(2 * s->n_full + s->n_strict_upper + s->n_strict_upper + s->Na) * s->n;
    *out = s;
    return 0;
}
void qsao_destroy(qsao_state *s) { delete s; }
const char *qsao_last_error(const qsao_state *s) { return s ? s->err.c_str() : "no handle"; }
int64_t qsao_vector_length(const qsao_state *s) { return s->n_vec; }

static int sa_check_singular(qsao_state *s) {
    if (s->singular) {
        s->err = "ERROR: ZGETRF failed (singular matrix?) at energy " + std::to_string(s->singular);
        int e = (int)s->singular;
        s->singular = 0;
        return e;
    }
    return 0;
}

// solve_scf (src/scf.f90:53-95)
int qsao_solve_scf(qsao_state *s, double Volt, int fresh_start, qs_scf_result *res) {
    auto t0 = std::chrono::steady_clock::now();
    if (fresh_start) sa_noninteracting(*s, Volt);
    if (int e = sa_check_singular(s)) return e;
    std::vector<double> x(s->n_vec);
    pack_gf(s->Gr.data(), s->GL.data(), x.data(), s->n_full, s->n_strict_upper, s->Na, s->n);
    s->V_scf = Volt;
    s->scf_iter = 0;
    bool converged, aborted = false;
    int n_iter = 0, n_resets = 0;
    double fmax = 0.0;
    std::vector<qs_scf_step> log;
    broyden_solve([&](int64_t n, const double *xx, double *F, bool &ab) { sa_residual(*s, n, xx, F, ab); aborted = aborted || ab; },
                  x.data(), s->n_vec, s->alpha_mix, s->nhist, s->maxscf, s->tolf, false, converged, n_iter, fmax, log,
                  n_resets);
    if (int e = sa_check_singular(s)) return e;
    bool runaway, unphysical;
    int i_worst;
    double n_worst, w_worst;
    sa_sanity(*s, s->Or, s->OL, runaway, unphysical, i_worst, n_worst, w_worst);
    if (converged && unphysical) converged = false;
    res->converged = converged && !aborted;
    res->n_iter = n_iter;
    res->fmax = fmax;
    res->aborted = aborted;
    res->runaway = runaway;
    res->unphysical = unphysical;
    res->i_worst = i_worst;
    res->n_worst = n_worst;
    res->w_worst = w_worst;
    res->n_resets = n_resets;
    res->n_log = 0;
    for (auto &e : log)
        if (res->log && res->n_log < res->log_cap) res->log[res->n_log++] = e;
    res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    res->n_mixed = 0;
    return 0;
}

// Current (src/observables.f90:18-52): 2 (delta/hbar) sum_w Re Tr{i GammaL [(fL - 1) G^< - fL G^>]}/2pi
int qsao_current(qsao_state *s, double Volt, double *J) {
    double JL = 0.0;
    for (int k = 0; k < s->n; k++) {
        const double fL = sa_fermi(*s, s->omega[k], Volt);
        cplx tr = 0.0;
        for (int a = 0; a < s->Na; a++)
            for (int c = 0; c < s->Na; c++)
                tr += IM * s->GammaL[a + (size_t)c * s->Na] *
                      ((fL - 1.0) * s->GL[s->ix(c, a, k)] - fL * s->GG[s->ix(c, a, k)]);
        JL += tr.real() / (2.0 * PI);
    }
    *J = 2.0 * JL * (s->delta / HBAR);
    return 0;
}

int qsao_get_observables(qsao_state *s, double *G_less_t0, double *spectral) {
    if (G_less_t0) std::memcpy(G_less_t0, s->Glt0.data(), sizeof(cplx) * s->Na);
    if (spectral)
        for (int k = 0; k < s->n; k++)
            for (int i = 0; i < s->Na; i++) spectral[i + (size_t)k * s->Na] = -2.0 * s->Gr[s->ix(i, i, k)].imag();
    return 0;
}

int qsao_initial_vector(qsao_state *s, double Volt, double *x) {
    sa_noninteracting(*s, Volt);
    pack_gf(s->Gr.data(), s->GL.data(), x, s->n_full, s->n_strict_upper, s->Na, s->n);
    return sa_check_singular(s);
}

int qsao_residual(qsao_state *s, double Volt, const double *x, double *F, int *abort_flag) {
    s->V_scf = Volt;
    bool ab = false;
    sa_residual(*s, s->n_vec, x, F, ab);
    *abort_flag = ab;
    return sa_check_singular(s);
}

int qsao_self_energies(qsao_state *s, const double *x, double *Sig2R, double *Sig2L, double *Sig3R, double *Sig3L) {
    unpack_gf(s->Gr.data(), s->GL.data(), x, s->n_full, s->n_strict_upper, s->Na, s->n);
    sa_complete_input(*s);
    sa_equal_time_lesser(*s);
    sa_self_energies(*s);
    const size_t bytes = sizeof(cplx) * s->S2R.size();
    if (Sig2R) std::memcpy(Sig2R, s->S2R.data(), bytes);
    if (Sig2L) std::memcpy(Sig2L, s->S2L.data(), bytes);
    if (Sig3R) std::memcpy(Sig3R, s->S3R.data(), bytes);
    if (Sig3L) std::memcpy(Sig3L, s->S3L.data(), bytes);
    return 0;
}

}  // extern "C"
