// sancho.cu -- SANCHO (the spinless chain to third order in U) on B200, and the C ABI of
// include/qsa200.h. Paths in the citations are relative to the reference project's SANCHO/
// directory.
//
// SANCHO keeps every Green's function in full (Na, Na, n_omega) storage and builds its
// self-energies from particle-hole and particle-particle bubbles as direct sums over the
// energy grid (src/self_energies.f90:49-207): O(Na^2 n^2) complex multiply-adds per SCF
// iteration, the whole cost of an iteration at any useful grid. On the device:
//
//   x (pack_gf layout)  --sa_unpack-->  E_r, E_a, E_<, E_>   element-major sequences:
//                                       element e = a + b Na holds its n energies
//                                       contiguously ([e*n + k]), the layout every lag sum
//                                       streams through shared memory
//   lag sums            one kernel template for the four direct sums of the method:
//                         chi(m)   = sum_k1 A(k1) B(k1 - m)   particle-hole bubbles
//                         phi(q)   = sum_k1 A(k1) B(q - k1)   particle-particle bubbles
//                         S_ph(w)  = sum_k  A(k) chi(w - k)   convolution with G_ij
//                         S_pp(w)  = sum_k  A(k) phi(w + k)   convolution with G_ji
//                       a block of 128 threads owns 256 consecutive outputs of one element
//                       (two adjacent ones a thread) and walks the summation index in tiles:
//                       128 values of each A sequence and the 383-long window of each B
//                       sequence the tile's outputs touch are staged in shared memory (zero
//                       outside the sequences, so no bounds test in the inner loop); every
//                       thread then runs the tile's multiply-adds from shared memory (A
//                       broadcast, one new B value per step for its two outputs)
//   D, E products       order 3: the U_k-weighted products of bubbles over the internal
//                       site k at every m and q (small Na x Na products per energy)
//   Dyson               W(w) = hbar w - H + i(GammaL + GammaR)/2 - Sigma^r(w), inverted by
//                       the solver's batched Gauss-Jordan kernels (all energies at once)
//   Keldysh + pack      G^< = G^r Sigma^<_tot G^a in two batched products, written straight
//                       into pack_gf's layout minus x (the SCF residual), with the
//                       diagonals for check_gf_sanity
//   Broyden             the solver's device Broyden (double-precision history, as the
//                       reference calls broyden_solve)
//
// The bubble sums run their summation index in the reference's order; the convolutions of
// step 3 run theirs backwards (ascending k instead of ascending m), so the results agree with
// the reference's to FP64 rounding, not bit for bit.
//
// The calls that take an x (qsa_residual, qsa_self_energies) and qsa_initial_vector leave
// that x as the handle's G_in, as the reference's module state does: a continued solve
// starts from it.
#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <string>
#include <vector>

#include "qs_common.cuh"
#include "qsa200.h"

namespace qs {
int broyden_solve_dev(qs_handle *h, BroydenResidual &res, double *&d_x, double *&d_F, double *&d_Fold,
                      double *&d_xold, void *d_hdF, void *d_hU, int64_t n, double alpha_mix, int nhist, int maxscf,
                      double tolf, bool sp, BroydenOut &out);
size_t broyden_red_len();
}  // namespace qs

using namespace qs;

struct qsa_handle {
    qs_handle q;  // stream, Broyden vectors and scratch, allocation list, error text
    int Na = 0, n = 0, order = 0, Nm = 0;
    int64_t n_vec = 0;
    double mu = 0, beta = 0, delta = 0, alpha_mix = 0.3, tolf = 1e-6;
    int nhist = 8, maxscf = 200;
    std::vector<double> omega;
    zc *d_H = nullptr, *d_GamL = nullptr, *d_GamR = nullptr;
    double *d_U = nullptr, *d_omega = nullptr;
    zc *d_E[4] = {};    // G_in element-major: r, a, <, >
    zc *d_chi[4] = {};  // > , <, r, a   [e*Nm + m + n - 1]
    zc *d_phi[4] = {};  // > , <, r, a   [e*Nm + q0]        (order 3)
    zc *d_D[3] = {};    // sum_k U_k chi chi:  >, <, r     (order 3)
    zc *d_P[3] = {};    // sum_k U_k phi phi:  >, <, r     (order 3)
    zc *d_S2R = nullptr, *d_S2L = nullptr, *d_S3R = nullptr, *d_S3L = nullptr;  // [e + k Na^2]
    zc *d_Glt0 = nullptr;
    zc *d_W = nullptr, *d_T = nullptr;  // Dyson batch (-> G^r out), G^r Sigma^< products
    zc *d_ws = nullptr;
    int ws_slots = 0;
    zc *d_gRd = nullptr, *d_gLd = nullptr;  // [k*Na + i]
    double *d_spec = nullptr;
    zc *d_sums = nullptr;
    int *d_info = nullptr;  // [0]: first singular energy + 1 (INT_MAX: none); [1..n]: per energy
    SanityOut last;         // check_gf_sanity of the last residual's G_out
    bool have_x = false;
};

namespace {

constexpr int LT = 128;          // threads per block and summation values per tile
constexpr int NP = 2 * LT;       // outputs per block: two adjacent ones per thread
constexpr int LW = LT + NP - 1;  // B window of a tile
constexpr int LH = (LW + 1) / 2; // the window is stored de-interleaved: even slots, then odd ones
constexpr double HB = 1.0;       // hbar (common/constants.f90:19)

// ---------------------------------------------------------------------------------
// pack_gf layout (common/linear_algebra.f90:155-191), block of 3 Na^2 doubles per energy:
// Re G^r (row-major i,j) | Im G^r | Re G^< strict upper (row-major, j > i) |
// Im G^< upper (row-major, j >= i)
// ---------------------------------------------------------------------------------
__device__ __forceinline__ int up_idx(int nb, int p, int q) { return p * nb - p * (p - 1) / 2 + (q - p); }
__device__ __forceinline__ int sup_idx(int nb, int p, int q) { return p * (nb - 1) - p * (p - 1) / 2 + (q - p - 1); }

__device__ __forceinline__ zc pk_gr(const double *b, int nb, int i, int j) {
    const int nf = nb * nb;
    return zc{b[i * nb + j], b[nf + i * nb + j]};
}
// unpack_gf rebuilds the lower triangle as G^<_ji = -conj(G^<_ij) (common/linear_algebra.f90:222-223)
__device__ __forceinline__ zc pk_gl(const double *b, int nb, int i, int j) {
    const int nf = nb * nb, nsu = (nf - nb) / 2;
    const int p = i <= j ? i : j, q = i <= j ? j : i;
    const double re = (p == q) ? 0.0 : b[2 * nf + sup_idx(nb, p, q)];
    const double im = b[2 * nf + nsu + up_idx(nb, p, q)];
    return (i <= j) ? zc{re, im} : zc{-re, im};
}

// unpack_gf + complete_input_gf (src/green_functions.f90:164-173) into element-major
// sequences: G^a_ab = conj(G^r_ba), G^>_ab = G^<_ab + G^r_ab - G^a_ab
__global__ void sa_unpack(int Na, int n, const double *__restrict__ x, zc *__restrict__ Er, zc *__restrict__ Ea,
                          zc *__restrict__ EL, zc *__restrict__ EG) {
    const int64_t blk = 3 * (int64_t)Na * Na, tot = (int64_t)n * Na * Na;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(t % n), e = (int)(t / n), a = e % Na, b = e / Na;
        const double *B = x + k * blk;
        const zc r = pk_gr(B, Na, a, b), ad = conj(pk_gr(B, Na, b, a)), l = pk_gl(B, Na, a, b);
        Er[t] = r;
        Ea[t] = ad;
        EL[t] = l;
        EG[t] = (l + r) - ad;
    }
}

// equal_time_lesser (src/green_functions.f90:98-114): G^<_ii(t=0) = delta/2pi sum_w G^<_ii(w)
__global__ void sa_glt0(int Na, int n, const zc *__restrict__ EL, double pp, zc *__restrict__ Glt0) {
    __shared__ zc red[256];
    const int i = blockIdx.x;
    const zc *s = EL + ((size_t)i + (size_t)i * Na) * n;
    zc acc{0.0, 0.0};
    for (int k = threadIdx.x; k < n; k += blockDim.x) acc = acc + s[k];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) Glt0[i] = pp * red[0];
}

// ---------------------------------------------------------------------------------
// Lag sums. Output p of an element, summation index j in [0, n): the B index is
// b = SG*j + TG*p + c. A tile covers j in [J0, J0 + LT) and the block's outputs
// p in [P0, P0 + NP), so it touches b in a window of LW values (slot = b - wbase).
// Thread t owns the adjacent outputs 2t and 2t + 1: at a given j the second needs the
// window value TG slots from the first's, which is the value the first needed one step
// earlier in the walk (j ascending for (SG, TG) = (+1, -1) and (-1, +1), descending for
// (+1, +1)); so each step loads one window value per B sequence for two outputs. The
// window is stored with its even slots first and its odd slots after them: the lanes of a
// warp read slots 2t + const, which land on consecutive 16-byte words.
// ---------------------------------------------------------------------------------
template <int SG, int TG>
struct LagMap {
    static constexpr bool ASC = !(SG > 0 && TG > 0);  // the order of the walk over a tile
    __device__ static int wbase(int J0, int P0, int c) {
        return SG * (SG > 0 ? J0 : J0 + LT - 1) + TG * (TG > 0 ? P0 : P0 + NP - 1) + c;
    }
    // window slot of (J0 + jj, P0 + tp), in [0, LW)
    __device__ static int slot(int jj, int tp) {
        return SG * (SG > 0 ? jj : jj - (LT - 1)) + TG * (TG > 0 ? tp : tp - (NP - 1));
    }
    // j range (inclusive) with b in [0, Lb) for some p of the block, within [0, n)
    __device__ static void jrange(int P0, int c, int Lb, int n, int &jlo, int &jhi) {
        const int t0 = TG * P0, t1 = TG * (P0 + NP - 1);
        const int tmin = min(t0, t1), tmax = max(t0, t1);
        if (SG > 0) {
            jlo = -tmax - c;
            jhi = Lb - 1 - tmin - c;
        } else {
            jlo = tmin + c - Lb + 1;
            jhi = tmax + c;
        }
        jlo = max(jlo, 0);
        jhi = min(jhi, n - 1);
    }
};
__device__ __forceinline__ int wpos(int u) { return (u & 1) * LH + (u >> 1); }

// stage NA sequences of A at [J0, J0 + LT) and NB sequences of B on the tile's window
template <int NA, int NB>
__device__ __forceinline__ void lag_stage(const zc *const (&A)[NA], const zc *const (&B)[NB], int n, int Lb, int J0,
                                          int wb, zc (*sA)[LT], zc (*sB)[2 * LH]) {
    const int t = threadIdx.x;
#pragma unroll
    for (int s = 0; s < NA; s++) {
        const int j = J0 + t;
        sA[s][t] = (j >= 0 && j < n) ? A[s][j] : zc{0.0, 0.0};
    }
#pragma unroll
    for (int s = 0; s < NB; s++)
        for (int u = t; u < LW; u += LT) {
            const int b = wb + u;
            sB[s][wpos(u)] = (b >= 0 && b < Lb) ? B[s][b] : zc{0.0, 0.0};
        }
}

// The tiles of one lag sum for the thread's outputs 2t, 2t + 1: step(a, cur, prev) gets
// the NA values of A at j, the NB window values of output 2t (cur) and of output 2t + 1
// (prev, the previous step's cur).
template <int SG, int TG, int NA, int NB, class Step>
__device__ __forceinline__ void lag_walk(const zc *const (&A)[NA], const zc *const (&B)[NB], int n, int Lb, int P0,
                                         int c, zc (*sA)[LT], zc (*sB)[2 * LH], Step step) {
    using M = LagMap<SG, TG>;
    int jlo, jhi;
    M::jrange(P0, c, Lb, n, jlo, jhi);
    const int tp = 2 * threadIdx.x;
    for (int J0 = jlo; J0 <= jhi; J0 += LT) {
        __syncthreads();
        lag_stage<NA, NB>(A, B, n, Lb, J0, M::wbase(J0, P0, c), sA, sB);
        __syncthreads();
        const int nj = min(LT, jhi - J0 + 1);
        zc prev[NB], cur[NB], av[NA];
        {
            const int w1 = wpos(M::slot(M::ASC ? 0 : nj - 1, tp) + TG);
#pragma unroll
            for (int s = 0; s < NB; s++) prev[s] = sB[s][w1];
        }
        for (int it = 0; it < nj; it++) {
            const int jj = M::ASC ? it : nj - 1 - it;
            const int w0 = wpos(M::slot(jj, tp));
#pragma unroll
            for (int s = 0; s < NB; s++) cur[s] = sB[s][w0];
#pragma unroll
            for (int s = 0; s < NA; s++) av[s] = sA[s][jj];
            step(av, cur, prev);
#pragma unroll
            for (int s = 0; s < NB; s++) prev[s] = cur[s];
        }
    }
}

// compute_bubbles (src/self_energies.f90:49-115). Grid (ceil(Nm/NP), Na^2), block LT.
//   PH (chi, m = p - (n-1)): A = {G^>, G^<, G^r, G^a}_ab (k1), B = {G^<, G^>, G^a, G^r}_ba (k1 - m)
//   PP (phi, q0 = p):        A = {G^>, G^<, G^r, G^a}_ab (k1), B = {G^>, G^<, G^r, G^a}_ab (q0 - k1)
// with the same products: s1 = A0 B0, s2 = A1 B1, s3 = A2 B0 + A1 B2, s4 = A3 B0 + A1 B3
// (chi^>, chi^<, chi^r, chi^a; phi likewise), each times delta/2pi.
template <bool PH>
__global__ void __launch_bounds__(LT) sa_bubbles(int Na, int n, const zc *__restrict__ Er, const zc *__restrict__ Ea,
                                                 const zc *__restrict__ EL, const zc *__restrict__ EG, double pp,
                                                 zc *__restrict__ oG, zc *__restrict__ oL, zc *__restrict__ oR,
                                                 zc *__restrict__ oA) {
    __shared__ zc sA[4][LT];
    __shared__ zc sB[4][2 * LH];
    const int Nm = 2 * n - 1, e = blockIdx.y, a = e % Na, b = e / Na;
    const int eb = PH ? (b + a * Na) : e;
    const size_t oe = (size_t)e * n, ob = (size_t)eb * n;
    const zc *const A[4] = {EG + oe, EL + oe, Er + oe, Ea + oe};
    const zc *const B[4] = {PH ? EL + ob : EG + ob, PH ? EG + ob : EL + ob, PH ? Ea + ob : Er + ob,
                            PH ? Er + ob : Ea + ob};
    const int c = PH ? (n - 1) : 0;  // chi: b = k1 - (p - (n-1)); phi: b = p - k1
    const int P0 = blockIdx.x * NP, p = P0 + 2 * threadIdx.x;
    zc s[2][4] = {};
    auto step = [&](const zc (&av)[4], const zc (&b0)[4], const zc (&b1)[4]) {
        cfma(s[0][0], av[0], b0[0]);
        cfma(s[0][1], av[1], b0[1]);
        cfma(s[0][2], av[2], b0[0]);
        cfma(s[0][2], av[1], b0[2]);
        cfma(s[0][3], av[3], b0[0]);
        cfma(s[0][3], av[1], b0[3]);
        cfma(s[1][0], av[0], b1[0]);
        cfma(s[1][1], av[1], b1[1]);
        cfma(s[1][2], av[2], b1[0]);
        cfma(s[1][2], av[1], b1[2]);
        cfma(s[1][3], av[3], b1[0]);
        cfma(s[1][3], av[1], b1[3]);
    };
    if (PH) lag_walk<1, -1, 4, 4>(A, B, n, n, P0, c, sA, sB, step);
    else lag_walk<-1, 1, 4, 4>(A, B, n, n, P0, c, sA, sB, step);
#pragma unroll
    for (int r = 0; r < 2; r++)
        if (p + r < Nm) {
            const size_t o = (size_t)e * Nm + p + r;
            oG[o] = pp * s[r][0];
            oL[o] = pp * s[r][1];
            oR[o] = pp * s[r][2];
            oA[o] = pp * s[r][3];
        }
}

// second_order_sigma / third_order_sigma step 3 (src/self_energies.f90:117-207).
// Grid (ceil(n/NP), Na^2), block LT; p = iw, j = kk.
//   particle-hole part: A = {G^<, G^>, G^r}_ij (kk), B = {X^<, X^>, X^r}_ij (m = iw - kk)
//   particle-particle part (order 3): A = {G^>, G^<, G^a}_ji (kk), B = {P^<, P^>, P^r}_ij (iw + kk)
// a^< += A0 B0, a^r += A2 B1 + A0 B2; Sigma = f a with f = c U_i U_j delta/2pi.
__global__ void __launch_bounds__(LT) sa_sigma(int Na, int n, const zc *__restrict__ Er, const zc *__restrict__ Ea,
                                               const zc *__restrict__ EL, const zc *__restrict__ EG,
                                               const zc *__restrict__ XL, const zc *__restrict__ XG,
                                               const zc *__restrict__ XR, const zc *__restrict__ PL,
                                               const zc *__restrict__ PG, const zc *__restrict__ PR,
                                               const double *__restrict__ U, zc fc, zc *__restrict__ SR,
                                               zc *__restrict__ SL) {
    __shared__ zc sA[3][LT];
    __shared__ zc sB[3][2 * LH];
    const int Nm = 2 * n - 1, e = blockIdx.y, i = e % Na, j = e / Na;
    const int P0 = blockIdx.x * NP, p = P0 + 2 * threadIdx.x;
    zc aL[2] = {}, aR[2] = {};
    auto step = [&](const zc (&av)[3], const zc (&b0)[3], const zc (&b1)[3]) {
        cfma(aL[0], av[0], b0[0]);
        cfma(aR[0], av[2], b0[1]);
        cfma(aR[0], av[0], b0[2]);
        cfma(aL[1], av[0], b1[0]);
        cfma(aR[1], av[2], b1[1]);
        cfma(aR[1], av[0], b1[2]);
    };
    {
        // chi index m + n - 1 = iw - kk + n - 1
        const size_t oe = (size_t)e * n, ox = (size_t)e * Nm;
        const zc *const A[3] = {EL + oe, EG + oe, Er + oe};
        const zc *const B[3] = {XL + ox, XG + ox, XR + ox};
        lag_walk<-1, 1, 3, 3>(A, B, n, Nm, P0, n - 1, sA, sB, step);
    }
    if (PL) {
        // q0 = iw + kk
        const size_t oe = ((size_t)j + (size_t)i * Na) * n, ox = (size_t)e * Nm;
        const zc *const A[3] = {EG + oe, EL + oe, Ea + oe};
        const zc *const B[3] = {PL + ox, PG + ox, PR + ox};
        lag_walk<1, 1, 3, 3>(A, B, n, Nm, P0, 0, sA, sB, step);
    }
    const zc f = (U[i] * U[j]) * fc;
#pragma unroll
    for (int r = 0; r < 2; r++)
        if (p + r < n) {
            const size_t o = (size_t)e + (size_t)(p + r) * Na * Na;
            SR[o] = f * aR[r];
            SL[o] = f * aL[r];
        }
}

// third_order_sigma step 2 (src/self_energies.f90:160-185): per m (or q0) and (i, j)
//   X^> = sum_k U_k (Y^r_ik Y^>_kj + Y^>_ik Y^a_kj), X^< likewise with Y^<, X^r = sum_k U_k Y^r_ik Y^r_kj
// for Y = chi (X = D) and Y = phi (X = P). Thread per (p, e), p fastest.
__global__ void sa_products(int Na, int Nm, const zc *__restrict__ YG, const zc *__restrict__ YL,
                            const zc *__restrict__ YR, const zc *__restrict__ YA, const double *__restrict__ U,
                            zc *__restrict__ XG, zc *__restrict__ XL, zc *__restrict__ XR) {
    const int64_t tot = (int64_t)Nm * Na * Na;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
        const int p = (int)(t % Nm), e = (int)(t / Nm), i = e % Na, j = e / Na;
        zc g{0, 0}, l{0, 0}, r{0, 0};
        for (int k = 0; k < Na; k++) {
            const size_t ik = ((size_t)i + (size_t)k * Na) * Nm + p, kj = ((size_t)k + (size_t)j * Na) * Nm + p;
            const double u = U[k];
            const zc rik = YR[ik];
            g = g + u * (rik * YG[kj] + YG[ik] * YA[kj]);
            l = l + u * (rik * YL[kj] + YL[ik] * YA[kj]);
            r = r + u * (rik * YR[kj]);
        }
        XG[t] = g;
        XL[t] = l;
        XR[t] = r;
    }
}

// interacting_gf (src/scf.f90:147-195) / noninteracting_gr_ga (src/green_functions.f90:55-72):
// W(w) = hbar w - H + (i/2hbar)(GammaL + GammaR) - Sigma^r(w), Sigma^r = Sigma2^r - i hbar U_j
// G^<_jj(t=0) on the diagonal (+ Sigma3^r). Thread per (e, k), e fastest.
__global__ void sa_dyson_build(int Na, int n, int order, const zc *__restrict__ H, const zc *__restrict__ GamL,
                               const zc *__restrict__ GamR, const double *__restrict__ omega,
                               const zc *__restrict__ S2R, const zc *__restrict__ S3R, const double *__restrict__ U,
                               const zc *__restrict__ Glt0, zc *__restrict__ W) {
    const int nf = Na * Na;
    const int64_t tot = (int64_t)n * nf;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
        const int e = (int)(t % nf), a = e % Na, b = e / Na;
        const int64_t k = t / nf;
        zc sr{0.0, 0.0};
        if (order >= 2) sr = S2R[t];
        if (order >= 1 && a == b) sr = sr - (zc{0.0, HB * U[a]} * Glt0[a]);
        if (order == 3) sr = sr + S3R[t];
        const zc g = GamL[e] + GamR[e];
        zc w = (-H[e] + zc{-0.5 / HB * g.y, 0.5 / HB * g.x}) - sr;
        if (a == b) w.x += HB * omega[k];
        W[t] = w;
    }
}

// fermi (src/green_functions.f90:46-53)
__device__ __forceinline__ double sa_fermi(double w, double V, double mu, double beta) {
    return 1.0 / (exp(HB * ((w - mu + V / HB) * beta)) + 1.0);
}

// T = G^r Sigma^<_tot, Sigma^<_tot = i(fL GammaL + fR GammaR)/hbar + Sigma2^< (+ Sigma3^<)
// (src/scf.f90:180-188, src/green_functions.f90:74-96). Thread per (e, k).
__global__ void sa_keldysh_T(int Na, int n, const zc *__restrict__ Gr, const zc *__restrict__ GamL,
                             const zc *__restrict__ GamR, const zc *__restrict__ S2L, const zc *__restrict__ S3L,
                             const double *__restrict__ omega, double V, double mu, double beta, zc *__restrict__ T) {
    const int nf = Na * Na;
    const int64_t tot = (int64_t)n * nf;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
        const int e = (int)(t % nf), a = e % Na, b = e / Na;
        const int64_t k = t / nf;
        const double fL = sa_fermi(omega[k], V, mu, beta), fR = sa_fermi(omega[k], 0.0, mu, beta);
        const zc *G = Gr + k * nf;
        zc acc{0.0, 0.0};
        for (int c = 0; c < Na; c++) {
            const int cb = c + b * Na;
            zc sl{0.0, 0.0};
            if (S2L) sl = S2L[k * nf + cb];
            if (S3L) sl = sl + S3L[k * nf + cb];
            const zc g = fL * GamL[cb] + fR * GamR[cb];
            sl = zc{-g.y / HB, g.x / HB} + sl;
            cfma(acc, G[a + c * Na], sl);
        }
        T[t] = acc;
    }
}

// G^< = T G^a per (a <= b) and energy, written with G^r into pack_gf's layout, minus x when
// x is given (the SCF residual F = pack(G_out) - x); diagonals for check_gf_sanity.
// Thread per (e, k), e fastest.
__global__ void sa_keldysh_pack(int Na, int n, const zc *__restrict__ Gr, const zc *__restrict__ T,
                                const double *__restrict__ x, double *__restrict__ out, zc *__restrict__ gRd,
                                zc *__restrict__ gLd) {
    const int nf = Na * Na, nsu = (nf - Na) / 2;
    const int64_t tot = (int64_t)n * nf, blk = 3 * (int64_t)nf;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
        const int e = (int)(t % nf), a = e % Na, b = e / Na;
        const int64_t k = t / nf;
        const zc *G = Gr + k * nf, *Tk = T + k * nf;
        double *o = out + k * blk;
        const double *xs = x ? x + k * blk : nullptr;
        const zc r = G[e];
        const int pr = a * Na + b;
        o[pr] = xs ? r.x - xs[pr] : r.x;
        o[nf + pr] = xs ? r.y - xs[nf + pr] : r.y;
        if (a <= b) {
            zc l{0.0, 0.0};
            for (int c = 0; c < Na; c++) cfma_conj(l, Tk[a + c * Na], G[b + c * Na]);
            if (a < b) {
                const int ps = 2 * nf + sup_idx(Na, a, b);
                o[ps] = xs ? l.x - xs[ps] : l.x;
            }
            const int pu = 2 * nf + nsu + up_idx(Na, a, b);
            o[pu] = xs ? l.y - xs[pu] : l.y;
            if (a == b) {
                gRd[k * Na + a] = r;
                gLd[k * Na + a] = l;
            }
        }
    }
}

// Current (src/observables.f90:18-52): per energy Re Tr{i GammaL [(fL - 1) G^< - fL G^>]}/2pi
// of G_in, summed over energies (one block)
__global__ void sa_current(int Na, int n, const zc *__restrict__ EL, const zc *__restrict__ EG,
                           const zc *__restrict__ GamL, const double *__restrict__ omega, double V, double mu,
                           double beta, double *__restrict__ out) {
    __shared__ double red[256];
    double acc = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const double fL = sa_fermi(omega[k], V, mu, beta);
        zc tr{0.0, 0.0};
        for (int a = 0; a < Na; a++)
            for (int c = 0; c < Na; c++) {
                const zc g = GamL[a + c * Na];
                const size_t ca = ((size_t)c + (size_t)a * Na) * n + k;
                const zc v = (fL - 1.0) * EL[ca] - fL * EG[ca];
                tr = tr + zc{-g.y, g.x} * v;
            }
        acc += tr.x / (2.0 * PI);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = red[0];
}

// write_spectral's A_ii(w) = -2 Im G^r_ii(w) of G_in, [k*Na + i]
__global__ void sa_spectral(int Na, int n, const zc *__restrict__ Er, double *__restrict__ spec) {
    const int64_t tot = (int64_t)n * Na;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot; t += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t % Na);
        const int64_t k = t / Na;
        spec[t] = -2.0 * Er[((size_t)i + (size_t)i * Na) * n + k].y;
    }
}

int grid_for(int64_t tot, int thr = 256) { return (int)std::max<int64_t>(1, std::min<int64_t>((tot + thr - 1) / thr, 148 * 16)); }

// launch bracketed by the optional per-family events (qsa_profile), counted, error-checked
#define SA_RUN(h, fam, ...)                        \
    do {                                           \
        const int _pi = prof_begin(&(h)->q, fam);  \
        __VA_ARGS__;                               \
        prof_end(&(h)->q, _pi);                    \
        QS_CUDA(&(h)->q, cudaGetLastError());      \
    } while (0)

// G_in from x: element-major sequences and G^<(t=0)
int sa_load_input(qsa_handle *h, const double *d_x) {
    const int Na = h->Na, n = h->n;
    const int64_t tot = (int64_t)n * Na * Na;
    SA_RUN(h, K_OTHER, sa_unpack<<<grid_for(tot), 256, 0, h->q.stream>>>(Na, n, d_x, h->d_E[0], h->d_E[1], h->d_E[2], h->d_E[3]));
    SA_RUN(h, K_OTHER, sa_glt0<<<Na, 256, 0, h->q.stream>>>(Na, n, h->d_E[2], h->delta / (2.0 * PI), h->d_Glt0));
    return 0;
}

// build_self_energies (src/self_energies.f90:40-47) from the loaded G_in
int sa_self_energies(qsa_handle *h) {
    if (h->order < 2) return 0;
    const int Na = h->Na, n = h->n, Nm = h->Nm;
    const double pp = h->delta / (2.0 * PI);
    cudaStream_t st = h->q.stream;
    zc *const *E = h->d_E;
    const dim3 gb((Nm + NP - 1) / NP, Na * Na), gs((n + NP - 1) / NP, Na * Na);
    SA_RUN(h, K_SIG2A, sa_bubbles<true><<<gb, LT, 0, st>>>(Na, n, E[0], E[1], E[2], E[3], pp, h->d_chi[0], h->d_chi[1], h->d_chi[2],
                                        h->d_chi[3]));
    if (h->order == 3) {
        SA_RUN(h, K_SIG2A, sa_bubbles<false><<<gb, LT, 0, st>>>(Na, n, E[0], E[1], E[2], E[3], pp, h->d_phi[0], h->d_phi[1],
                                             h->d_phi[2], h->d_phi[3]));
    }
    // -(i hbar)^2 and -(i hbar)^3
    const zc c2{HB * HB, 0.0}, c3{0.0, HB * HB * HB};
    SA_RUN(h, K_SIG2C, sa_sigma<<<gs, LT, 0, st>>>(Na, n, E[0], E[1], E[2], E[3], h->d_chi[1], h->d_chi[0], h->d_chi[2], nullptr,
                                nullptr, nullptr, h->d_U, pp * c2, h->d_S2R, h->d_S2L));
    if (h->order == 3) {
        const int64_t tot = (int64_t)Nm * Na * Na;
        SA_RUN(h, K_SIG2B, sa_products<<<grid_for(tot), 256, 0, st>>>(Na, Nm, h->d_chi[0], h->d_chi[1], h->d_chi[2], h->d_chi[3],
                                                   h->d_U, h->d_D[0], h->d_D[1], h->d_D[2]));
        SA_RUN(h, K_SIG2B, sa_products<<<grid_for(tot), 256, 0, st>>>(Na, Nm, h->d_phi[0], h->d_phi[1], h->d_phi[2], h->d_phi[3],
                                                   h->d_U, h->d_P[0], h->d_P[1], h->d_P[2]));
        SA_RUN(h, K_SIG2C, sa_sigma<<<gs, LT, 0, st>>>(Na, n, E[0], E[1], E[2], E[3], h->d_D[1], h->d_D[0], h->d_D[2], h->d_P[1],
                                    h->d_P[0], h->d_P[2], h->d_U, pp * c3, h->d_S3R, h->d_S3L));
    }
    return 0;
}

int sa_read_info(qsa_handle *h) {
    int info = INT_MAX;
    QS_CUDA(&h->q, cudaMemcpyAsync(&info, h->d_info, sizeof(int), cudaMemcpyDeviceToHost, h->q.stream));
    QS_CUDA(&h->q, cudaStreamSynchronize(h->q.stream));
    if (info != INT_MAX) {
        h->q.err = "ERROR: ZGETRF failed (singular matrix?) at energy " + std::to_string(info);
        const int v = INT_MAX;
        QS_CUDA(&h->q, cudaMemcpyAsync(h->d_info, &v, sizeof(int), cudaMemcpyHostToDevice, h->q.stream));
        QS_CUDA(&h->q, cudaStreamSynchronize(h->q.stream));
        return info;
    }
    return 0;
}

// One sweep over all energies: Dyson with (interacting) or without Sigma, Keldysh, pack into
// out (minus x when given), the sanity sums. interacting = false: the non-interacting G.
int sa_sweep(qsa_handle *h, double V, bool interacting, double *d_out, const double *d_x) {
    const int Na = h->Na, n = h->n;
    const int64_t tot = (int64_t)n * Na * Na;
    cudaStream_t st = h->q.stream;
    const int ord = interacting ? h->order : 0;
    const bool s2 = interacting && h->order >= 2, s3 = interacting && h->order == 3;
    SA_RUN(h, K_DYSON, sa_dyson_build<<<grid_for(tot), 256, 0, st>>>(Na, n, ord, h->d_H, h->d_GamL, h->d_GamR, h->d_omega,
                                                  s2 ? h->d_S2R : nullptr, s3 ? h->d_S3R : nullptr, h->d_U, h->d_Glt0,
                                                  h->d_W));
    const int pi = prof_begin(&h->q, K_DYSON, false);  // the inversion counts its own launch
    int rc = invert_batched_dev(st, Na, n, h->d_W, h->d_info, h->d_ws, h->ws_slots);
    prof_end(&h->q, pi);
    if (rc) {
        h->q.err = "batched Dyson inversion failed to launch";
        return rc;
    }
    if ((rc = sa_read_info(h))) return rc;
    SA_RUN(h, K_KELDYSH, sa_keldysh_T<<<grid_for(tot), 256, 0, st>>>(Na, n, h->d_W, h->d_GamL, h->d_GamR, s2 ? h->d_S2L : nullptr,
                                                s3 ? h->d_S3L : nullptr, h->d_omega, V, h->mu, h->beta, h->d_T));
    SA_RUN(h, K_KELDYSH, sa_keldysh_pack<<<grid_for(tot), 256, 0, st>>>(Na, n, h->d_W, h->d_T, d_x, d_out, h->d_gRd, h->d_gLd));
    // check_gf_sanity sums
    if ((rc = sum_over_energies(&h->q, h->d_gLd, Na, Na, n, h->d_sums))) return rc;
    if ((rc = sum_over_energies(&h->q, h->d_gRd, Na, Na, n, h->d_sums + Na))) return rc;
    std::vector<zc> hs(2 * Na);
    QS_CUDA(&h->q, cudaMemcpyAsync(hs.data(), h->d_sums, sizeof(zc) * 2 * Na, cudaMemcpyDeviceToHost, st));
    QS_CUDA(&h->q, cudaStreamSynchronize(st));
    std::vector<zc> sl(hs.begin(), hs.begin() + Na);
    std::vector<double> sr(Na);
    for (int i = 0; i < Na; i++) sr[i] = hs[Na + i].y;
    h->last = check_diag_sanity(Na, sl, sr, h->delta, nullptr);
    return 0;
}

// scf_residual (src/scf.f90:102-136)
int sa_residual(qsa_handle *h, double V, const double *d_x, double *d_F, bool &abort) {
    int rc;
    if ((rc = sa_load_input(h, d_x))) return rc;
    if ((rc = sa_self_energies(h))) return rc;
    if ((rc = sa_sweep(h, V, true, d_F, d_x))) return rc;
    abort = h->last.runaway;
    if (abort) QS_CUDA(&h->q, cudaMemsetAsync(d_F, 0, sizeof(double) * h->n_vec, h->q.stream));
    return 0;
}

struct SanchoResidual : BroydenResidual {
    qsa_handle *h = nullptr;
    double V = 0.0;
    const double *last_x = nullptr;
    int operator()(const double *d_x, double *d_F, bool &abort) override {
        last_x = d_x;
        return sa_residual(h, V, d_x, d_F, abort);
    }
};

}  // namespace

extern "C" {

int qsa_create(const qsa_problem *p, qsa_handle **out) {
    if (!p || !out) return -1;
    *out = nullptr;
    if (p->N_sites < 1 || p->N_sites > 512 || p->n_omega < 1 || p->order < 0 || p->order > 3 || !p->H ||
        !p->GammaL || !p->GammaR || !p->U_site || !p->omega || p->nhist < 0 || p->maxscf < 1)
        return -1;
    auto *h = new qsa_handle();
    qs_handle *q = &h->q;
    h->Na = p->N_sites;
    h->n = p->n_omega;
    h->order = p->order;
    h->Nm = 2 * h->n - 1;
    h->mu = p->mu;
    h->beta = p->beta;
    h->delta = p->delta;
    h->alpha_mix = p->alpha_mix;
    h->tolf = p->tolf;
    h->nhist = p->nhist;
    h->maxscf = p->maxscf;
    h->omega.assign(p->omega, p->omega + h->n);
    q->device = p->device;
    const int Na = h->Na, n = h->n;
    const size_t nf = (size_t)Na * Na, zc_ = sizeof(zc), tot = nf * n, tm = nf * h->Nm;
    // src/sancho.f90:106-109: n_vec = (2 n_full + 2 n_strict_upper + Nsites) n_omega = 3 Na^2 n
    h->n_vec = 3 * (int64_t)nf * n;
    q->n_vec = h->n_vec;
    int rc = 0;
    cudaError_t e = cudaSetDevice(p->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete h;
        return -(int)e;
    }
    auto up = [&](void **d, const void *src, size_t bytes) {
        int r = dalloc(q, d, bytes);
        if (r) return r;
        cudaError_t ce = cudaMemcpyAsync(*d, src, bytes, cudaMemcpyHostToDevice, q->stream);
        if (ce != cudaSuccess) {
            q->err = cudaGetErrorString(ce);
            return -(int)ce;
        }
        return 0;
    };
    const int64_t n_vec = h->n_vec;
    q->red_len = broyden_red_len();
    if ((rc = up((void **)&h->d_H, p->H, nf * zc_)) || (rc = up((void **)&h->d_GamL, p->GammaL, nf * zc_)) ||
        (rc = up((void **)&h->d_GamR, p->GammaR, nf * zc_)) || (rc = up((void **)&h->d_U, p->U_site, Na * 8)) ||
        (rc = up((void **)&h->d_omega, p->omega, (size_t)n * 8)) ||
        (rc = dalloc(q, (void **)&q->d_x, n_vec * 8)) || (rc = dalloc(q, (void **)&q->d_F, n_vec * 8)) ||
        (rc = dalloc(q, (void **)&q->d_Fold, n_vec * 8)) || (rc = dalloc(q, (void **)&q->d_xold, n_vec * 8)) ||
        (rc = dalloc(q, (void **)&q->d_red, q->red_len * 8)) ||
        (h->nhist > 0 && ((rc = dalloc(q, &q->d_hdF, broyden_ld(n_vec) * 8 * h->nhist)) ||
                          (rc = dalloc(q, &q->d_hU, broyden_ld(n_vec) * 8 * h->nhist)))) ||
        (rc = dalloc(q, (void **)&h->d_Glt0, Na * zc_)) || (rc = dalloc(q, (void **)&h->d_W, tot * zc_)) ||
        (rc = dalloc(q, (void **)&h->d_T, tot * zc_)) || (rc = dalloc(q, (void **)&h->d_gRd, (size_t)n * Na * zc_)) ||
        (rc = dalloc(q, (void **)&h->d_gLd, (size_t)n * Na * zc_)) ||
        (rc = dalloc(q, (void **)&h->d_spec, (size_t)n * Na * 8)) ||
        (rc = dalloc(q, (void **)&h->d_sums, 2 * (size_t)Na * zc_)) ||
        (rc = dalloc(q, (void **)&h->d_info, sizeof(int) * ((size_t)n + 1)))) {
    }
    for (int k = 0; k < 4 && !rc; k++) rc = dalloc(q, (void **)&h->d_E[k], tot * zc_);
    if (!rc && h->order >= 2) {
        for (int k = 0; k < 4 && !rc; k++) rc = dalloc(q, (void **)&h->d_chi[k], tm * zc_);
        if (!rc) rc = dalloc(q, (void **)&h->d_S2R, tot * zc_);
        if (!rc) rc = dalloc(q, (void **)&h->d_S2L, tot * zc_);
    }
    if (!rc && h->order == 3) {
        for (int k = 0; k < 4 && !rc; k++) rc = dalloc(q, (void **)&h->d_phi[k], tm * zc_);
        for (int k = 0; k < 3 && !rc; k++) rc = dalloc(q, (void **)&h->d_D[k], tm * zc_);
        for (int k = 0; k < 3 && !rc; k++) rc = dalloc(q, (void **)&h->d_P[k], tm * zc_);
        if (!rc) rc = dalloc(q, (void **)&h->d_S3R, tot * zc_);
        if (!rc) rc = dalloc(q, (void **)&h->d_S3L, tot * zc_);
    }
    if (!rc && !dyson_fits_smem(Na)) {
        h->ws_slots = std::min(n, 148 * 2);
        rc = dalloc(q, (void **)&h->d_ws, (size_t)h->ws_slots * nf * zc_);
    }
    if (!rc) {
        const int v = INT_MAX;
        e = cudaMemcpyAsync(h->d_info, &v, sizeof(int), cudaMemcpyHostToDevice, q->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(q->stream);
        if (e != cudaSuccess) rc = -(int)e;
    }
    if (rc) {
        release_all(q);
        cudaStreamDestroy(q->stream);
        delete h;
        return rc;
    }
    *out = h;
    return 0;
}

void qsa_destroy(qsa_handle *h) {
    if (!h) return;
    cudaSetDevice(h->q.device);
    release_all(&h->q);
    cudaStreamDestroy(h->q.stream);
    delete h;
}

const char *qsa_last_error(const qsa_handle *h) { return h ? h->q.err.c_str() : "no handle"; }

// per-family device time as qs_profile: dyson (W build + inversion), keldysh (products +
// pack), sig2_fwdA slot = bubbles, sig2_mid slot = order-3 products, sig2_invC slot =
// self-energy convolutions, broyden, reductions, other (unpack, G^<(t=0), outputs)
int qsa_profile(qsa_handle *h, int enable, double *ms, int64_t *launches, int nfam) {
    return qs_profile(&h->q, enable, ms, launches, nfam);
}
int64_t qsa_vector_length(const qsa_handle *h) { return h ? h->n_vec : -1; }

// solve_scf (src/scf.f90:53-95)
int qsa_solve_scf(qsa_handle *h, double Volt, int fresh_start, qs_scf_result *res) {
    qs_handle *q = &h->q;
    QS_CUDA(q, cudaSetDevice(q->device));
    const auto t0 = std::chrono::steady_clock::now();
    int rc;
    // fresh: the non-interacting G (noninteracting_gr_ga + noninteracting_gl_gg); otherwise
    // the last residual's G_in (continuation)
    if ((fresh_start || !h->have_x) && (rc = sa_sweep(h, Volt, false, q->d_x, nullptr))) return rc;
    SanchoResidual r;
    r.h = h;
    r.V = Volt;
    BroydenOut bo;
    rc = broyden_solve_dev(q, r, q->d_x, q->d_F, q->d_Fold, q->d_xold, q->d_hdF, q->d_hU, h->n_vec, h->alpha_mix,
                           h->nhist, h->maxscf, h->tolf, false, bo);
    if (rc) return rc;
    // keep the last evaluated iterate (its G_in is what the observables read) in d_x
    if (r.last_x && r.last_x != q->d_x) std::swap(q->d_x, q->d_xold);
    h->have_x = true;
    QS_CUDA(q, cudaStreamSynchronize(q->stream));
    const SanityOut &s = h->last;
    bool converged = bo.converged && !bo.aborted;
    if (converged && s.unphysical) converged = false;
    res->converged = converged;
    res->n_iter = bo.n_iter;
    res->fmax = bo.fmax;
    res->aborted = bo.aborted;
    res->runaway = s.runaway;
    res->unphysical = s.unphysical;
    res->i_worst = s.i_worst;
    res->n_worst = s.n_worst;
    res->w_worst = s.w_worst;
    res->n_resets = bo.n_resets;
    res->n_log = 0;
    for (auto &e : bo.log)
        if (res->log && res->n_log < res->log_cap) res->log[res->n_log++] = e;
    res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    res->n_mixed = 0;
    return 0;
}

int qsa_current(qsa_handle *h, double Volt, double *J) {
    qs_handle *q = &h->q;
    QS_CUDA(q, cudaSetDevice(q->device));
    SA_RUN(h, K_OTHER, sa_current<<<1, 256, 0, q->stream>>>(h->Na, h->n, h->d_E[2], h->d_E[3], h->d_GamL, h->d_omega, Volt, h->mu,
                                         h->beta, q->d_red));
    double JL = 0.0;
    QS_CUDA(q, cudaMemcpyAsync(&JL, q->d_red, sizeof(double), cudaMemcpyDeviceToHost, q->stream));
    QS_CUDA(q, cudaStreamSynchronize(q->stream));
    *J = 2.0 * JL * (h->delta / HB);
    return 0;
}

int qsa_get_observables(qsa_handle *h, double *G_less_t0, double *spectral) {
    qs_handle *q = &h->q;
    QS_CUDA(q, cudaSetDevice(q->device));
    if (G_less_t0)
        QS_CUDA(q, cudaMemcpyAsync(G_less_t0, h->d_Glt0, sizeof(zc) * h->Na, cudaMemcpyDeviceToHost, q->stream));
    if (spectral) {
        const int64_t tot = (int64_t)h->n * h->Na;
        SA_RUN(h, K_OTHER, sa_spectral<<<grid_for(tot), 256, 0, q->stream>>>(h->Na, h->n, h->d_E[0], h->d_spec));
        QS_CUDA(q, cudaMemcpyAsync(spectral, h->d_spec, sizeof(double) * tot, cudaMemcpyDeviceToHost, q->stream));
    }
    QS_CUDA(q, cudaStreamSynchronize(q->stream));
    return 0;
}

int qsa_initial_vector(qsa_handle *h, double Volt, double *x) {
    qs_handle *q = &h->q;
    QS_CUDA(q, cudaSetDevice(q->device));
    int rc;
    if ((rc = sa_sweep(h, Volt, false, q->d_x, nullptr))) return rc;
    if ((rc = sa_load_input(h, q->d_x))) return rc;
    h->have_x = true;
    QS_CUDA(q, cudaMemcpyAsync(x, q->d_x, sizeof(double) * h->n_vec, cudaMemcpyDeviceToHost, q->stream));
    QS_CUDA(q, cudaStreamSynchronize(q->stream));
    return 0;
}

int qsa_residual(qsa_handle *h, double Volt, const double *x, double *F, int *abort_flag) {
    qs_handle *q = &h->q;
    QS_CUDA(q, cudaSetDevice(q->device));
    QS_CUDA(q, cudaMemcpyAsync(q->d_x, x, sizeof(double) * h->n_vec, cudaMemcpyHostToDevice, q->stream));
    h->have_x = true;
    bool ab = false;
    int rc = sa_residual(h, Volt, q->d_x, q->d_F, ab);
    if (rc) return rc;
    QS_CUDA(q, cudaMemcpyAsync(F, q->d_F, sizeof(double) * h->n_vec, cudaMemcpyDeviceToHost, q->stream));
    QS_CUDA(q, cudaStreamSynchronize(q->stream));
    if (abort_flag) *abort_flag = ab ? 1 : 0;
    return 0;
}

int qsa_self_energies(qsa_handle *h, const double *x, double *Sig2R, double *Sig2L, double *Sig3R, double *Sig3L) {
    qs_handle *q = &h->q;
    QS_CUDA(q, cudaSetDevice(q->device));
    QS_CUDA(q, cudaMemcpyAsync(q->d_x, x, sizeof(double) * h->n_vec, cudaMemcpyHostToDevice, q->stream));
    h->have_x = true;
    int rc;
    if ((rc = sa_load_input(h, q->d_x))) return rc;
    if ((rc = sa_self_energies(h))) return rc;
    const size_t bytes = sizeof(zc) * (size_t)h->Na * h->Na * h->n;
    auto get = [&](double *dst, const zc *src) -> int {
        if (!dst) return 0;
        if (!src) {
            std::fill(dst, dst + 2 * (size_t)h->Na * h->Na * h->n, 0.0);
            return 0;
        }
        QS_CUDA(q, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, q->stream));
        return 0;
    };
    if ((rc = get(Sig2R, h->d_S2R)) || (rc = get(Sig2L, h->d_S2L)) || (rc = get(Sig3R, h->d_S3R)) ||
        (rc = get(Sig3L, h->d_S3L)))
        return rc;
    QS_CUDA(q, cudaStreamSynchronize(q->stream));
    return 0;
}

}  // extern "C"
