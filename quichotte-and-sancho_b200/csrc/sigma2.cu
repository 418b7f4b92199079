// sigma2.cu -- second-order self-energies Sigma2^r, Sigma2^< for all energies at once
// (sigma2_compute, src/self_energies.f90:135-219), as three FFT kernels over the energy
// axis with the 2x2 spin algebra fused between the forward and the inverse transforms.
//
// The reference zero-pads G_ij(w) from n to Nf >= 2n-1 (good_fft_size), forward-transforms
// every active element of G^r and G^<, forms per site pair (I,J) and frequency l the 2x2
// products of blocks (I,J) at +l and (J,I) at -l, and inverse-transforms the result
// (scaled by c = U_I U_J hbar^2 (delta/2pi)^2 / Nf) back to the first n energies.
//
// Here Nf = N1*N2 and every transform is split in the four-step way (w = N2 m1 + m2,
// l = l1 + N1 l2):
//   kernel A  per element sequence: length-N1 FFTs over m1, twiddle W^{m2 l1}  -> Y[l1][m2]
//   kernel B  per site pair and column pair {l1, N1-l1}: length-N2 FFTs over m2 (the
//             spectrum), the 2x2 algebra (the partner -l of l = l1 + N1 l2 lies in column
//             N1-l1), inverse length-N2 FFTs, twiddle W^{-m2 l1}                   -> V[l1][m2]
//   kernel C  per output 2x2 block: inverse length-N1 FFTs over l1, scale by c, keep the
//             first n energies                                                    -> Sigma[w]
// The spectra never leave shared memory in kernel B. G^< is anti-Hermitian
// (unpack_gf rebuilds G^<_ji = -conj(G^<_ij), common/linear_algebra.f90:222-223), so only
// its upper triangle is transformed: FL_ji(l) = -conj(FL_ij(-l)).
#include <algorithm>
#include <cmath>

#include "fft.cuh"
#include "qs_common.cuh"

namespace qs {

// ---------------------------------------------------------------------------------
// Kernel A: forward length-N1 transforms of the zero-padded element sequences.
// ---------------------------------------------------------------------------------
template <typename T>
__global__ void sig2_fwdA(const double *__restrict__ X, int64_t nblk, int n, const int2 *__restrict__ desc, int nY,
                          FftPlan fp, const cplx<T> *__restrict__ tw, cplx<T> *__restrict__ Y, int SA, int GA) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N1 = fp.N1, N2 = fp.N2, Nf = fp.Nf;
    const int s0 = blockIdx.x * SA, m20 = blockIdx.y * GA;
    const int nseq = SA * GA;
    cplx<T> *buf = (cplx<T> *)smem_raw;
    cplx<T> *tmp = buf + (size_t)nseq * N1;
    const int total = nseq * N1;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int sl = t % SA, r = t / SA;
        int gl = r % GA, m1 = r / GA;
        int s = s0 + sl, m2 = m20 + gl;
        int64_t w = (int64_t)N2 * m1 + m2;
        cplx<T> v{0, 0};
        if (s < nY && m2 < N2 && w < n) {
            int2 d = desc[s];
            const double *blk = X + w * nblk;
            v.x = d.x >= 0 ? (T)blk[d.x] : (T)0;
            v.y = (T)blk[d.y];
        }
        buf[(size_t)(sl * GA + gl) * N1 + m1] = v;
    }
    __syncthreads();
    cplx<T> *res = smem_fft(buf, tmp, nseq, fp.p1, -1, tw, Nf);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int gl = t % GA, r = t / GA;
        int l1 = r % N1, sl = r / N1;
        int s = s0 + sl, m2 = m20 + gl;
        if (s < nY && m2 < N2) {
            cplx<T> v = res[(size_t)(sl * GA + gl) * N1 + l1] * tw[m2 * l1];
            Y[(size_t)s * Nf + (size_t)l1 * N2 + m2] = v;
        }
    }
}

// 2x2 complex block helpers
template <typename T> struct B2 { cplx<T> a[2][2]; };
template <typename T> __device__ __forceinline__ B2<T> mm2(const B2<T> &X, const B2<T> &Y) {
    B2<T> Z;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) Z.a[i][j] = X.a[i][0] * Y.a[0][j] + X.a[i][1] * Y.a[1][j];
    return Z;
}
template <typename T> __device__ __forceinline__ B2<T> dag2(const B2<T> &X) {
    B2<T> Z;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) Z.a[i][j] = conj(X.a[j][i]);
    return Z;
}
template <typename T> __device__ __forceinline__ B2<T> neg2(const B2<T> &X) {
    B2<T> Z;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) Z.a[i][j] = -X.a[i][j];
    return Z;
}
// adj2 (src/self_energies.f90:222-228): Tr(M) 1 - M
template <typename T> __device__ __forceinline__ B2<T> adj2(const B2<T> &M) {
    B2<T> A;
    A.a[0][0] = M.a[1][1];
    A.a[0][1] = -M.a[0][1];
    A.a[1][0] = -M.a[1][0];
    A.a[1][1] = M.a[0][0];
    return A;
}

// The per-frequency algebra of src/self_energies.f90:175-199 for one block (i,j):
// inputs r_ij, L_ij at +l and r_ji, L_ji at -l; outputs sR, sL.
template <typename T>
__device__ __forceinline__ void pair_algebra(const B2<T> &r_ij, const B2<T> &L_ij, const B2<T> &r_ji, const B2<T> &L_ji,
                                             B2<T> &sR, B2<T> &sL) {
    B2<T> a_ij = dag2(r_ji), a_ji = dag2(r_ij), G_ij, G_ji;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) {
            G_ij.a[i][j] = L_ij.a[i][j] + r_ij.a[i][j] - a_ij.a[i][j];
            G_ji.a[i][j] = L_ji.a[i][j] + r_ji.a[i][j] - a_ji.a[i][j];
        }
    B2<T> chi1 = mm2(L_ji, G_ij);
    B2<T> t1 = mm2(L_ji, r_ij), t2 = mm2(a_ji, L_ij), chi2;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) chi2.a[i][j] = t1.a[i][j] + t2.a[i][j];
    B2<T> u1 = mm2(r_ij, adj2(chi1)), u2 = mm2(L_ij, adj2(chi2));
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) sR.a[i][j] = u1.a[i][j] + u2.a[i][j];
    B2<T> chiL = mm2(G_ji, L_ij);
    sL = mm2(L_ij, adj2(chiL));
}

// ---------------------------------------------------------------------------------
// Kernel B: spectra, 2x2 algebra, inverse length-N2 transforms, for one site pair
// (I <= J) and the column pair {c, N1-c}.
// ---------------------------------------------------------------------------------
template <typename T>
__global__ void sig2_mid(const cplx<T> *__restrict__ Y, cplx<T> *__restrict__ V, const int2 *__restrict__ pairs, int nA,
                         FftPlan fp, const cplx<T> *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N1 = fp.N1, N2 = fp.N2, Nf = fp.Nf;
    const int2 pr = pairs[blockIdx.x];
    const int I = pr.x, J = pr.y, io = 2 * I, jo = 2 * J;
    const int c = blockIdx.y;
    const int cp = (N1 - c) % N1;
    const int ncols = (cp == c) ? 1 : 2;
    const int cols[2] = {c, cp};
    const bool diag = (I == J);
    const int nfull = nA * nA;
    auto id_r = [&](int i, int j) { return i + j * nA; };
    auto id_l = [&](int i, int j) { return nfull + (j * (j + 1)) / 2 + i; };  // i <= j

    cplx<T> *Sa = (cplx<T> *)smem_raw;            // 24 N2
    cplx<T> *Sb = Sa + (size_t)24 * N2;           // 24 N2
    cplx<T> *O = Sb + (size_t)24 * N2;            // 32 N2: [stage R/L][blk][col][elem][N2]

    // 1. load the 12 input sequences of each column
    const int nin = ncols * 12 * N2;
    for (int t = threadIdx.x; t < nin; t += blockDim.x) {
        int m2 = t % N2, r = t / N2;
        int k = r % 12, ci = r / 12;
        int a = k & 1, b = (k >> 1) & 1;
        int sid = -1;
        if (k < 4) sid = id_r(io + a, jo + b);
        else if (k < 8) sid = id_r(jo + a, io + b);
        else if (!diag) sid = id_l(io + a, jo + b);
        else if (k == 8) sid = id_l(io, io);
        else if (k == 9) sid = id_l(io, io + 1);
        else if (k == 10) sid = id_l(io + 1, io + 1);
        cplx<T> v{0, 0};
        if (sid >= 0) v = Y[(size_t)sid * Nf + (size_t)cols[ci] * N2 + m2];
        Sa[(size_t)(ci * 12 + k) * N2 + m2] = v;
    }
    __syncthreads();
    cplx<T> *S = smem_fft(Sa, Sb, ncols * 12, fp.p2, -1, tw, Nf);
    cplx<T> *Fr = (S == Sa) ? Sb : Sa;

    auto sv = [&](int ci, int k, int l2) { return S[(size_t)(ci * 12 + k) * N2 + l2]; };
    // L block of (I,J) at (ci, l2); for I == J the (1,0) element comes from the partner
    auto LIJ = [&](int ci, int l2) {
        B2<T> L;
        if (!diag) {
            L.a[0][0] = sv(ci, 8, l2);
            L.a[1][0] = sv(ci, 9, l2);
            L.a[0][1] = sv(ci, 10, l2);
            L.a[1][1] = sv(ci, 11, l2);
        } else {
            int col = cols[ci];
            int pci = (ncols == 1) ? 0 : 1 - ci;
            int pl2 = (col == 0) ? (N2 - l2) % N2 : N2 - 1 - l2;
            L.a[0][0] = sv(ci, 8, l2);
            L.a[0][1] = sv(ci, 9, l2);
            L.a[1][1] = sv(ci, 10, l2);
            L.a[1][0] = -conj(sv(pci, 9, pl2));
        }
        return L;
    };
    auto RB = [&](int ci, int base, int l2) {
        B2<T> R;
        R.a[0][0] = sv(ci, base + 0, l2);
        R.a[1][0] = sv(ci, base + 1, l2);
        R.a[0][1] = sv(ci, base + 2, l2);
        R.a[1][1] = sv(ci, base + 3, l2);
        return R;
    };
    const int nblkout = diag ? 1 : 2;
    // 2. 2x2 algebra at every position of the loaded columns
    for (int t = threadIdx.x; t < ncols * N2; t += blockDim.x) {
        int l2 = t % N2, ci = t / N2;
        int col = cols[ci];
        int pci = (ncols == 1) ? 0 : 1 - ci;
        int pl2 = (col == 0) ? (N2 - l2) % N2 : N2 - 1 - l2;
        B2<T> sR, sL;
        // block (I,J) at l
        {
            B2<T> r_ij = RB(ci, 0, l2), L_ij = LIJ(ci, l2), r_ji = RB(pci, 4, pl2);
            B2<T> L_ji = diag ? LIJ(pci, pl2) : neg2(dag2(L_ij));
            pair_algebra(r_ij, L_ij, r_ji, L_ji, sR, sL);
#pragma unroll
            for (int e = 0; e < 4; e++) {
                O[((size_t)((0 * 2 + 0) * 2 + ci) * 4 + e) * N2 + l2] = sR.a[e & 1][e >> 1];
                O[((size_t)((1 * 2 + 0) * 2 + ci) * 4 + e) * N2 + l2] = sL.a[e & 1][e >> 1];
            }
        }
        if (!diag) {  // block (J,I) at l
            B2<T> Lp = LIJ(pci, pl2);
            B2<T> r_ij = RB(ci, 4, l2), L_ij = neg2(dag2(Lp)), r_ji = RB(pci, 0, pl2);
            pair_algebra(r_ij, L_ij, r_ji, Lp, sR, sL);
#pragma unroll
            for (int e = 0; e < 4; e++) {
                O[((size_t)((0 * 2 + 1) * 2 + ci) * 4 + e) * N2 + l2] = sR.a[e & 1][e >> 1];
                O[((size_t)((1 * 2 + 1) * 2 + ci) * 4 + e) * N2 + l2] = sL.a[e & 1][e >> 1];
            }
        }
    }
    __syncthreads();
    // 3. inverse length-N2 transforms, twiddle, store; stage 0 = Sigma^R, 1 = Sigma^<
    for (int stage = 0; stage < 2; stage++) {
        cplx<T> *Os = O + (size_t)stage * 16 * N2;
        // sequences of this stage: [blk][col][elem] -> only the used (blk, col) ones exist;
        // transform all 16 (unused ones hold garbage and are not stored)
        cplx<T> *res = smem_fft(Os, Fr, 16, fp.p2, +1, tw, Nf);
        const int nout = nblkout * ncols * 4 * N2;
        for (int t = threadIdx.x; t < nout; t += blockDim.x) {
            int m2 = t % N2, r = t / N2;
            int e = r % 4, r2 = r / 4;
            int ci = r2 % ncols, b = r2 / ncols;
            int a = e & 1, bb = e >> 1;
            int row = (b == 0 ? io : jo) + a, colm = (b == 0 ? jo : io) + bb;
            int col = cols[ci];
            cplx<T> v = res[((size_t)(b * 2 + ci) * 4 + e) * N2 + m2] * twid(tw, m2 * col, +1);
            size_t sid = (size_t)stage * nfull + id_r(row, colm);
            V[sid * Nf + (size_t)col * N2 + m2] = v;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------
// Kernel C: inverse length-N1 transforms, scaling, first n energies -> Sigma (w-major).
// ---------------------------------------------------------------------------------
template <typename T>
__global__ void sig2_invC(const cplx<T> *__restrict__ V, zc *__restrict__ SigR, zc *__restrict__ SigL, int nA, int nAs,
                          int n, const double *__restrict__ Upair, FftPlan fp, const cplx<T> *__restrict__ tw, int GC) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N1 = fp.N1, N2 = fp.N2, Nf = fp.Nf;
    const int I = blockIdx.x % nAs, J = blockIdx.x / nAs;
    const int io = 2 * I, jo = 2 * J;
    const int m20 = blockIdx.y * GC;
    const int nfull = nA * nA;
    const double c = Upair[I + J * nAs];  // U_I U_J hbar^2 (delta/2pi)^2 / Nf, 0 if no interaction
    const int nseq = 8 * GC;
    if (c == 0.0) {
        // src/self_energies.f90:167-171: zero blocks
        const int tot = 8 * GC * N1;
        for (int t = threadIdx.x; t < tot; t += blockDim.x) {
            int a = t & 1, bb = (t >> 1) & 1, st = (t >> 2) & 1, r = t >> 3;
            int gl = r % GC, m1 = r / GC;
            int m2 = m20 + gl;
            int64_t w = (int64_t)N2 * m1 + m2;
            if (m2 < N2 && w < n) {
                zc *S = st ? SigL : SigR;
                S[w * nfull + (io + a) + (size_t)(jo + bb) * nA] = zc{0.0, 0.0};
            }
        }
        return;
    }
    cplx<T> *buf = (cplx<T> *)smem_raw;
    cplx<T> *tmp = buf + (size_t)nseq * N1;
    const int total = nseq * N1;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int gl = t % GC, r = t / GC;
        int sl = r % 8, l1 = r / 8;
        int m2 = m20 + gl;
        int e = sl & 3, st = sl >> 2;
        int a = e & 1, bb = e >> 1;
        cplx<T> v{0, 0};
        if (m2 < N2) {
            size_t sid = (size_t)st * nfull + (io + a) + (size_t)(jo + bb) * nA;
            v = V[sid * Nf + (size_t)l1 * N2 + m2];
        }
        buf[(size_t)(sl * GC + gl) * N1 + l1] = v;
    }
    __syncthreads();
    cplx<T> *res = smem_fft(buf, tmp, nseq, fp.p1, +1, tw, Nf);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int a = t & 1, bb = (t >> 1) & 1, st = (t >> 2) & 1, r = t >> 3;
        int gl = r % GC, m1 = r / GC;
        int m2 = m20 + gl;
        int64_t w = (int64_t)N2 * m1 + m2;
        if (m2 < N2 && w < n) {
            int sl = st * 4 + a + 2 * bb;
            cplx<T> v = res[(size_t)(sl * GC + gl) * N1 + m1];
            zc *S = st ? SigL : SigR;
            S[w * nfull + (io + a) + (size_t)(jo + bb) * nA] = zc{c * (double)v.x, c * (double)v.y};
        }
    }
}

// ---------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------
static void factor_len(int L, FftLen &P) {
    P.L = L;
    P.nrad = 0;
    int m = L;
    for (int r : {8, 4, 2, 3, 5, 7})
        while (m % r == 0) {
            P.rad[P.nrad++] = r;
            m /= r;
        }
}

// good_fft_size (src/self_energies.f90:75-89)
static int good_fft_size(int nmin) {
    for (int n = nmin;; n++) {
        int m = n;
        for (int r : {2, 3, 5, 7})
            while (m % r == 0) m /= r;
        if (m == 1) return n;
    }
}

int sigma2_setup(qs_handle *h) {
    const int n = h->n, nA = h->nA;
    FftPlan &fp = h->fft;
    fp.Nf = good_fft_size(2 * n - 1);
    // N2: the divisor of Nf nearest to sqrt(Nf), at most 128 (shared memory of kernel B)
    int best = 1;
    double sq = std::sqrt((double)fp.Nf);
    for (int d = 1; d <= 128; d++)
        if (fp.Nf % d == 0 && std::fabs(d - sq) < std::fabs(best - sq)) best = d;
    fp.N2 = best;
    fp.N1 = fp.Nf / best;
    factor_len(fp.N1, fp.p1);
    factor_len(fp.N2, fp.p2);
    // twiddles W_Nf^k in extended precision
    std::vector<zc> tw(fp.Nf);
    for (int k = 0; k < fp.Nf; k++) {
        long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)fp.Nf;
        tw[k] = zc{(double)cosl(a), (double)sinl(a)};
    }
    int rc;
    if ((rc = dalloc(h, (void **)&h->d_tw, sizeof(zc) * fp.Nf))) return rc;
    QS_CUDA(h, cudaMemcpyAsync(h->d_tw, tw.data(), sizeof(zc) * fp.Nf, cudaMemcpyHostToDevice, h->stream));
    // Y sequences: every G^r element, the upper triangle of G^<
    const int nfull = nA * nA;
    std::vector<int2> desc;
    desc.reserve(nfull + nA * (nA + 1) / 2);
    for (int j = 0; j < nA; j++)
        for (int i = 0; i < nA; i++) desc.push_back(int2{2 * (i + j * nA), 2 * (i + j * nA) + 1});
    for (int j = 0; j < nA; j++)
        for (int i = 0; i <= j; i++) {
            if (i < j) {
                int o = 2 * nfull + 2 * (j * (j - 1) / 2 + i);
                desc.push_back(int2{o, o + 1});
            } else {
                desc.push_back(int2{-1, 2 * nfull + nA * (nA - 1) + i});
            }
        }
    h->nY = desc.size();
    h->nV = (size_t)2 * nfull;
    if ((rc = dalloc(h, (void **)&h->d_ydesc, sizeof(int2) * desc.size()))) return rc;
    QS_CUDA(h, cudaMemcpyAsync(h->d_ydesc, desc.data(), sizeof(int2) * desc.size(), cudaMemcpyHostToDevice, h->stream));
    if ((rc = dalloc(h, (void **)&h->d_Y, sizeof(zc) * h->nY * fp.Nf))) return rc;
    if ((rc = dalloc(h, (void **)&h->d_V, sizeof(zc) * h->nV * fp.Nf))) return rc;
    if ((rc = dalloc(h, (void **)&h->d_SigR, sizeof(zc) * (size_t)nfull * n))) return rc;
    if ((rc = dalloc(h, (void **)&h->d_SigL, sizeof(zc) * (size_t)nfull * n))) return rc;
    // pair tables and scale factors c = U_I U_J hbar^2 (delta/2pi)^2 / Nf
    const double pp = h->delta / (2.0 * PI);
    std::vector<double> Upair((size_t)h->nAs * h->nAs);
    std::vector<int2> pairs;
    for (int J = 0; J < h->nAs; J++)
        for (int I = 0; I < h->nAs; I++) {
            double UI = h->U_site[h->act[2 * I]], UJ = h->U_site[h->act[2 * J]];
            double up = UI * UJ;
            Upair[I + (size_t)J * h->nAs] = up == 0.0 ? 0.0 : up * 1.0 * 1.0 * pp * pp / (double)fp.Nf;
            if (I <= J && up != 0.0) pairs.push_back(int2{I, J});
        }
    double *dU;
    int2 *dP;
    if ((rc = dalloc(h, (void **)&dU, sizeof(double) * Upair.size()))) return rc;
    QS_CUDA(h, cudaMemcpyAsync(dU, Upair.data(), sizeof(double) * Upair.size(), cudaMemcpyHostToDevice, h->stream));
    if ((rc = dalloc(h, (void **)&dP, sizeof(int2) * std::max<size_t>(pairs.size(), 1)))) return rc;
    if (!pairs.empty())
        QS_CUDA(h, cudaMemcpyAsync(dP, pairs.data(), sizeof(int2) * pairs.size(), cudaMemcpyHostToDevice, h->stream));
    h->sig2_Upair = dU;
    h->sig2_pairs = dP;
    h->sig2_npairs = (int)pairs.size();
    // tile sizes
    int GA = std::min(fp.N2, 8);
    int SA = std::max(1, std::min(16, 4096 / (fp.N1 * GA)));
    while (SA * GA * fp.N1 > 4096 && GA > 1) GA /= 2;
    h->sig2_SA = SA;
    h->sig2_GA = GA;
    int GC = std::max(1, std::min(fp.N2, 512 / fp.N1));
    h->sig2_GC = GC;
    size_t smA = sizeof(zc) * 2 * (size_t)SA * GA * fp.N1;
    size_t smB = sizeof(zc) * 80 * (size_t)fp.N2;
    size_t smC = sizeof(zc) * 2 * (size_t)8 * GC * fp.N1;
    if (smA > SMEM_MAX || smB > SMEM_MAX || smC > SMEM_MAX) {
        h->err = "sigma2: FFT tiles exceed shared memory";
        return -1;
    }
    QS_CUDA(h, cudaFuncSetAttribute(sig2_fwdA<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smA));
    QS_CUDA(h, cudaFuncSetAttribute(sig2_mid<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smB));
    QS_CUDA(h, cudaFuncSetAttribute(sig2_invC<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smC));
    h->sig2_smem[0] = smA;
    h->sig2_smem[1] = smB;
    h->sig2_smem[2] = smC;
    // every buffer is zeroed on h->stream by dalloc: the tables are copied on the same
    // stream (after the zeroing) and the host staging vectors must outlive the copies
    QS_CUDA(h, cudaStreamSynchronize(h->stream));
    return 0;
}

int sigma2_compute(qs_handle *h, const double *d_x) {
    const FftPlan &fp = h->fft;
    const int nA = h->nA;
    dim3 gA((unsigned)((h->nY + h->sig2_SA - 1) / h->sig2_SA), (unsigned)((fp.N2 + h->sig2_GA - 1) / h->sig2_GA));
    int pa = prof_begin(h, K_SIG2A);
    sig2_fwdA<double><<<gA, 256, h->sig2_smem[0], h->stream>>>(d_x, h->nblk, h->n, h->d_ydesc, (int)h->nY, fp, h->d_tw,
                                                             h->d_Y, h->sig2_SA, h->sig2_GA);
    prof_end(h, pa);
    QS_CUDA(h, cudaGetLastError());
    if (h->sig2_npairs > 0) {
        dim3 gB((unsigned)h->sig2_npairs, (unsigned)(fp.N1 / 2 + 1));
        int pb = prof_begin(h, K_SIG2B);
        sig2_mid<double><<<gB, 256, h->sig2_smem[1], h->stream>>>(h->d_Y, h->d_V, h->sig2_pairs, nA, fp, h->d_tw);
        prof_end(h, pb);
        QS_CUDA(h, cudaGetLastError());
    }
    dim3 gC((unsigned)(h->nAs * h->nAs), (unsigned)((fp.N2 + h->sig2_GC - 1) / h->sig2_GC));
    int pc = prof_begin(h, K_SIG2C);
    sig2_invC<double><<<gC, 256, h->sig2_smem[2], h->stream>>>(h->d_V, h->d_SigR, h->d_SigL, nA, h->nAs, h->n,
                                                             h->sig2_Upair, fp, h->d_tw, h->sig2_GC);
    prof_end(h, pc);
    QS_CUDA(h, cudaGetLastError());
    return 0;
}

}  // namespace qs
