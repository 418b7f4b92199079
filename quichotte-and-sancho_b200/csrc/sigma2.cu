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
// Block tile: SA adjacent sequences x GA adjacent m2 (SA*16 B contiguous per energy block
// read, GA*16 B contiguous per Y row written); one warp per sequence.
// ---------------------------------------------------------------------------------
// N1C > 0: compile-time N1 (power of two) with 4 x 4 tiles, so the index arithmetic of the
// load and store loops reduces to shifts and masks; N1C = 0: any N1 and tile.
template <typename T, int N1C>
__global__ void __launch_bounds__(256, 2) sig2_fwdA(const double *__restrict__ X, int64_t nblk, int n,
                                                 const int2 *__restrict__ desc, int nY, FftPlan fp,
                                                 const zc *__restrict__ tw, cplx<T> *__restrict__ Y, int SA_rt,
                                                 int GA_rt) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N1 = N1C ? N1C : fp.N1, N2 = fp.N2, Nf = fp.Nf, PL = padded_len(N1);
    const int SA = N1C ? 4 : SA_rt, GA = N1C ? 4 : GA_rt;
    const int s0 = blockIdx.x * SA, m20 = blockIdx.y * GA;
    const int nseq = SA * GA;
    cplx<T> *buf = (cplx<T> *)smem_raw;
    cplx<T> *scr = buf + (size_t)nseq * PL + (size_t)(threadIdx.x >> 5) * PL;  // this warp's scratch
    cplx<T> *twL = buf + (size_t)(nseq + (blockDim.x >> 5)) * PL;               // the length-N1 table
    fft_table_fill(twL, N1, tw, N2);
    // only m1 < ceil((n - m2)/N2) can be non-zero (zero padding beyond n energies)
    const int m1max = (n + N2 - 1) / N2;
    for (int t = threadIdx.x; t < nseq * N1; t += blockDim.x) {
        int sl = t % SA, r = t / SA;
        int gl = r % GA, m1 = r / GA;
        int s = s0 + sl, m2 = m20 + gl;
        int64_t w = (int64_t)N2 * m1 + m2;
        cplx<T> v{0, 0};
        if (m1 < m1max && s < nY && m2 < N2 && w < n) {
            int2 d = desc[s];
            const double *blk = X + w * nblk;
            v.x = d.x >= 0 ? (T)blk[d.x] : (T)0;
            v.y = (T)blk[d.y];
        }
        buf[(sl * GA + gl) * PL + pidx(m1)] = v;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    {
        const int G = fft_group(N1);
        for (int q = warp * G; q < nseq; q += nw * G) warp_fft_group(buf + q * PL, PL, min(G, nseq - q), scr, fp.p1, -1, twL);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nseq * N1; t += blockDim.x) {
        int gl = t % GA, r = t / GA;
        int l1 = r % N1, sl = r / N1;
        int s = s0 + sl, m2 = m20 + gl;
        if (s < nY && m2 < N2) {
            cplx<T> v = buf[(sl * GA + gl) * PL + pidx(l1)] * cvt<T>(tw[m2 * l1]);
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

// asynchronous 16-byte (8-byte for float) copy global -> shared; zero-fill when !valid
template <typename T> __device__ __forceinline__ void cp_async_elem(cplx<T> *dst, const cplx<T> *src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(cplx<T>) == 16) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 16 : 0) : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// ---------------------------------------------------------------------------------
// Kernel B: spectra, 2x2 algebra, inverse length-N2 transforms, for one site pair
// (I <= J) and the column pair {c, N1-c} per work item. Persistent blocks walk the items;
// the 24 input sequences of the next item are copied asynchronously into the second input
// buffer while the current item is transformed. Shared memory: 2 x 24 input and 32 output
// sequences (padded), one scratch sequence per warp and the twiddle tables; one warp per
// transform (or per group of transforms, for the power-of-two lengths).
// ---------------------------------------------------------------------------------
template <typename T, int N2C>
__device__ __forceinline__ void mid_load(const cplx<T> *__restrict__ Y, cplx<T> *S, int item, int ncp,
                                         const int2 *__restrict__ pairs, int nA, const FftPlan &fp, int PL) {
    const int N1 = fp.N1, N2 = N2C ? N2C : fp.N2, Nf = fp.Nf;
    const int2 pr = pairs[item / ncp];
    const int io = 2 * pr.x, jo = 2 * pr.y;
    const bool diag = (pr.x == pr.y);
    const int c = item % ncp, cp = (N1 - c) % N1;
    const int ncols = (cp == c) ? 1 : 2;
    const int nfull = nA * nA;
    // the 12 input sequences of each column: R_IJ (k 0-3), R_JI (4-7), L (8-11)
    for (int t = threadIdx.x; t < ncols * 12 * N2; t += blockDim.x) {
        int m2 = t % N2, r = t / N2;
        int k = r % 12, ci = r / 12;
        int a = k & 1, b = (k >> 1) & 1;
        int sid = -1;
        if (k < 4) sid = io + a + (jo + b) * nA;
        else if (k < 8) sid = jo + a + (io + b) * nA;
        else if (!diag) sid = nfull + ((jo + b) * (jo + b + 1)) / 2 + io + a;  // upper (io+a, jo+b)
        else if (k == 8) sid = nfull + (io * (io + 1)) / 2 + io;                   // (io, io)
        else if (k == 9) sid = nfull + ((io + 1) * (io + 2)) / 2 + io;             // (io, io+1)
        else if (k == 10) sid = nfull + ((io + 1) * (io + 2)) / 2 + io + 1;        // (io+1, io+1)
        const cplx<T> *src = sid >= 0 ? Y + (size_t)sid * Nf + (size_t)(ci ? cp : c) * N2 + m2 : Y;
        cp_async_elem(S + (ci * 12 + k) * PL + pidx(m2), src, sid >= 0);
    }
}

// N2C > 0: compile-time N2 (power of two); N2C = 0: any N2
template <typename T, int N2C>
__global__ void __launch_bounds__(512) sig2_mid(const cplx<T> *__restrict__ Y, cplx<T> *__restrict__ V,
                                                const int2 *__restrict__ pairs, int nA, FftPlan fp,
                                                const zc *__restrict__ tw, int nitems) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N1 = fp.N1, N2 = N2C ? N2C : fp.N2, Nf = fp.Nf, PL = padded_len(N2);
    const int ncp = N1 / 2 + 1;
    const int nfull = nA * nA;
    cplx<T> *S0 = (cplx<T> *)smem_raw;  // 2 x 24 sequences: [ci*12 + k]
    cplx<T> *O = S0 + 48 * PL;          // 32 sequences: [((stage*2 + b)*2 + ci)*4 + e]
    cplx<T> *scr = O + 32 * PL + (threadIdx.x >> 5) * PL;  // this warp's scratch
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    cplx<T> *twc = O + (32 + nw) * PL;  // W_Nf^{m2 col} of the item's two columns
    cplx<T> *twL = twc + 2 * N2;        // the length-N2 table
    fft_table_fill(twL, N2, tw, N1);
    const int G = fft_group(N2);

    if (blockIdx.x < nitems) mid_load<T, N2C>(Y, S0, blockIdx.x, ncp, pairs, nA, fp, PL);
    cp_async_commit();
    int cur = 0;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int nxt = item + gridDim.x;
        if (nxt < nitems) mid_load<T, N2C>(Y, S0 + (cur ^ 1) * 24 * PL, nxt, ncp, pairs, nA, fp, PL);
        cp_async_commit();
        cp_async_wait1();  // this thread's copies of the current item have landed
        __syncthreads();
        cplx<T> *S = S0 + cur * 24 * PL;
        const int2 pr = pairs[item / ncp];
        const int I = pr.x, J = pr.y, io = 2 * I, jo = 2 * J;
        const int c = item % ncp;
        const int cp = (N1 - c) % N1;
        const int ncols = (cp == c) ? 1 : 2;
        const bool diag = (I == J);
        const int nblko = diag ? 1 : 2;
        for (int t = threadIdx.x; t < 2 * N2; t += blockDim.x)  // used after two barriers
            twc[t] = cvt<T>(tw[(size_t)(t % N2) * ((t < N2) ? c : cp)]);

        for (int q = warp * G; q < ncols * 12; q += nw * G)
            warp_fft_group(S + q * PL, PL, min(G, ncols * 12 - q), scr, fp.p2, -1, twL);
        __syncthreads();

        auto sv = [&](int ci, int k, int l2) { return S[(ci * 12 + k) * PL + pidx(l2)]; };
        auto partner = [&](int ci, int l2, int &pci, int &pl2) {
            const int col = ci ? cp : c;
            pci = (ncols == 1) ? 0 : 1 - ci;
            pl2 = (col == 0) ? (N2 - l2) % N2 : N2 - 1 - l2;
        };
        auto LIJ = [&](int ci, int l2) {
            B2<T> L;
            if (!diag) {
                L.a[0][0] = sv(ci, 8, l2);
                L.a[1][0] = sv(ci, 9, l2);
                L.a[0][1] = sv(ci, 10, l2);
                L.a[1][1] = sv(ci, 11, l2);
            } else {
                int pci, pl2;
                partner(ci, l2, pci, pl2);
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
        auto put = [&](int b, int ci, int l2, const B2<T> &sR, const B2<T> &sL) {
#pragma unroll
            for (int e = 0; e < 4; e++) {
                O[(((0 * 2 + b) * 2 + ci) * 4 + e) * PL + pidx(l2)] = sR.a[e & 1][e >> 1];
                O[(((1 * 2 + b) * 2 + ci) * 4 + e) * PL + pidx(l2)] = sL.a[e & 1][e >> 1];
            }
        };
        // 2x2 algebra at every position of the loaded columns (block (I,J), then (J,I));
        // ncols and nblko are 1 or 2
        for (int t = threadIdx.x; t < nblko * ncols * N2; t += blockDim.x) {
            int l2 = t % N2, r = t / N2;
            int ci = (ncols == 2) ? (r & 1) : 0, b = (ncols == 2) ? (r >> 1) : r;
            int pci, pl2;
            partner(ci, l2, pci, pl2);
            B2<T> sR, sL;
            if (b == 0) {
                B2<T> L_ij = LIJ(ci, l2);
                pair_algebra(RB(ci, 0, l2), L_ij, RB(pci, 4, pl2), diag ? LIJ(pci, pl2) : neg2(dag2(L_ij)), sR, sL);
            } else {
                B2<T> Lp = LIJ(pci, pl2);
                pair_algebra(RB(ci, 4, l2), neg2(dag2(Lp)), RB(pci, 0, pl2), Lp, sR, sL);
            }
            put(b, ci, l2, sR, sL);
        }
        __syncthreads();
        // inverse length-N2 transforms of the used output sequences; groups of G <= 4
        // sequences share (stage, b, ci) and are adjacent in O (e, e+1, ..)
        const int nout = 2 * nblko * ncols * 4;  // [stage][b][ci][e] restricted to used b, ci
        for (int q = warp * G; q < nout; q += nw * G) {
            int e = q % 4, r = q / 4;
            int ci = (ncols == 2) ? (r & 1) : 0, r2 = (ncols == 2) ? (r >> 1) : r;
            int b = (nblko == 2) ? (r2 & 1) : 0, stage = (nblko == 2) ? (r2 >> 1) : r2;
            warp_fft_group(O + (((stage * 2 + b) * 2 + ci) * 4 + e) * PL, PL, G, scr, fp.p2, +1, twL);
        }
        __syncthreads();
        // twiddle W_Nf^{-m2 col}, store
        for (int t = threadIdx.x; t < nout * N2; t += blockDim.x) {
            int m2 = t % N2, q = t / N2;
            int e = q % 4, r = q / 4;
            int ci = (ncols == 2) ? (r & 1) : 0, r2 = (ncols == 2) ? (r >> 1) : r;
            int b = (nblko == 2) ? (r2 & 1) : 0, stage = (nblko == 2) ? (r2 >> 1) : r2;
            int a = e & 1, bb = e >> 1;
            int row = (b == 0 ? io : jo) + a, colm = (b == 0 ? jo : io) + bb;
            int col = ci ? cp : c;
            cplx<T> v = O[(((stage * 2 + b) * 2 + ci) * 4 + e) * PL + pidx(m2)] * conj(twc[ci * N2 + m2]);
            size_t sid = (size_t)stage * nfull + row + (size_t)colm * nA;
            V[sid * Nf + (size_t)col * N2 + m2] = v;
        }
        __syncthreads();  // S[cur], O and twc are rewritten by the next items
        cur ^= 1;
    }
}

// ---------------------------------------------------------------------------------
// Kernel C: inverse length-N1 transforms, scaling, first n energies -> Sigma (w-major).
// Block = one column jo+bb of the output 2x2 block (I,J): the 4 sequences Sigma^R and
// Sigma^< of rows io, io+1 (two 32 B stores per energy) x GC adjacent m2.
// ---------------------------------------------------------------------------------
// N1C > 0: compile-time N1 (power of two) with GC = 4; N1C = 0: any N1 and GC
template <typename T, int N1C>
__global__ void __launch_bounds__(256, 2) sig2_invC(const cplx<T> *__restrict__ V, zc *__restrict__ SigR,
                                                 zc *__restrict__ SigL, int nA, int nAs, int n,
                                                 const double *__restrict__ Upair, FftPlan fp,
                                                 const zc *__restrict__ tw, int GC_rt) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N1 = N1C ? N1C : fp.N1, N2 = fp.N2, Nf = fp.Nf, PL = padded_len(N1);
    const int GC = N1C ? 4 : GC_rt;
    const int bb = blockIdx.x & 1, pairid = blockIdx.x >> 1;
    const int I = pairid % nAs, J = pairid / nAs;
    const int io = 2 * I, jo = 2 * J;
    const int m20 = blockIdx.y * GC;
    const int nfull = nA * nA;
    const double c = Upair[I + J * nAs];  // U_I U_J hbar^2 (delta/2pi)^2 / Nf, 0 if no interaction
    const int nseq = 4 * GC;              // [sl = st*2 + a][gl]
    const int m1max = (n + N2 - 1) / N2;
    if (c == 0.0) {
        // src/self_energies.f90:167-171: zero blocks
        for (int t = threadIdx.x; t < 4 * GC * m1max; t += blockDim.x) {
            int a = t & 1, st = (t >> 1) & 1, r = t >> 2;
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
    cplx<T> *scr = buf + (size_t)nseq * PL + (size_t)(threadIdx.x >> 5) * PL;  // this warp's scratch
    cplx<T> *twL = buf + (size_t)(nseq + (blockDim.x >> 5)) * PL;               // the length-N1 table
    fft_table_fill(twL, N1, tw, N2);
    for (int t = threadIdx.x; t < nseq * N1; t += blockDim.x) {
        int gl = t % GC, r = t / GC;
        int sl = r % 4, l1 = r / 4;
        int m2 = m20 + gl;
        int a = sl & 1, st = sl >> 1;
        cplx<T> v{0, 0};
        if (m2 < N2) {
            size_t sid = (size_t)st * nfull + (io + a) + (size_t)(jo + bb) * nA;
            v = V[sid * Nf + (size_t)l1 * N2 + m2];
        }
        buf[(sl * GC + gl) * PL + pidx(l1)] = v;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    {
        const int G = fft_group(N1);
        for (int q = warp * G; q < nseq; q += nw * G) warp_fft_group(buf + q * PL, PL, min(G, nseq - q), scr, fp.p1, +1, twL);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nseq * m1max; t += blockDim.x) {
        int a = t & 1, st = (t >> 1) & 1, r = t >> 2;
        int gl = r % GC, m1 = r / GC;
        int m2 = m20 + gl;
        int64_t w = (int64_t)N2 * m1 + m2;
        if (m2 < N2 && w < n) {
            cplx<T> v = buf[((st * 2 + a) * GC + gl) * PL + pidx(m1)];
            zc *S = st ? SigL : SigR;
            S[w * nfull + (io + a) + (size_t)(jo + bb) * nA] = zc{c * (double)v.x, c * (double)v.y};
        }
    }
}

// ---------------------------------------------------------------------------------
// Persistent forms of kernels A and C for the power-of-two lengths N1 = 64..256 with 4 x 4
// tiles (16 sequences a tile, 512 threads): one block per SM walks the tiles, and the
// input values of the next tile are copied asynchronously into the second buffer while the
// current tile is transformed, so the HBM reads overlap the transforms and the stores.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

// Kernel A: tile = SA adjacent sequences x GA adjacent m2 (SA = 4, GA = 4: one block of 16
// warps per SM; SA = 4, GA = 2: two blocks of 8 warps, whose phases interleave; SA = 2,
// GA = 8: one block of 16 warps whose Y rows are written in 128-byte runs, FP64 only);
// tiles ordered sequence-tile fastest. The FP64 values are copied into a staging buffer;
// with T = float they are converted into a work buffer before the transforms (Y then holds
// FP32 spectra).
template <typename T, int N1, int GA, int SA = 4>
__global__ void __launch_bounds__(32 * SA * GA, 16 / (SA * GA)) sig2_fwdA_p(const double *__restrict__ X, int64_t nblk,
                                                                        int n, const int2 *__restrict__ desc, int nY,
                                                                        FftPlan fp, const zc *__restrict__ tw,
                                                                        cplx<T> *__restrict__ Y, int nitems) {
    constexpr int NS = SA * GA;  // one warp per sequence: blockDim.x = 32 NS
    constexpr bool F64 = sizeof(T) == 8;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N2 = fp.N2, Nf = fp.Nf, PL = padded_len(N1);
    const int nst = (nY + SA - 1) / SA;
    const int m1max = (n + N2 - 1) / N2;  // zero padding beyond n energies
    zc *stg0 = (zc *)smem_raw;      // 2 x NS staging sequences
    zc *twc0 = stg0 + 2 * NS * PL;  // 2 x W_Nf^{m2 l1} of a tile's GA columns, [l1][m2 - m20]
    cplx<T> *wb = F64 ? nullptr : (cplx<T> *)(twc0 + 2 * GA * N1);          // FP32 work sequences
    cplx<T> *twL = F64 ? (cplx<T> *)(twc0 + 2 * GA * N1) : wb + NS * PL;    // the length-N1 table
    fft_table_fill(twL, N1, tw, N2);
    // lanes: m2 fastest, then sequence (64-byte global runs, conflict-free shared stores);
    // blockDim.x is a multiple of NS, so a thread keeps its (sequence, m2) on every tile
    const int gl_t = threadIdx.x % GA, sl_t = (threadIdx.x / GA) % SA;
    auto load = [&](int it, zc *b, zc *twc) {
        const int s0 = (it % nst) * SA, m20 = (it / nst) * GA;
        const int s = s0 + sl_t, m2 = m20 + gl_t;
        const int2 d = s < nY ? desc[s] : int2{-1, 0};
        for (int t = threadIdx.x; t < NS * N1; t += blockDim.x) {
            const int m1 = t / NS;
            const int64_t w = (int64_t)N2 * m1 + m2;
            zc *dst = b + (sl_t * GA + gl_t) * PL + pidx(m1);
            if (m1 < m1max && s < nY && w < n) {
                const double *blk = X + w * nblk;
                if (d.x >= 0 && d.y == d.x + 1 && ((reinterpret_cast<uintptr_t>(blk + d.x) & 15) == 0)) {
                    cp_async16(dst, blk + d.x);
                } else {
                    if (d.x >= 0) cp_async8(&dst->x, blk + d.x);
                    else dst->x = 0.0;
                    cp_async8(&dst->y, blk + d.y);
                }
            } else {
                *dst = zc{0.0, 0.0};
            }
        }
        for (int t = threadIdx.x; t < GA * N1; t += blockDim.x) {
            const int g2 = t % GA, l1 = t / GA;
            cp_async16(&twc[t], &tw[(size_t)(m20 + g2) * l1]);
        }
    };
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5, G = fft_group(N1);
    if (blockIdx.x < nitems) load(blockIdx.x, stg0, twc0);
    cp_async_commit();
    int cur = 0;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int nxt = it + gridDim.x;
        if (nxt < nitems) load(nxt, stg0 + (cur ^ 1) * NS * PL, twc0 + (cur ^ 1) * GA * N1);
        cp_async_commit();
        const int s0 = (it % nst) * SA, m20 = (it / nst) * GA;
        const zc *twc = twc0 + cur * GA * N1;
        cp_async_wait1();
        __syncthreads();
        cplx<T> *b;
        if constexpr (F64) {
            b = stg0 + cur * NS * PL;
        } else {
            const zc *sb = stg0 + cur * NS * PL;
            for (int t = threadIdx.x; t < NS * PL; t += blockDim.x) wb[t] = cvt<T>(sb[t]);
            __syncthreads();
            b = wb;
        }
        for (int q = warp * G; q < NS; q += nw * G) warp_fft_pow2<T, N1>(b + q * PL, PL, min(G, NS - q), -1, twL);
        __syncthreads();
        // lanes: m2 fastest, then sequence, then l1
        for (int t = threadIdx.x; t < NS * N1; t += blockDim.x) {
            const int gl = t % GA, sl = (t / GA) % SA, l1 = t / NS;
            const int s = s0 + sl, m2 = m20 + gl;
            if (s < nY) Y[(size_t)s * Nf + (size_t)l1 * N2 + m2] = b[(sl * GA + gl) * PL + pidx(l1)] * cvt<T>(twc[l1 * GA + gl]);
        }
        __syncthreads();  // the buffers are rewritten by the next tiles
        cur ^= 1;
    }
}

// Kernel C: tile = one column jo+bb of a 2x2 output block x GC adjacent m2 (GC = 4: one
// block of 16 warps per SM; GC = 2: two blocks of 8 warps); tiles ordered m2 fastest
// (neighbouring blocks read neighbouring pieces of the same V rows)
template <typename T, int N1, int GC>
__global__ void __launch_bounds__(128 * GC, 4 / GC) sig2_invC_p(const cplx<T> *__restrict__ V, zc *__restrict__ SigR,
                                                              zc *__restrict__ SigL, int nA, int nAs, int n,
                                                              const double *__restrict__ Upair, FftPlan fp,
                                                              const zc *__restrict__ tw, int nitems) {
    constexpr int NS = 4 * GC;  // one warp per sequence: blockDim.x = 32 NS
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N2 = fp.N2, Nf = fp.Nf, PL = padded_len(N1);
    const int nmt = N2 / GC, nfull = nA * nA;
    const int m1max = (n + N2 - 1) / N2;
    cplx<T> *buf0 = (cplx<T> *)smem_raw;
    cplx<T> *twL = buf0 + 2 * NS * PL;  // the length-N1 table
    fft_table_fill(twL, N1, tw, N2);
    auto tile = [&](int it, int &io, int &jo, int &bb, int &m20, double &c) {
        const int pc = it / nmt;
        m20 = (it % nmt) * GC;
        bb = pc & 1;
        const int pairid = pc >> 1, I = pairid % nAs, J = pairid / nAs;
        io = 2 * I;
        jo = 2 * J;
        c = Upair[I + J * nAs];  // U_I U_J hbar^2 (delta/2pi)^2 / Nf, 0 if no interaction
    };
    auto load = [&](int it, cplx<T> *b) {
        int io, jo, bb, m20;
        double c;
        tile(it, io, jo, bb, m20, c);
        if (c == 0.0) return;  // src/self_energies.f90:167-171: a zero block, nothing to read
        for (int t = threadIdx.x; t < NS * N1; t += blockDim.x) {
            const int gl = t % GC, r = t / GC, sl = r & 3, l1 = r >> 2;
            const int a = sl & 1, st = sl >> 1;
            const size_t sid = (size_t)st * nfull + (io + a) + (size_t)(jo + bb) * nA;
            cp_async_elem(b + (sl * GC + gl) * PL + pidx(l1), V + sid * Nf + (size_t)l1 * N2 + m20 + gl, true);
        }
    };
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5, G = fft_group(N1);
    if (blockIdx.x < nitems) load(blockIdx.x, buf0);
    cp_async_commit();
    int cur = 0;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int nxt = it + gridDim.x;
        if (nxt < nitems) load(nxt, buf0 + (cur ^ 1) * NS * PL);
        cp_async_commit();
        cp_async_wait1();
        __syncthreads();
        int io, jo, bb, m20;
        double c;
        tile(it, io, jo, bb, m20, c);
        cplx<T> *b = buf0 + cur * NS * PL;
        if (c != 0.0)
            for (int q = warp * G; q < NS; q += nw * G) warp_fft_pow2<T, N1>(b + q * PL, PL, min(G, NS - q), +1, twL);
        __syncthreads();
        // lanes: row a fastest (32-byte global runs), then m2, then stage (conflict-free reads)
        for (int t = threadIdx.x; t < NS * m1max; t += blockDim.x) {
            const int a = t & 1, gl = (t >> 1) % GC, st = (t / (2 * GC)) & 1, m1 = t / NS;
            const int64_t w = (int64_t)N2 * m1 + m20 + gl;
            if (w < n) {
                cplx<T> v = (c != 0.0) ? b[((st * 2 + a) * GC + gl) * PL + pidx(m1)] : cplx<T>{0, 0};
                zc *S = st ? SigL : SigR;
                S[w * nfull + (io + a) + (size_t)(jo + bb) * nA] = zc{c * (double)v.x, c * (double)v.y};
            }
        }
        __syncthreads();  // the buffer is rewritten by the next tiles
        cur ^= 1;
    }
}

// Kernel C with a tile of two site pairs (I, I+1) of one output column (J, bb): the 16
// sequences are Sigma^R and Sigma^< of rows 2I .. 2I+3 x 2 adjacent m2, so each energy's four
// rows go out as one 64-byte run (V is read in 32-byte runs). One block of 16 warps per SM.
template <typename T, int N1>
__global__ void __launch_bounds__(512, 1) sig2_invC_p2(const cplx<T> *__restrict__ V, zc *__restrict__ SigR,
                                                       zc *__restrict__ SigL, int nA, int nAs, int n,
                                                       const double *__restrict__ Upair, FftPlan fp,
                                                       const zc *__restrict__ tw, int nitems) {
    constexpr int GC = 2, NR = 4, NS = 2 * NR * GC;  // stage x row x m2
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N2 = fp.N2, Nf = fp.Nf, PL = padded_len(N1);
    const int nmt = N2 / GC, nfull = nA * nA, nI2 = (nAs + 1) / 2;
    const int m1max = (n + N2 - 1) / N2;
    cplx<T> *buf0 = (cplx<T> *)smem_raw;
    cplx<T> *twL = buf0 + 2 * NS * PL;
    fft_table_fill(twL, N1, tw, N2);
    // item -> output column, first row, m2 block, the two pairs' scales (0: no interaction
    // or no second pair)
    auto tile = [&](int it, int &io, int &jo, int &bb, int &m20, double &c0, double &c1) {
        const int pc = it / nmt;
        m20 = (it % nmt) * GC;
        bb = pc & 1;
        const int q = pc >> 1, I = 2 * (q % nI2), J = q / nI2;
        io = 2 * I;
        jo = 2 * J;
        c0 = Upair[I + J * nAs];
        c1 = (I + 1 < nAs) ? Upair[I + 1 + J * nAs] : 0.0;
    };
    auto load = [&](int it, cplx<T> *b) {
        int io, jo, bb, m20;
        double c0, c1;
        tile(it, io, jo, bb, m20, c0, c1);
        for (int t = threadIdx.x; t < NS * N1; t += blockDim.x) {
            const int gl = t % GC, r = t / GC, sl = r % (2 * NR), l1 = r / (2 * NR);
            const int a = sl % NR, st = sl / NR;
            if ((a < 2 ? c0 : c1) == 0.0) continue;  // a zero block: nothing to read
            const size_t sid = (size_t)st * nfull + (io + a) + (size_t)(jo + bb) * nA;
            cp_async_elem(b + (sl * GC + gl) * PL + pidx(l1), V + sid * Nf + (size_t)l1 * N2 + m20 + gl, true);
        }
    };
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5, G = fft_group(N1);
    if (blockIdx.x < nitems) load(blockIdx.x, buf0);
    cp_async_commit();
    int cur = 0;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int nxt = it + gridDim.x;
        if (nxt < nitems) load(nxt, buf0 + (cur ^ 1) * NS * PL);
        cp_async_commit();
        cp_async_wait1();
        __syncthreads();
        int io, jo, bb, m20;
        double c0, c1;
        tile(it, io, jo, bb, m20, c0, c1);
        cplx<T> *b = buf0 + cur * NS * PL;
        for (int q = warp * G; q < NS; q += nw * G) {
            // sequence q = (st NR + a) GC + gl; skip the transforms of zero blocks
            const int a = (q / GC) % NR;
            if ((a < 2 ? c0 : c1) != 0.0) warp_fft_pow2<T, N1>(b + q * PL, PL, min(G, NS - q), +1, twL);
        }
        __syncthreads();
        // lanes: row a fastest (64-byte global runs), then m2, then stage
        for (int t = threadIdx.x; t < NS * m1max; t += blockDim.x) {
            const int a = t % NR, gl = (t / NR) % GC, st = (t / (NR * GC)) & 1, m1 = t / NS;
            const int64_t w = (int64_t)N2 * m1 + m20 + gl;
            const double c = a < 2 ? c0 : c1;
            if (w < n && (a < 2 || io + a < nA)) {
                cplx<T> v = (c != 0.0) ? b[((st * NR + a) * GC + gl) * PL + pidx(m1)] : cplx<T>{0, 0};
                zc *S = st ? SigL : SigR;
                S[w * nfull + (io + a) + (size_t)(jo + bb) * nA] = zc{c * (double)v.x, c * (double)v.y};
            }
        }
        __syncthreads();  // the buffer is rewritten by the next tiles
        cur ^= 1;
    }
}

// ---------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------
static void factor_len(int L, FftLen &P) {
    P.L = L;
    P.nrad = 0;
    P.code = 0;
    int m = L;
    for (int r : {8, 4, 2, 3, 5, 7})
        while (m % r == 0) {
            P.code |= (unsigned)r << (4 * P.nrad);
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

// the kernel instantiations for a plan and element type: compile-time lengths for the
// power-of-two splits, persistent forms of kernels A and C for those
template <typename T>
using FwdAFn = void (*)(const double *, int64_t, int, const int2 *, int, FftPlan, const zc *, cplx<T> *, int, int);
template <typename T> using MidFn = void (*)(const cplx<T> *, cplx<T> *, const int2 *, int, FftPlan, const zc *, int);
template <typename T>
using InvCFn = void (*)(const cplx<T> *, zc *, zc *, int, int, int, const double *, FftPlan, const zc *, int);
template <typename T> static FwdAFn<T> pick_fwdA(int N1, int SA, int GA) {
    if (SA == 4 && GA == 4) switch (N1) {
            case 64: return sig2_fwdA<T, 64>;
            case 128: return sig2_fwdA<T, 128>;
            case 256: return sig2_fwdA<T, 256>;
        }
    return sig2_fwdA<T, 0>;
}
template <typename T> static MidFn<T> pick_mid(int N2) {
    switch (N2) {
        case 64: return sig2_mid<T, 64>;
        case 128: return sig2_mid<T, 128>;
    }
    return sig2_mid<T, 0>;
}
template <typename T> static InvCFn<T> pick_invC(int N1, int GC) {
    if (GC == 4) switch (N1) {
            case 64: return sig2_invC<T, 64>;
            case 128: return sig2_invC<T, 128>;
            case 256: return sig2_invC<T, 256>;
        }
    return sig2_invC<T, 0>;
}
template <typename T>
using FwdAPFn = void (*)(const double *, int64_t, int, const int2 *, int, FftPlan, const zc *, cplx<T> *, int);
template <typename T>
using InvCPFn = void (*)(const cplx<T> *, zc *, zc *, int, int, int, const double *, FftPlan, const zc *, int);
// persistent kernels A / C for power-of-two N1; w = 4 (16-sequence tiles, one block per
// SM) or 2 (8-sequence tiles, two blocks per SM)
template <typename T> static FwdAPFn<T> pick_fwdA_p(int N1, int w) {
    if (w == 8) {  // two sequences x eight m2 (FP64: the twiddle columns of 8 m2 fit next to the staging)
        if (sizeof(T) != 8) return nullptr;
        switch (N1) {
            case 64: return sig2_fwdA_p<T, 64, 8, 2>;
            case 128: return sig2_fwdA_p<T, 128, 8, 2>;
            case 256: return sig2_fwdA_p<T, 256, 8, 2>;
        }
        return nullptr;
    }
    if (w == 2) switch (N1) {
            case 64: return sig2_fwdA_p<T, 64, 2>;
            case 128: return sig2_fwdA_p<T, 128, 2>;
            case 256: return sig2_fwdA_p<T, 256, 2>;
        }
    switch (N1) {
        case 64: return sig2_fwdA_p<T, 64, 4>;
        case 128: return sig2_fwdA_p<T, 128, 4>;
        case 256: return sig2_fwdA_p<T, 256, 4>;
    }
    return nullptr;
}
template <typename T> static InvCPFn<T> pick_invC_p(int N1, int w) {
    if (w == 8) {  // two site pairs x two m2 (FP64)
        if (sizeof(T) != 8) return nullptr;
        switch (N1) {
            case 64: return sig2_invC_p2<T, 64>;
            case 128: return sig2_invC_p2<T, 128>;
            case 256: return sig2_invC_p2<T, 256>;
        }
        return nullptr;
    }
    if (w == 2) switch (N1) {
            case 64: return sig2_invC_p<T, 64, 2>;
            case 128: return sig2_invC_p<T, 128, 2>;
            case 256: return sig2_invC_p<T, 256, 2>;
        }
    switch (N1) {
        case 64: return sig2_invC_p<T, 64, 4>;
        case 128: return sig2_invC_p<T, 128, 4>;
        case 256: return sig2_invC_p<T, 256, 4>;
    }
    return nullptr;
}
// kernel A's tile: w adjacent m2 x (w == 8 ? 2 : 4) adjacent sequences
static int fwdA_sa(int w) { return w == 8 ? 2 : 4; }
template <typename T> static size_t smem_fwdA_p(int N1, int w) {
    const size_t PL = padded_len(N1), ns = (size_t)fwdA_sa(w) * w;
    return sizeof(zc) * (2 * ns * PL + 2 * (size_t)w * N1) + (sizeof(T) == 8 ? 0 : sizeof(cplx<T>) * ns * PL) +
           sizeof(cplx<T>) * fft_table_len(N1);
}
template <typename T> static size_t smem_invC_p(int N1, int w) {
    const size_t ns = (w == 8) ? 16 : (size_t)4 * w;
    return sizeof(cplx<T>) * ((size_t)2 * ns * padded_len(N1) + (size_t)fft_table_len(N1));
}
template <typename T> static size_t smem_A(const qs_handle *h) {
    return sizeof(cplx<T>) * ((size_t)(h->sig2_SA * h->sig2_GA + 8) * padded_len(h->fft.N1) + fft_table_len(h->fft.N1));
}
template <typename T> static size_t smem_B(const qs_handle *h) {
    return sizeof(cplx<T>) *
           ((size_t)(2 * 24 + 32 + 16) * padded_len(h->fft.N2) + 2 * h->fft.N2 + fft_table_len(h->fft.N2));
}
template <typename T> static size_t smem_C(const qs_handle *h) {
    return sizeof(cplx<T>) * ((size_t)(4 * h->sig2_GC + 8) * padded_len(h->fft.N1) + fft_table_len(h->fft.N1));
}
// the persistent forms need N2 a multiple of the 4-column tile (true for N2 >= 64 here)
static bool persistent_AC(const FftPlan &fp) { return pick_fwdA_p<double>(fp.N1, 4) && fp.N2 % 4 == 0; }

template <typename T> static int sigma2_attributes(qs_handle *h) {
    const FftPlan &fp = h->fft;
    QS_CUDA(h, smem_cap((const void *)pick_fwdA<T>(fp.N1, h->sig2_SA, h->sig2_GA)));
    QS_CUDA(h, smem_cap((const void *)pick_mid<T>(fp.N2)));
    QS_CUDA(h, smem_cap((const void *)pick_invC<T>(fp.N1, h->sig2_GC)));
    if (persistent_AC(fp))
        for (int w : {2, 4}) {
            QS_CUDA(h, smem_cap((const void *)pick_fwdA_p<T>(fp.N1, w)));
            QS_CUDA(h, smem_cap((const void *)pick_invC_p<T>(fp.N1, w)));
        }
    if (persistent_AC(fp) && pick_fwdA_p<T>(fp.N1, 8)) QS_CUDA(h, smem_cap((const void *)pick_fwdA_p<T>(fp.N1, 8)));
    if (persistent_AC(fp) && pick_invC_p<T>(fp.N1, 8)) QS_CUDA(h, smem_cap((const void *)pick_invC_p<T>(fp.N1, 8)));
    return 0;
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
    // tile sizes: one warp per sequence, 64 B contiguous global accesses where possible
    if (fp.N1 > 512 || fp.N2 > 128) {
        h->err = "sigma2: FFT length " + std::to_string(fp.Nf) + " needs N1 <= 512 and N2 <= 128";
        return -1;
    }
    const int PL1 = padded_len(fp.N1);
    int GA = std::min(fp.N2, 4), SA = 4;
    while ((size_t)(SA * GA + 8) * PL1 * sizeof(zc) > 112 * 1024 && GA > 1) GA /= 2;
    while ((size_t)(SA * GA + 8) * PL1 * sizeof(zc) > 112 * 1024 && SA > 1) SA /= 2;
    int GC = std::min(fp.N2, 4);
    while ((size_t)(4 * GC + 8) * PL1 * sizeof(zc) > 112 * 1024 && GC > 1) GC /= 2;
    h->sig2_SA = SA;
    h->sig2_GA = GA;
    h->sig2_GC = GC;
    if (smem_A<double>(h) > SMEM_MAX || smem_B<double>(h) > SMEM_MAX || smem_C<double>(h) > SMEM_MAX) {
        h->err = "sigma2: FFT tiles exceed shared memory";
        return -1;
    }
    if ((rc = sigma2_attributes<double>(h))) return rc;
    if (h->precision == QS_PREC_MIXED && (rc = sigma2_attributes<float>(h))) return rc;
    // every buffer is zeroed on h->stream by dalloc: the tables are copied on the same
    // stream (after the zeroing) and the host staging vectors must outlive the copies
    QS_CUDA(h, cudaStreamSynchronize(h->stream));
    return 0;
}

// Y and V hold FP32 spectra when T = float (in the first half of the same allocations)
template <typename T> static int sigma2_run(qs_handle *h, const double *d_x) {
    const FftPlan &fp = h->fft;
    const int nA = h->nA;
    const bool pers = persistent_AC(fp);
    cplx<T> *Y = (cplx<T> *)h->d_Y, *V = (cplx<T> *)h->d_V;
    const int cand[2] = {4, 2};  // tile widths, autotuned per size (results are identical)
    const int key = tune_key(nA, h->n) + (sizeof(T) == 4 ? 1 << 20 : 0);
    if (pers) {
        // kernel A: the FP64 form also has the 2 x 8 tile (128-byte Y runs)
        const int candA[3] = {4, 2, 8};
        const bool wide = sizeof(T) == 8 && fp.N2 % 8 == 0 &&
                          smem_fwdA_p<T>(fp.N1, 8) + 2048 <= (size_t)SMEM_MAX;
        int rc = tune_launch(h, TUNE_SIG2_A, key, candA, wide ? 3 : 2, 4, [&](int w) -> int {
            const int sa = fwdA_sa(w);
            const int nitems = (int)((h->nY + sa - 1) / sa) * (fp.N2 / w);
            const int per_sm = 16 / (sa * w);
            const auto fn = pick_fwdA_p<T>(fp.N1, w);
            int pa = prof_begin(h, K_SIG2A);
            fn<<<std::min(nitems, 148 * per_sm), 32 * sa * w, smem_fwdA_p<T>(fp.N1, w), h->stream>>>(
                d_x, h->nblk, h->n, h->d_ydesc, (int)h->nY, fp, h->d_tw, Y, nitems);
            prof_end(h, pa);
            QS_CUDA(h, cudaGetLastError());
            return 0;
        });
        if (rc) return rc;
    } else {
        int pa = prof_begin(h, K_SIG2A);
        dim3 gA((unsigned)((h->nY + h->sig2_SA - 1) / h->sig2_SA), (unsigned)((fp.N2 + h->sig2_GA - 1) / h->sig2_GA));
        pick_fwdA<T>(fp.N1, h->sig2_SA, h->sig2_GA)<<<gA, 256, smem_A<T>(h), h->stream>>>(
            d_x, h->nblk, h->n, h->d_ydesc, (int)h->nY, fp, h->d_tw, Y, h->sig2_SA, h->sig2_GA);
        prof_end(h, pa);
        QS_CUDA(h, cudaGetLastError());
    }
    if (h->sig2_npairs > 0) {
        const int nitems = h->sig2_npairs * (fp.N1 / 2 + 1);
        const int gB = std::min(nitems, 148);  // persistent: one block per SM
        int pb = prof_begin(h, K_SIG2B);
        pick_mid<T>(fp.N2)<<<gB, 512, smem_B<T>(h), h->stream>>>(Y, V, h->sig2_pairs, nA, fp, h->d_tw, nitems);
        prof_end(h, pb);
        QS_CUDA(h, cudaGetLastError());
    }
    if (pers) {
        // kernel C: the FP64 form also has the two-site-pair tile (64-byte Sigma runs)
        const int candC[3] = {4, 2, 8};
        const bool wide = sizeof(T) == 8 && fp.N2 % 2 == 0;
        int rc = tune_launch(h, TUNE_SIG2_C, key, candC, wide ? 3 : 2, 4, [&](int w) -> int {
            const int nitems = (w == 8) ? 2 * ((h->nAs + 1) / 2) * h->nAs * (fp.N2 / 2)
                                        : 2 * h->nAs * h->nAs * (fp.N2 / w);
            const int thr = (w == 8) ? 512 : 128 * w, per_sm = (w == 8) ? 1 : 4 / w;
            int pc = prof_begin(h, K_SIG2C);
            pick_invC_p<T>(fp.N1, w)<<<std::min(nitems, 148 * per_sm), thr, smem_invC_p<T>(fp.N1, w), h->stream>>>(
                V, h->d_SigR, h->d_SigL, nA, h->nAs, h->n, h->sig2_Upair, fp, h->d_tw, nitems);
            prof_end(h, pc);
            QS_CUDA(h, cudaGetLastError());
            return 0;
        });
        if (rc) return rc;
    } else {
        int pc = prof_begin(h, K_SIG2C);
        dim3 gC((unsigned)(2 * h->nAs * h->nAs), (unsigned)((fp.N2 + h->sig2_GC - 1) / h->sig2_GC));
        pick_invC<T>(fp.N1, h->sig2_GC)<<<gC, 256, smem_C<T>(h), h->stream>>>(
            V, h->d_SigR, h->d_SigL, nA, h->nAs, h->n, h->sig2_Upair, fp, h->d_tw, h->sig2_GC);
        prof_end(h, pc);
        QS_CUDA(h, cudaGetLastError());
    }
    return 0;
}

int sigma2_compute(qs_handle *h, const double *d_x, bool fp32) {
    if (fp32) {
        if (h->precision != QS_PREC_MIXED) {
            h->err = "sigma2: FP32 transforms need a QS_PREC_MIXED handle";
            return -1;
        }
        return sigma2_run<float>(h, d_x);
    }
    return sigma2_run<double>(h, d_x);
}

}  // namespace qs
