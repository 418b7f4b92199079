// sweep.cu -- the energy sweep (sweep / G_at_energy, src/scf.f90:280-415) as batched
// kernels over the whole energy grid:
//   dyson_gj        G^r(w) = [hbar w - H + (i/2hbar)(GammaL+GammaR) - Sigma^r(w)]^-1 by
//                   in-place Gauss-Jordan elimination with partial pivoting, one thread
//                   block per energy, the matrix staged in shared memory (global
//                   workspace when N^2 complex does not fit), pivot search by warp
//                   shuffles (invert_complex, common/linear_algebra.f90:58-88)
//   keldysh_scf2    G^< = G^r Sigma^< G^a on the active block as two complex GEMMs per
//                   energy, written straight into the SCF vector with its diagonals
//                   (modes M_INIT2 / M_SCF2, src/scf.f90:340-355)
//   final_outputs   modes M_SCF1 / M_FINAL (src/scf.f90:357-410): on-site and intra-atom
//                   blocks of G^<, Im G^r_ii, the current integrand
// plus the reductions over energies (equal_time_lesser, gather_onsite, gather_atoms,
// Current, the sanity sums) and the pack_gf / unpack_gf layout conversions.
#include <algorithm>
#include <cmath>

#include "qs_common.cuh"

namespace qs {


// ---------------------------------------------------------------------------------
// Block-wide argmax of cabs1 over rows k..N-1 of column k (first maximum wins, as
// LAPACK's izamax).
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void warp_argmax(double &v, int &i) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double v2 = __shfl_down_sync(0xffffffffu, v, o);
        int i2 = __shfl_down_sync(0xffffffffu, i, o);
        if (v2 > v || (v2 == v && i2 < i)) {
            v = v2;
            i = i2;
        }
    }
}

struct DysonArgs {
    int N, nA, iw0, iw1;
    const zc *Hemb, *Sig1, *SigR;
    const int *pos;  // full index -> active index, -1 if inactive
    const int *act;
    const double *omega;
    int use_sigma, order2;
    int out_mode;  // 0: G_AA for energy iw at Gout[iw*nA^2]; 1: full G at Gout[(iw-iw0)*N^2]
    zc *Gout;
    zc *ws;        // global workspace (N^2 per block) when the matrix is not in shared memory
    int *info;     // min over energies of (iw + 1) with a zero pivot; INT_MAX if none
    const zc *Ain; // batched-inversion mode: matrices to invert (nullptr for the sweep)
    int *info_each;
};

__global__ void __launch_bounds__(512) dyson_gj(DysonArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N = a.N;
    const bool in_smem = (a.ws == nullptr);
    zc *M = in_smem ? (zc *)smem_raw : a.ws + (size_t)blockIdx.x * N * N;
    __shared__ unsigned short perm[512];
    __shared__ double wv[16];
    __shared__ int wi[16];
    __shared__ int piv_s;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int NG = nthr / N;  // threads per row in the update (>= 1, N <= 512)
    const int myrow = tid % N, mygrp = tid / N;
    const bool upd = mygrp < NG;

    for (int iw = a.iw0 + blockIdx.x; iw < a.iw1; iw += gridDim.x) {
        // ---- build w1 = Hemb - (Sig1 + Sigma2^r(w)) on act x act, + hbar w on the diagonal
        if (a.Ain) {
            const zc *A = a.Ain + (size_t)(iw - a.iw0) * N * N;
            for (int idx = tid; idx < N * N; idx += nthr) M[idx] = A[idx];
        } else {
            const double w = a.omega[iw];
            const zc *SR = a.SigR + (size_t)iw * a.nA * a.nA;
            for (int idx = tid; idx < N * N; idx += nthr) {
                int i = idx % N, j = idx / N;
                zc v = a.Hemb[idx];
                if (a.use_sigma) {
                    int pi = a.pos[i], pj = a.pos[j];
                    if (pi >= 0 && pj >= 0) {
                        zc s = a.Sig1[idx];
                        if (a.order2) s = s + SR[pi + (size_t)pj * a.nA];
                        v = v - s;
                    }
                }
                if (i == j) v.x += w;
                M[idx] = v;
            }
        }
        __syncthreads();
        bool singular = false;
        int first_zero = 0;  // 1 + the first step with a zero pivot (LAPACK's INFO)
        // ---- Gauss-Jordan with row interchanges
        for (int k = 0; k < N; k++) {
            // pivot search
            double v = -1.0;
            int vi = N;
            for (int i = k + tid; i < N; i += nthr) {
                double c = cabs1(M[i + (size_t)k * N]);
                if (c > v) { v = c; vi = i; }
            }
            warp_argmax(v, vi);
            if ((tid & 31) == 0) { wv[tid >> 5] = v; wi[tid >> 5] = vi; }
            __syncthreads();
            if (tid < 32) {
                int nw = nthr >> 5;
                v = tid < nw ? wv[tid] : -1.0;
                vi = tid < nw ? wi[tid] : N;
                warp_argmax(v, vi);
                if (vi >= N) vi = k;  // no comparable entry (NaN column): keep row k, in range
                if (tid == 0) { piv_s = vi; perm[k] = vi; }
            }
            __syncthreads();
            const int p = piv_s;
            if (p != k) {
                for (int j = tid; j < N; j += nthr) {
                    zc t = M[k + (size_t)j * N];
                    M[k + (size_t)j * N] = M[p + (size_t)j * N];
                    M[p + (size_t)j * N] = t;
                }
                __syncthreads();
            }
            zc pivot = M[k + (size_t)k * N];
            if (pivot.x == 0.0 && pivot.y == 0.0) {
                if (!singular) first_zero = k + 1;
                singular = true;
            }
            zc inv = singular ? zc{0.0, 0.0} : crecip(pivot);
            zc f = upd ? M[myrow + (size_t)k * N] : zc{0.0, 0.0};
            __syncthreads();
            // scale the pivot row (M[k][k] is replaced by 1 first, so it ends as 1/pivot)
            for (int j = tid; j < N; j += nthr) {
                zc t = (j == k) ? zc{1.0, 0.0} : M[k + (size_t)j * N];
                M[k + (size_t)j * N] = t * inv;
            }
            __syncthreads();
            // rank-1 update of every other row (column k is replaced by 0 first)
            if (upd && myrow != k) {
                for (int j = mygrp; j < N; j += NG) {
                    zc t = (j == k) ? zc{0.0, 0.0} : M[myrow + (size_t)j * N];
                    zc r = M[k + (size_t)j * N];
                    t.x = fma(-f.x, r.x, t.x);
                    t.x = fma(f.y, r.y, t.x);
                    t.y = fma(-f.x, r.y, t.y);
                    t.y = fma(-f.y, r.x, t.y);
                    M[myrow + (size_t)j * N] = t;
                }
            }
            __syncthreads();
        }
        // undo the row interchanges by column interchanges in reverse order
        if (tid < N) {
            for (int k = N - 1; k >= 0; k--) {
                int p = perm[k];
                if (p != k) {
                    zc t = M[tid + (size_t)k * N];
                    M[tid + (size_t)k * N] = M[tid + (size_t)p * N];
                    M[tid + (size_t)p * N] = t;
                }
            }
        }
        __syncthreads();
        if (singular && tid == 0) {
            atomicMin(a.info, iw + 1);
            if (a.info_each) a.info_each[iw - a.iw0] = first_zero;
        }
        // ---- output
        if (a.out_mode == 0) {
            const int nA = a.nA;
            zc *G = a.Gout + (size_t)iw * nA * nA;
            for (int idx = tid; idx < nA * nA; idx += nthr) {
                int p = idx % nA, q = idx / nA;
                G[idx] = M[a.act[p] + (size_t)a.act[q] * N];
            }
        } else {
            zc *G = a.Gout + (size_t)(iw - a.iw0) * N * N;
            for (int idx = tid; idx < N * N; idx += nthr) G[idx] = M[idx];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------
// Blocked Gauss-Jordan (panel width GJ_B) for matrices held in shared memory. For every
// panel K = [k0, k0+b): warp 0 factors the N x b panel (pivot search by shuffles, full-row
// interchanges, scaling and elimination restricted to the panel columns); then the whole
// block applies the panel's transformation to the other columns as one rank-b update,
//   A[i, j] += sum_t A[i, K_t] A[K_t, j]            (i, j outside K; register tiles 4 x 4)
//   A[K, j]  = A[K, K] A[K, j]                       (the pivot rows, one column per thread)
// which equals the unblocked elimination (row interchanges commute with the deferred update
// because they act on whole rows). Interchanges are undone on the columns at the end.
// ---------------------------------------------------------------------------------
constexpr int GJ_B = 16;  // panel width = the k extent of one FP64 tensor-core MMA

// shared-memory position of element (i, j): column-major with the leading dimension padded
// to a multiple of 8 units (16 B each) and the unit index XORed with (j mod 8), so that a
// warp walking along a row (fixed i, consecutive j) hits all banks; columns start on
// 128-byte boundaries, so the XOR stays inside the column and the map is one-to-one
__host__ __device__ __forceinline__ int swz_ld(int N) { return ((N + 7) / 8) * 8; }
__device__ __forceinline__ int swz(int i, int j, int N) { return (i + j * swz_ld(N)) ^ (j & 7); }
__host__ __device__ __forceinline__ int swz_units(int N) { return N * swz_ld(N); }

// 15 warps: one per 8-column tile of a 120-column matrix in the update, and 136 registers a
// thread for the panel's register-resident rows
constexpr int BGJ_THREADS = 480;

// named barrier of the panel warps (ids 1.. are free; 0 is __syncthreads)
__device__ __forceinline__ void panel_bar(int nthreads) { asm volatile("bar.sync 1, %0;\n" ::"r"(nthreads) : "memory"); }

// argmax over a warp with the result in every lane (first maximum wins)
__device__ __forceinline__ void warp_argmax_all(double &v, int &i) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double v2 = __shfl_xor_sync(0xffffffffu, v, o);
        int i2 = __shfl_xor_sync(0xffffffffu, i, o);
        if (v2 > v || (v2 == v && i2 < i)) {
            v = v2;
            i = i2;
        }
    }
}

// Storage of the matrix of the blocked Gauss-Jordan: GM = false, the swizzled shared-memory
// layout above (16 <= N <= 120 in FP64); GM = true, column-major in the block's slot of a
// global workspace (120 < N <= 256: the working set of the concurrent blocks stays largely in
// L2, and every access of the update is a 128-byte run of 8 consecutive rows).
template <bool GM> __device__ __forceinline__ int bix(int i, int j, int N) { return GM ? i + j * N : swz(i, j, N); }
// panel warps: one thread per row
template <bool GM> __host__ __device__ __forceinline__ int bgj_pw(int N) { return GM ? (N + 31) / 32 : 4; }
constexpr int BGJ_MAXN_GM = 256;

// Blocked Gauss-Jordan inversion with the matrix in (swizzled) shared memory (GM = false,
// 16 <= N <= 120) or in a global workspace (GM = true, 120 < N <= 256). Per panel
// K = [k0, k0 + 16):
//   panel   the panel warps (4, or ceil(N/32) <= 8), thread i holding row i of the panel
//           columns in registers: per column
//           k the pivot search, the exchange of rows k and p (the panel part through shared
//           memory, the rest of the two rows in place), and the elimination restricted to
//           the panel columns; two 128-thread barriers per column
//   update  every warp owns 16 x 8 column tiles j outside K: A[i, j] += A[i, K] A[K, j] for
//           rows i outside K, then A[K, j] = A[K, K] A[K, j], complex products on the FP64
//           tensor cores; the warp reads its A[K, j] fragment before it rewrites those rows,
//           so no block barrier separates the two
// The row interchanges are undone by column interchanges in reverse order at the end.
// NT = 480 (15 warps, one block per SM) or, with the matrix in the global workspace, NT = 256
// (8 warps, two blocks per SM: one block's latency-bound panel overlaps the other's update).
template <bool GM, int NT = BGJ_THREADS>
__global__ void __launch_bounds__(NT, NT <= 256 ? 2 : 1) dyson_bgj_t(DysonArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int PWM = GM ? 8 : 4;  // panel warps at most
    const int N = a.N;
    zc *M = GM ? a.ws + (size_t)blockIdx.x * N * N : (zc *)smem_raw;
    // static shared memory of the shared-memory form stays below 1536 bytes (use_blocked):
    // N = 120 takes the rest
    __shared__ unsigned char perm[GM ? BGJ_MAXN_GM : 128];
    __shared__ unsigned long long cand_k[PWM];  // each panel warp's pivot key (0: no row searched)
    __shared__ int cand_i[PWM];
    __shared__ zc cand_row[PWM][GJ_B];  // each panel warp's pivot candidate row (panel part)
    __shared__ zc krow[GJ_B];           // the panel part of row k before the exchange
    __shared__ int first_zero_s;
    const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nthr >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const int mtiles = (N + 15) / 16, ntiles = (N + 7) / 8;
    const int npw = bgj_pw<GM>(N);  // panel warps

    for (int iw = a.iw0 + blockIdx.x; iw < a.iw1; iw += gridDim.x) {
        if (a.Ain) {
            const zc *A = a.Ain + (size_t)(iw - a.iw0) * N * N;
            for (int idx = tid; idx < N * N; idx += nthr) M[bix<GM>(idx % N, idx / N, N)] = A[idx];
        } else {
            const double w = a.omega[iw];
            const zc *SR = a.SigR + (size_t)iw * a.nA * a.nA;
#pragma unroll 4
            for (int idx = tid; idx < N * N; idx += nthr) {
                int i = idx % N, j = idx / N;
                zc v = a.Hemb[idx];
                if (a.use_sigma) {
                    int pi = a.pos[i], pj = a.pos[j];
                    if (pi >= 0 && pj >= 0) {
                        zc sg = a.Sig1[idx];
                        if (a.order2) sg = sg + SR[pi + (size_t)pj * a.nA];
                        v = v - sg;
                    }
                }
                if (i == j) v.x += w;
                M[bix<GM>(i, j, N)] = v;
            }
        }
        if (tid == 0) first_zero_s = 0;
        bool singular = false;
        __syncthreads();
        for (int k0 = 0; k0 < N; k0 += GJ_B) {
            const int kb = min(GJ_B, N - k0);
            // ---- panel
            if (warp < npw) {
                const int i = tid;  // this thread's row
                // R[j] holds panel column (c + j) mod 16 at step c: the current column is always
                // R[0] and the step loop need not be unrolled (padding columns stay zero)
                zc R[GJ_B];
#pragma unroll
                for (int c = 0; c < GJ_B; c++) R[c] = (i < N && c < kb) ? M[bix<GM>(i, k0 + c, N)] : zc{0, 0};
#pragma unroll 1
                for (int c = 0; c < kb; c++) {
                    const int k = k0 + c;
                    const bool valid = (i >= k && i < N);
                    // every thread prepares 1 / R[0] in case its row becomes the pivot row; the
                    // division overlaps the pivot search
                    const bool z = (R[0].x == 0.0 && R[0].y == 0.0);
                    zc inv_own{0.0, 0.0};
                    if (!singular && !z) {
                        const double id = 1.0 / fma(R[0].x, R[0].x, R[0].y * R[0].y);
                        inv_own = zc{R[0].x * id, -R[0].y * id};
                    }
                    // pivot search: the warp maximum of cabs1, then its lowest lane (first
                    // maximum). cabs1 >= 0, so its bit pattern orders like its value: two
                    // integer warp reductions (high word + 1, 0 for rows not searched; then the
                    // low word among the lanes holding the maximal high word) replace a chain
                    // of FP64 shuffles
                    // (a NaN is an ordinary large key here, so a pivot row is always found)
                    const double v = valid ? cabs1(R[0]) : 0.0;
                    const unsigned long long bits = (unsigned long long)__double_as_longlong(v);
                    const unsigned hk = valid ? min((unsigned)(bits >> 32), 0xfffffffeu) + 1u : 0u, lk = (unsigned)bits;
                    const unsigned mh = __reduce_max_sync(0xffffffffu, hk);
                    const unsigned ml = __reduce_max_sync(0xffffffffu, hk == mh ? lk : 0u);
                    const unsigned bal = __ballot_sync(0xffffffffu, valid && hk == mh && lk == ml);
                    const int wl = bal ? __ffs(bal) - 1 : 32;
                    if (lane == 0) {
                        cand_k[warp] = ((unsigned long long)mh << 32) | ml;
                        cand_i[warp] = bal ? 32 * warp + wl : N;
                    }
                    if (lane == wl) {  // this warp's candidate publishes its scaled row
#pragma unroll
                        for (int j = 0; j < GJ_B; j++) cand_row[warp][j] = (j == 0) ? inv_own : R[j] * inv_own;
                    }
                    if (i == k) {
#pragma unroll
                        for (int j = 0; j < GJ_B; j++) krow[j] = R[j];
                    }
                    panel_bar(32 * npw);
                    // the largest key; on a tie the lower warp (lower rows) wins, as the first
                    // maximum. The warp holding row k has a key > 0, so p is a row in [k, N).
                    unsigned long long bk = cand_k[0];
                    int wb = 0;
                    for (int q = 1; q < npw; q++) {
                        const unsigned long long ck = cand_k[q];
                        if (ck > bk) {
                            bk = ck;
                            wb = q;
                        }
                    }
                    const int p = cand_i[wb];
                    if (bk == (1ull << 32) && !singular) {  // cabs1 of the pivot is +0
                        singular = true;           // every panel thread sees the same pivot
                        if (tid == 0) first_zero_s = k + 1;
                    }
                    if (tid == 0) perm[k] = (unsigned char)p;
                    // rows k and p exchange their panel parts: row p takes the old row k
                    if (p != k && i == p) {
#pragma unroll
                        for (int j = 0; j < GJ_B; j++) R[j] = krow[j];
                    }
                    // eliminate with the scaled pivot row S (S_0 = 1 / pivot), then rotate the
                    // window by one column
                    const zc *S = cand_row[wb];
                    const zc f = R[0];
                    const bool pr = (i == k);
                    zc first;
#pragma unroll
                    for (int j = 0; j < GJ_B; j++) {
                        const zc r = S[j];
                        zc tt;
                        if (pr) {
                            tt = r;
                        } else {
                            tt = (j == 0) ? zc{0.0, 0.0} : R[j];
                            tt.x = fma(-f.x, r.x, tt.x);
                            tt.x = fma(f.y, r.y, tt.x);
                            tt.y = fma(-f.x, r.y, tt.y);
                            tt.y = fma(-f.y, r.x, tt.y);
                        }
                        if (j == 0) first = tt;
                        else R[j - 1] = tt;
                    }
                    R[GJ_B - 1] = first;
                    // the rest of rows k and p (thread i moves column i, its own earlier
                    // exchanges first)
                    if (p != k && i < N && (i < k0 || i >= k0 + kb)) {
                        zc tt = M[bix<GM>(k, i, N)];
                        M[bix<GM>(k, i, N)] = M[bix<GM>(p, i, N)];
                        M[bix<GM>(p, i, N)] = tt;
                    }
                    panel_bar(32 * npw);  // cand_row and krow are rewritten by the next column
                }
                // after kb steps R[j] holds column (kb + j) mod 16
                if (i < N) {
#pragma unroll
                    for (int j = 0; j < GJ_B; j++) {
                        const int c = (kb + j) & (GJ_B - 1);
                        if (c < kb) M[bix<GM>(i, k0 + c, N)] = R[j];
                    }
                }
            }
            __syncthreads();
            // ---- update, one 16 x 8 column tile at a time per warp
            for (int ct = warp; ct < ntiles; ct += nwarps) {
                const int j0 = 8 * ct;
                if (j0 >= k0 && j0 + 8 <= k0 + kb) continue;  // the whole column tile is in K
                double br[4], bi[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int kr = t4 + 4 * q, c = j0 + g;
                    zc v = (kr < kb && c < N) ? M[bix<GM>(k0 + kr, c, N)] : zc{0, 0};
                    br[q] = v.x;
                    bi[q] = v.y;
                }
#pragma unroll 1
                for (int rt = 0; rt < mtiles; rt++) {
                    const int i0 = 16 * rt;
                    if (i0 >= k0 && i0 + 16 <= k0 + kb) continue;  // the whole row tile is in K
                    double ar[8], ai[8], cr[4], ci[4];
#pragma unroll
                    for (int q = 0; q < 8; q++) {
                        const int r = i0 + g + 8 * (q & 1), c = t4 + 4 * (q >> 1);
                        zc v = (r < N && c < kb) ? M[bix<GM>(r, k0 + c, N)] : zc{0, 0};
                        ar[q] = v.x;
                        ai[q] = v.y;
                    }
                    bool own[4];
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const int r = i0 + g + 8 * (q >> 1), c = j0 + 2 * t4 + (q & 1);
                        own[q] = r < N && c < N && (r < k0 || r >= k0 + kb) && (c < k0 || c >= k0 + kb);
                        zc v = own[q] ? M[bix<GM>(r, c, N)] : zc{0, 0};
                        cr[q] = v.x;
                        ci[q] = v.y;
                    }
                    zmma16816(cr, ci, ar, ai, br, bi);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const int r = i0 + g + 8 * (q >> 1), c = j0 + 2 * t4 + (q & 1);
                        if (own[q]) M[bix<GM>(r, c, N)] = zc{cr[q], ci[q]};
                    }
                }
                // the pivot rows
                double ar[8], ai[8], cr[4] = {0, 0, 0, 0}, ci[4] = {0, 0, 0, 0};
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const int r = g + 8 * (q & 1), c = t4 + 4 * (q >> 1);
                    zc v = (r < kb && c < kb) ? M[bix<GM>(k0 + r, k0 + c, N)] : zc{0, 0};
                    ar[q] = v.x;
                    ai[q] = v.y;
                }
                zmma16816(cr, ci, ar, ai, br, bi);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int r = g + 8 * (q >> 1), c = j0 + 2 * t4 + (q & 1);
                    if (r < kb && c < N && (c < k0 || c >= k0 + kb)) M[bix<GM>(k0 + r, c, N)] = zc{cr[q], ci[q]};
                }
            }
            __syncthreads();
        }
        // undo the row interchanges by column interchanges in reverse order
        if (tid < N) {
            for (int k = N - 1; k >= 0; k--) {
                int p = perm[k];
                if (p != k) {
                    zc tt = M[bix<GM>(tid, k, N)];
                    M[bix<GM>(tid, k, N)] = M[bix<GM>(tid, p, N)];
                    M[bix<GM>(tid, p, N)] = tt;
                }
            }
        }
        __syncthreads();
        if (first_zero_s && tid == 0) {
            atomicMin(a.info, iw + 1);
            if (a.info_each) a.info_each[iw - a.iw0] = first_zero_s;
        }
        if (a.out_mode == 0) {
            const int nA = a.nA;
            zc *G = a.Gout + (size_t)iw * nA * nA;
            for (int idx = tid; idx < nA * nA; idx += nthr) {
                int p = idx % nA, q = idx / nA;
                G[idx] = M[bix<GM>(a.act[p], a.act[q], N)];
            }
        } else {
            zc *G = a.Gout + (size_t)(iw - a.iw0) * N * N;
            for (int idx = tid; idx < N * N; idx += nthr) G[idx] = M[bix<GM>(idx % N, idx / N, N)];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------
// Block-level complex GEMM C(MxN) = A(MxK) B(KxN) over 32x32 output tiles, 256 threads,
// each thread 2x2 outputs. Operands come from loader functors; the store functor gets
// (i, j, value). With `upper`, tiles strictly below the diagonal are skipped.
// ---------------------------------------------------------------------------------
constexpr int TB = 32, TK = 16;

template <class LA, class LB, class ST>
__device__ void cta_gemm(int M, int N, int K, LA la, LB lb, ST st, zc *sA, zc *sB, bool upper) {
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int mt = (M + TB - 1) / TB, nt = (N + TB - 1) / TB;
    for (int tile = 0; tile < mt * nt; tile++) {
        const int bi = tile % mt, bj = tile / mt;
        if (upper && bi > bj) continue;
        zc acc[2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};
        for (int k0 = 0; k0 < K; k0 += TK) {
            // sA[kk][r] (TK x TB), sB[kk][c] (TK x TB)
            for (int idx = tid; idx < TB * TK; idx += 256) {
                int r = idx % TB, kk = idx / TB;
                int i = bi * TB + r, k = k0 + kk;
                sA[kk * TB + r] = (i < M && k < K) ? la(i, k) : zc{0, 0};
            }
            for (int idx = tid; idx < TB * TK; idx += 256) {
                int kk = idx % TK, c = idx / TK;
                int j = bj * TB + c, k = k0 + kk;
                sB[kk * TB + c] = (j < N && k < K) ? lb(k, j) : zc{0, 0};
            }
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < TK; kk++) {
                zc a0 = sA[kk * TB + ty], a1 = sA[kk * TB + ty + 16];
                zc b0 = sB[kk * TB + tx], b1 = sB[kk * TB + tx + 16];
                cfma(acc[0][0], a0, b0);
                cfma(acc[0][1], a0, b1);
                cfma(acc[1][0], a1, b0);
                cfma(acc[1][1], a1, b1);
            }
            __syncthreads();
        }
#pragma unroll
        for (int r = 0; r < 2; r++)
#pragma unroll
            for (int c = 0; c < 2; c++) {
                int i = bi * TB + ty + 16 * r, j = bj * TB + tx + 16 * c;
                if (i < M && j < N) st(i, j, acc[r][c]);
            }
    }
}

// modes M_INIT2 / M_SCF2: T = G^r SL, G^< = T G^r^dagger (upper triangle), packed.
__global__ void __launch_bounds__(256) keldysh_scf2(KeldyshArgs a) {
    __shared__ zc sA[TB * TK], sB[TB * TK];
    const int nA = a.nA, nfull = nA * nA;
    zc *T = a.Tws + (size_t)blockIdx.x * nfull;
    for (int iw = blockIdx.x; iw < a.n; iw += gridDim.x) {
        const zc *G = a.G + (size_t)iw * nfull;
        const double w = a.omega[iw];
        const double fL = fermi_d(w, a.V, a.mu, a.beta), fR = fermi_d(w, 0.0, a.mu, a.beta);
        const zc *SL2 = a.SigL ? a.SigL + (size_t)iw * nfull : nullptr;
        // SL = i (fL GamL_s + fR GamR_s) / hbar  (+ Sigma2^<)   (src/scf.f90:333-336)
        auto ldSL = [&](int k, int j) {
            size_t idx = k + (size_t)j * nA;
            zc g{fL * a.GamLs[idx].x + fR * a.GamRs[idx].x, fL * a.GamLs[idx].y + fR * a.GamRs[idx].y};
            zc s{-g.y, g.x};
            if (SL2) s = s + SL2[idx];
            return s;
        };
        cta_gemm(
            nA, nA, nA, [&](int i, int k) { return G[i + (size_t)k * nA]; }, ldSL,
            [&](int i, int j, zc v) { T[i + (size_t)j * nA] = v; }, sA, sB, false);
        __syncthreads();
        double *blk = a.out + (size_t)iw * a.nblk;
        const double *xb = a.xsub ? a.xsub + (size_t)iw * a.nblk : nullptr;
        const int64_t offL = 2 * (int64_t)nfull, offD = offL + (int64_t)nA * (nA - 1);
        cta_gemm(
            nA, nA, nA, [&](int i, int k) { return T[i + (size_t)k * nA]; },
            [&](int k, int j) { return conj(G[j + (size_t)k * nA]); },
            [&](int i, int j, zc v) {
                if (i < j) {
                    int64_t o = offL + 2 * ((int64_t)j * (j - 1) / 2 + i);
                    blk[o] = xb ? v.x - xb[o] : v.x;
                    blk[o + 1] = xb ? v.y - xb[o + 1] : v.y;
                } else if (i == j) {
                    blk[offD + i] = xb ? v.y - xb[offD + i] : v.y;
                    if (a.gLd) a.gLd[(size_t)iw * nA + i] = v;
                }
            },
            sA, sB, true);
        // G^r part of the block
        for (int idx = threadIdx.x; idx < nfull; idx += blockDim.x) {
            zc g = G[idx];
            blk[2 * idx] = xb ? g.x - xb[2 * idx] : g.x;
            blk[2 * idx + 1] = xb ? g.y - xb[2 * idx + 1] : g.y;
            int i = idx % nA, j = idx / nA;
            if (i == j && a.gRd) a.gRd[(size_t)iw * nA + i] = g;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------
// The same step on the FP64 tensor cores for 48 <= nA <= 128: T = G^r SL and the upper
// triangle of G^< = T G^r^dagger as complex m16n8k16 MMAs (4 real MMAs per complex tile),
// operands padded to 128 and staged through shared memory in 16-wide k panels by cp.async,
// double-buffered. 8 warps, one block per SM walking the energies; a warp owns a 32-row
// block of 8-column tiles. SL and T go through two scratch matrices of the block (L2).
// ---------------------------------------------------------------------------------
constexpr int KD_MP = 128, KD_LDA = 130, KD_LDN = 20;  // padded order; [k][m] / [n][k] panel strides
constexpr int KD_ASZ = 16 * KD_LDA, KD_BSZ = KD_MP * KD_LDN, KD_STAGE = KD_ASZ + KD_BSZ;
constexpr size_t KD_SMEM = 2 * KD_STAGE * sizeof(zc);

__device__ __forceinline__ void cpa16(void *dst, const void *src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 16 : 0) : "memory");
}

// C(m0 + 0..31, n0 + 0..8NT-1) = A B over k < nA. A: nA x nA column-major; B(k, n) =
// Bm[k + n nA], staged [n][k]; only columns nlo..nhi-1 of B are staged. Every thread of the
// block calls it (the panel copies); warps with !active skip the MMAs, and tiles beyond nA
// are skipped (warp-uniform).
template <int NT>
__device__ __forceinline__ void kd_gemm(const zc *__restrict__ A, const zc *__restrict__ Bm, int nA, int nlo, int nhi,
                                        int m0, int n0, bool active, zc *sm, double (&cr)[2][NT][4],
                                        double (&ci)[2][NT][4]) {
    const int tid = threadIdx.x, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
    const int nk = (nA + 15) / 16, nw = nhi - nlo;
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < NT; ni++)
#pragma unroll
            for (int q = 0; q < 4; q++) cr[mi][ni][q] = ci[mi][ni][q] = 0.0;
    auto load = [&](int kc, int st) {
        zc *As = sm + st * KD_STAGE, *Bs = As + KD_ASZ;
        const int k0 = kc * 16;
        for (int idx = tid; idx < 16 * KD_MP; idx += blockDim.x) {
            const int m = idx & (KD_MP - 1), kk = idx >> 7;
            const bool v = m < nA && k0 + kk < nA;
            cpa16(&As[kk * KD_LDA + m], v ? A + m + (size_t)(k0 + kk) * nA : A, v);
        }
        for (int idx = tid; idx < 16 * nw; idx += blockDim.x) {
            const int kk = idx & 15, nn = nlo + (idx >> 4);
            const bool v = nn < nA && k0 + kk < nA;
            cpa16(&Bs[nn * KD_LDN + kk], v ? Bm + (k0 + kk) + (size_t)nn * nA : Bm, v);
        }
    };
    load(0, 0);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    for (int kc = 0; kc < nk; kc++) {
        if (kc + 1 < nk) load(kc + 1, (kc + 1) & 1);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        __syncthreads();
        if (active) {
            const zc *As = sm + (kc & 1) * KD_STAGE, *Bs = As + KD_ASZ;
            double ar[2][8], ai[2][8];
#pragma unroll
            for (int mi = 0; mi < 2; mi++)
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const zc v = As[(t4 + 4 * (q >> 1)) * KD_LDA + m0 + 16 * mi + g + 8 * (q & 1)];
                    ar[mi][q] = v.x;
                    ai[mi][q] = v.y;
                }
#pragma unroll
            for (int ni = 0; ni < NT; ni++) {
                const int c0 = n0 + 8 * ni;
                if (c0 >= nA) continue;
                const bool t0 = m0 < nA, t1 = m0 + 16 < nA;
                if (!t0 && !t1) continue;
                double br[4], bi[4], nbi[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const zc v = Bs[(c0 + g) * KD_LDN + t4 + 4 * q];
                    br[q] = v.x;
                    bi[q] = v.y;
                    nbi[q] = -v.y;
                }
                if (t0 && t1) {  // the two row tiles interleaved: dependent MMAs are three apart
                    dmma16816(cr[0][ni], ar[0], br);
                    dmma16816(cr[1][ni], ar[1], br);
                    dmma16816(ci[0][ni], ar[0], bi);
                    dmma16816(ci[1][ni], ar[1], bi);
                    dmma16816(cr[0][ni], ai[0], nbi);
                    dmma16816(cr[1][ni], ai[1], nbi);
                    dmma16816(ci[0][ni], ai[0], br);
                    dmma16816(ci[1][ni], ai[1], br);
                } else if (t0) {
                    dmma16816(cr[0][ni], ar[0], br);
                    dmma16816(ci[0][ni], ar[0], bi);
                    dmma16816(cr[0][ni], ai[0], nbi);
                    dmma16816(ci[0][ni], ai[0], br);
                } else {
                    dmma16816(cr[1][ni], ar[1], br);
                    dmma16816(ci[1][ni], ar[1], bi);
                    dmma16816(cr[1][ni], ai[1], nbi);
                    dmma16816(ci[1][ni], ai[1], br);
                }
            }
        }
        __syncthreads();  // the stage is refilled two chunks later
    }
}

// The upper triangle of G^< = T G^dagger as a list of 16 x 8 tiles (row tile rt, column
// tile ct with 16 rt <= 8 ct + 7, inside nA): pass p gives warp w the tiles p*64 + 8 s + w,
// s < 8, so the warps share every pass evenly. Operand panels as in kd_gemm (B conjugate-
// transposed from G); put(i, j, re, im) receives every element of the warp's tiles.
constexpr int KD_SLOTS = 8;
constexpr int KD_NCMAX = 16;  // contact states up to which the lead term is a low-rank correction
__device__ __forceinline__ int kd_upper_tiles(int nA) {
    int cnt = 0;
    for (int ct = 0; 8 * ct < nA; ct++) cnt += min((8 * ct + 7) / 16 + 1, (nA + 15) / 16);
    return cnt;
}
// the t-th upper tile in column-major order of tiles
__device__ __forceinline__ void kd_upper_tile(int nA, int t, int &rt, int &ct) {
    for (ct = 0; 8 * ct < nA; ct++) {
        const int h = min((8 * ct + 7) / 16 + 1, (nA + 15) / 16);
        if (t < h) {
            rt = t;
            return;
        }
        t -= h;
    }
    rt = -1;
}

template <class PUT>
__device__ __forceinline__ void kd_upper_gemm(const zc *__restrict__ T, const zc *__restrict__ G, int nA, zc *sm,
                                              PUT put) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t4 = lane & 3;
    const int nk = (nA + 15) / 16, ntl = kd_upper_tiles(nA);
    for (int base = 0; base < ntl; base += 8 * KD_SLOTS) {
        int rts[KD_SLOTS], cts[KD_SLOTS];
#pragma unroll
        for (int q = 0; q < KD_SLOTS; q++) {
            const int t = base + 8 * q + warp;
            if (t < ntl) kd_upper_tile(nA, t, rts[q], cts[q]);
            else rts[q] = -1;
        }
        double cr[KD_SLOTS][4], ci[KD_SLOTS][4];
#pragma unroll
        for (int q = 0; q < KD_SLOTS; q++)
#pragma unroll
            for (int e = 0; e < 4; e++) cr[q][e] = ci[q][e] = 0.0;
        auto load = [&](int kc, int st) {
            zc *As = sm + st * KD_STAGE, *Bs = As + KD_ASZ;
            const int k0 = kc * 16;
            for (int idx = tid; idx < 16 * KD_MP; idx += blockDim.x) {
                const int m = idx & (KD_MP - 1), kk = idx >> 7;
                const bool v = m < nA && k0 + kk < nA;
                cpa16(&As[kk * KD_LDA + m], v ? T + m + (size_t)(k0 + kk) * nA : T, v);
                cpa16(&Bs[kk * KD_LDA + m], v ? G + m + (size_t)(k0 + kk) * nA : G, v);
            }
        };
        load(0, 0);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        for (int kc = 0; kc < nk; kc++) {
            if (kc + 1 < nk) load(kc + 1, (kc + 1) & 1);
            asm volatile("cp.async.commit_group;\n" ::: "memory");
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
            __syncthreads();
            const zc *As = sm + (kc & 1) * KD_STAGE, *Bs = As + KD_ASZ;
#pragma unroll
            for (int q = 0; q < KD_SLOTS; q++) {
                if (rts[q] < 0) continue;
                const int r0 = 16 * rts[q], c0 = 8 * cts[q];
                double ar[8], ai[8], br[4], bi[4], nbi[4];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const zc v = As[(t4 + 4 * (e >> 1)) * KD_LDA + r0 + g + 8 * (e & 1)];
                    ar[e] = v.x;
                    ai[e] = v.y;
                }
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const zc v = Bs[(t4 + 4 * e) * KD_LDA + c0 + g];  // B(k, n) = conj(G(n, k))
                    br[e] = v.x;
                    bi[e] = -v.y;
                    nbi[e] = v.y;
                }
                dmma16816(cr[q], ar, br);
                dmma16816(ci[q], ar, bi);
                dmma16816(cr[q], ai, nbi);
                dmma16816(ci[q], ai, br);
            }
            __syncthreads();  // the stage is refilled two chunks later
        }
#pragma unroll
        for (int q = 0; q < KD_SLOTS; q++) {
            if (rts[q] < 0) continue;
#pragma unroll
            for (int e = 0; e < 4; e++)
                put(16 * rts[q] + g + 8 * (e >> 1), 8 * cts[q] + 2 * t4 + (e & 1), cr[q][e], ci[q][e]);
        }
    }
}

__global__ void __launch_bounds__(256, 1) keldysh_tc(KeldyshArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    zc *sm = (zc *)smem_raw;
    const int nA = a.nA, nfull = nA * nA;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
    zc *T = a.Tws + (size_t)(2 * blockIdx.x) * nfull;
    zc *S = T + nfull;
    const int64_t offL = 2 * (int64_t)nfull, offD = offL + (int64_t)nA * (nA - 1);
    for (int iw = blockIdx.x; iw < a.n; iw += gridDim.x) {
        const zc *G = a.G + (size_t)iw * nfull;
        const double w = a.omega[iw];
        const double fL = fermi_d(w, a.V, a.mu, a.beta), fR = fermi_d(w, 0.0, a.mu, a.beta);
        const zc *SL2 = a.SigL ? a.SigL + (size_t)iw * nfull : nullptr;
        // SL = i (fL GamL_s + fR GamR_s) / hbar + Sigma2^<   (src/scf.f90:333-336). With
        // few contact states (the usual case) the first product takes Sigma2^< itself as
        // its B operand and the lead term is added to the contact columns of T afterwards
        // (a rank-nc correction); otherwise SL is built in the block's scratch (the loads
        // of 8 elements a thread issued before their stores).
        const bool lowrank = SL2 && a.nc >= 0 && a.nc <= KD_NCMAX;
        const zc *Bop = lowrank ? SL2 : S;
        for (int base = threadIdx.x; !lowrank && base < nfull; base += 8 * blockDim.x) {
            zc gl[8], gr[8], s2[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int idx = base + u * blockDim.x;
                const bool v = idx < nfull;
                gl[u] = v ? a.GamLs[idx] : zc{0, 0};
                gr[u] = v ? a.GamRs[idx] : zc{0, 0};
                s2[u] = (v && SL2) ? SL2[idx] : zc{0, 0};
            }
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int idx = base + u * blockDim.x;
                if (idx < nfull) S[idx] = zc{-(fL * gl[u].y + fR * gr[u].y) + s2[u].x, fL * gl[u].x + fR * gr[u].x + s2[u].y};
            }
        }
        __threadfence_block();
        __syncthreads();
        // T = G SL, in two column halves of 64
        for (int hh = 0; hh < 2; hh++) {
            if (64 * hh >= nA) break;
            double cr[2][4][4], ci[2][4][4];
            const int m0 = 32 * (warp & 3), n0 = 64 * hh + 32 * (warp >> 2);
            kd_gemm<4>(G, Bop, nA, 64 * hh, 64 * hh + 64, m0, n0, m0 < nA && n0 < nA, sm, cr, ci);
#pragma unroll
            for (int mi = 0; mi < 2; mi++)
#pragma unroll
                for (int ni = 0; ni < 4; ni++)
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const int r = m0 + 16 * mi + g + 8 * (q >> 1), c = n0 + 8 * ni + 2 * t4 + (q & 1);
                        if (r < nA && c < nA) T[r + (size_t)c * nA] = zc{cr[mi][ni][q], ci[mi][ni][q]};
                    }
        }
        __threadfence_block();
        __syncthreads();
        if (lowrank && a.nc > 0) {
            // T(r, b) += sum over contact states c of G(r, c) i (fL GamL_s + fR GamR_s)(c, b), b a contact state
            for (int t = threadIdx.x; t < nA * a.nc; t += blockDim.x) {
                const int r = t % nA, b = a.cidx[t / nA];
                zc acc = T[r + (size_t)b * nA];
                for (int q = 0; q < a.nc; q++) {
                    const int c = a.cidx[q];
                    const size_t cb = c + (size_t)b * nA;
                    const zc gl = a.GamLs[cb], gr = a.GamRs[cb];
                    cfma(acc, G[r + (size_t)c * nA], zc{-(fL * gl.y + fR * gr.y), fL * gl.x + fR * gr.x});
                }
                T[r + (size_t)b * nA] = acc;
            }
            __threadfence_block();
            __syncthreads();
        }
        double *blk = a.out + (size_t)iw * a.nblk;
        const double *xb = a.xsub ? a.xsub + (size_t)iw * a.nblk : nullptr;
        auto put = [&](int r, int c, double vr, double vi) {
            if (r >= nA || c >= nA || r > c) return;
            if (r < c) {
                const int64_t o = offL + 2 * ((int64_t)c * (c - 1) / 2 + r);
                blk[o] = xb ? vr - xb[o] : vr;
                blk[o + 1] = xb ? vi - xb[o + 1] : vi;
            } else {
                blk[offD + r] = xb ? vi - xb[offD + r] : vi;
                if (a.gLd) a.gLd[(size_t)iw * nA + r] = zc{vr, vi};
            }
        };
        // upper triangle of G^< = T G^dagger, 16 x 8 tiles shared evenly by the warps
        kd_upper_gemm(T, G, nA, sm, put);
        // G^r part of the block (8 elements a thread in flight)
        for (int base = threadIdx.x; base < nfull; base += 8 * blockDim.x) {
            zc gv[8];
            double xr[8], xi[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int idx = base + u * blockDim.x;
                const bool v = idx < nfull;
                gv[u] = v ? G[idx] : zc{0, 0};
                xr[u] = (v && xb) ? xb[2 * idx] : 0.0;
                xi[u] = (v && xb) ? xb[2 * idx + 1] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int idx = base + u * blockDim.x;
                if (idx < nfull) {
                    blk[2 * idx] = gv[u].x - xr[u];
                    blk[2 * idx + 1] = gv[u].y - xi[u];
                }
            }
        }
        if (a.gRd)
            for (int i = threadIdx.x; i < nA; i += blockDim.x) a.gRd[(size_t)iw * nA + i] = G[i + (size_t)i * nA];
        __syncthreads();  // S and T are rewritten for the next energy
    }
}

struct FinalArgs {
    int N, nS, nA, nCL, N_sites, N_atoms, iw0, iw1, mode;
    const zc *G;  // full G per energy of the chunk
    const int *sup, *act, *pos, *cl, *site_int, *atom_first, *atom_norb, *atom_off;
    const zc *GamLs, *GamRs, *GamLcl, *SigL;
    const double *omega;
    double V, mu, beta;
    zc *Tws;
    double *dosd, *trU, *trD;
    zc *onsL, *atomL, *gRd, *gLd;
    int atomL_ld;
};

// modes M_SCF1 and M_FINAL (src/scf.f90:357-410)
__global__ void __launch_bounds__(256) final_outputs(FinalArgs a) {
    __shared__ zc sA[TB * TK], sB[TB * TK];
    __shared__ zc Xs[32 * 32];  // nCL <= 32 (checked in qs_create)
    const int N = a.N, nS = a.nS;
    const bool fin = (a.mode == M_FINAL);
    const int Mrows = fin ? N : a.nA;
    zc *T = a.Tws + (size_t)blockIdx.x * Mrows * nS;
    for (int iw = a.iw0 + blockIdx.x; iw < a.iw1; iw += gridDim.x) {
        const zc *G = a.G + (size_t)(iw - a.iw0) * N * N;
        auto g = [&](int i, int j) { return G[i + (size_t)j * N]; };
        const double w = a.omega[iw];
        const double fL = fermi_d(w, a.V, a.mu, a.beta), fR = fermi_d(w, 0.0, a.mu, a.beta);
        const zc *SL2 = a.SigL ? a.SigL + (size_t)iw * a.nA * a.nA : nullptr;
        auto ldSL = [&](int k, int j) {
            size_t idx = k + (size_t)j * nS;
            zc gg{fL * a.GamLs[idx].x + fR * a.GamRs[idx].x, fL * a.GamLs[idx].y + fR * a.GamRs[idx].y};
            zc s{-gg.y, gg.x};
            if (SL2) s = s + SL2[idx];
            return s;
        };
        // T = w1(rows, sup) SL
        cta_gemm(
            Mrows, nS, nS, [&](int i, int k) { return g(fin ? i : a.act[i], a.sup[k]); }, ldSL,
            [&](int i, int j, zc v) { T[i + (size_t)j * Mrows] = v; }, sA, sB, false);
        __syncthreads();
        // sum_q T(r, q) conj(w1(c, sup(q)))
        auto blkv = [&](int r, int c) {
            zc acc{0, 0};
            for (int q = 0; q < nS; q++) cfma_conj(acc, T[r + (size_t)q * Mrows], g(c, a.sup[q]));
            return acc;
        };
        if (fin) {
            for (int i = threadIdx.x; i < N; i += blockDim.x) a.dosd[(size_t)iw * N + i] = g(i, i).y;
            for (int t = threadIdx.x; t < 4 * a.N_sites; t += blockDim.x) {
                int s = t >> 2, e = t & 3, aa = e & 1, bb = e >> 1;
                a.onsL[(size_t)iw * 4 * a.N_sites + t] = blkv(2 * s + aa, 2 * s + bb);
            }
            if (a.atomL) {
                for (int at = 0; at < a.N_atoms; at++) {
                    int lo = 2 * (a.atom_first[at] - 1), m = 2 * a.atom_norb[at];
                    for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
                        int aa = t % m, bb = t / m;
                        a.atomL[(size_t)iw * a.atomL_ld + a.atom_off[at] + t] = blkv(lo + aa, lo + bb);
                    }
                }
            }
            // current integrand through the left lead (src/scf.f90:390-409)
            const int nCL = a.nCL;
            for (int t = threadIdx.x; t < nCL * nCL; t += blockDim.x) {
                int k = t % nCL, aa = t / nCL;
                int ck = a.cl[k], ca = a.cl[aa];
                zc glc = blkv(ck, ca);
                zc gka = g(ck, ca), gak = conj(g(ca, ck));
                zc gg = glc + gka - gak;
                Xs[t] = zc{(fL - 1.0) * glc.x - fL * gg.x, (fL - 1.0) * glc.y - fL * gg.y};
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                zc tu{0, 0}, td{0, 0};
                for (int aa = 0; aa < nCL; aa++) {
                    zc mc{0, 0};
                    for (int k = 0; k < nCL; k++) cfma(mc, a.GamLcl[aa + (size_t)k * nCL], Xs[k + (size_t)aa * nCL]);
                    mc = zc{-mc.y, mc.x};
                    if ((a.cl[aa] & 1) == 0) tu = tu + mc;  // 0-based even = spin up
                    else td = td + mc;
                }
                a.trU[iw] = tu.x / (2.0 * PI);
                a.trD[iw] = td.x / (2.0 * PI);
            }
        } else {
            for (int k = threadIdx.x; k < a.nA; k += blockDim.x) {
                int ak = a.act[k];
                a.gRd[(size_t)iw * a.nA + k] = g(ak, ak);
                a.gLd[(size_t)iw * a.nA + k] = blkv(k, ak);
            }
            for (int t = threadIdx.x; t < 4 * a.N_sites; t += blockDim.x) {
                int s = t >> 2, e = t & 3, aa = e & 1, bb = e >> 1;
                if (!a.site_int[s]) continue;
                int lo = 2 * s, p1 = a.pos[lo];
                a.onsL[(size_t)iw * 4 * a.N_sites + t] = blkv(p1 + aa, lo + bb);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------
// Reductions over energies: out[c] = sum_r A[r*ld + c], deterministic.
// ---------------------------------------------------------------------------------
template <typename V>
__global__ void colsum(const V *__restrict__ A, int64_t ld, int ncols, int64_t nrows, V *__restrict__ out) {
    __shared__ V part[8][32];
    const int c = blockIdx.x * 32 + (threadIdx.x & 31), lane = threadIdx.x >> 5;
    V acc{};
    if (c < ncols)
        for (int64_t r = lane; r < nrows; r += 8) {
            V v = A[r * ld + c];
            acc = acc + v;
        }
    part[lane][threadIdx.x & 31] = acc;
    __syncthreads();
    if (lane == 0 && c < ncols) {
        V s = part[0][threadIdx.x];
        for (int l = 1; l < 8; l++) s = s + part[l][threadIdx.x];
        out[c] = s;
    }
}

int sum_over_energies(qs_handle *h, const zc *d_A, int64_t ld, int ncols, int64_t nrows, zc *d_out) {
    if (ncols <= 0) return 0;
    int pi = prof_begin(h, K_REDUCE);
    colsum<zc><<<(ncols + 31) / 32, 256, 0, h->stream>>>(d_A, ld, ncols, nrows, d_out);
    prof_end(h, pi);
    QS_CUDA(h, cudaGetLastError());
    return 0;
}
int sum_over_energies_real(qs_handle *h, const double *d_A, int64_t ld, int ncols, int64_t nrows, double *d_out) {
    if (ncols <= 0) return 0;
    int pi = prof_begin(h, K_REDUCE);
    colsum<double><<<(ncols + 31) / 32, 256, 0, h->stream>>>(d_A, ld, ncols, nrows, d_out);
    prof_end(h, pi);
    QS_CUDA(h, cudaGetLastError());
    return 0;
}

// ---------------------------------------------------------------------------------
// pack_gf layout <-> device layout (per energy block of 3 nA^2 doubles)
//   reference (common/linear_algebra.f90:155-191): Re G^r (row-major i,j) | Im G^r |
//     Re G^< strict upper (row-major, j > i) | Im G^< upper (row-major, j >= i)
// ---------------------------------------------------------------------------------
__global__ void ref_dl_perm(int nA, int64_t Nw, const double *__restrict__ src, double *__restrict__ dst, int to_dl) {
    const int64_t nblk = 3 * (int64_t)nA * nA;
    const int nfull = nA * nA, nsu = (nfull - nA) / 2;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < Nw * nblk; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t w = t / nblk;
        int e = (int)(t - w * nblk);
        // e indexes the reference block; compute its device position
        int64_t dpos;
        if (e < 2 * nfull) {
            int part = e / nfull, r = e % nfull;  // r = i*nA + j
            int i = r / nA, j = r % nA;
            dpos = 2 * ((int64_t)i + (int64_t)j * nA) + part;
        } else if (e < 2 * nfull + nsu) {
            int r = e - 2 * nfull;  // r-th strict-upper element in row-major order
            // row i holds nA-1-i elements
            int i = 0, acc = 0;
            while (acc + (nA - 1 - i) <= r) { acc += nA - 1 - i; i++; }
            int j = i + 1 + (r - acc);
            dpos = 2 * (int64_t)nfull + 2 * ((int64_t)j * (j - 1) / 2 + i);
        } else {
            int r = e - 2 * nfull - nsu;  // r-th upper element (j >= i), row-major
            int i = 0, acc = 0;
            while (acc + (nA - i) <= r) { acc += nA - i; i++; }
            int j = i + (r - acc);
            if (i == j) dpos = 2 * (int64_t)nfull + (int64_t)nA * (nA - 1) + i;
            else dpos = 2 * (int64_t)nfull + 2 * ((int64_t)j * (j - 1) / 2 + i) + 1;
        }
        if (to_dl) dst[w * nblk + dpos] = src[t];
        else dst[t] = src[w * nblk + dpos];
    }
}

int convert_ref_to_dl(cudaStream_t st, int nA, int64_t Nw, const double *ref, double *dl) {
    count_launch();
    ref_dl_perm<<<1184, 256, 0, st>>>(nA, Nw, ref, dl, 1);
    return (int)cudaGetLastError();
}
int convert_dl_to_ref(cudaStream_t st, int nA, int64_t Nw, const double *dl, double *ref) {
    count_launch();
    ref_dl_perm<<<1184, 256, 0, st>>>(nA, Nw, dl, ref, 0);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------------
static int dyson_threads(int N) { return N <= 128 ? (N <= 64 ? 256 : 512) : 512; }
static size_t dyson_smem(int N) { return sizeof(zc) * (size_t)N * N; }
static bool dyson_fits(int N) { return dyson_fits_smem(N); }

static bool use_blocked(int N) { return N >= 16 && N <= 128 && (size_t)swz_units(N) * 16 + 1536 <= (size_t)SMEM_MAX; }
// the blocked kernel with the matrix in the global workspace: orders above the shared-memory
// limit up to 256
static bool use_blocked_gm(int N) { return !use_blocked(N) && N > 16 && N <= BGJ_MAXN_GM; }
static inline auto dyson_bgj = dyson_bgj_t<false>;
constexpr int BGJ_THREADS2 = 256;  // the two-blocks-per-SM form (workspace)
// the workspace form runs for 16 < N <= 256 (also below the shared-memory limit, as the
// two-blocks-per-SM variant of the tuner)
static bool use_bgj_ws(int N) { return N > 16 && N <= BGJ_MAXN_GM; }

static int launch_dyson(qs_handle *h, DysonArgs &a, int nblocks, int variant) {
    const int N = a.N;
    if (variant == DYSON_BLOCKED2 && use_bgj_ws(N) && h->d_Gws) {
        // two blocks of 8 warps per SM, each matrix in its block's slot of the workspace
        a.ws = h->d_Gws;
        nblocks = std::min<int>(std::min(nblocks, 2 * 148), (int)h->ws_slots);
        int pi = prof_begin(h, K_DYSON);
        dyson_bgj_t<true, BGJ_THREADS2><<<nblocks, BGJ_THREADS2, 0, h->stream>>>(a);
        prof_end(h, pi);
        QS_CUDA(h, cudaGetLastError());
        return 0;
    }
    if (variant == DYSON_BLOCKED && use_blocked_gm(N) && h->d_Gws) {
        // one block per SM: the concurrent matrices (148 x N^2 x 16 B) stay mostly in L2
        a.ws = h->d_Gws;
        nblocks = std::min<int>(std::min(nblocks, 148), (int)h->ws_slots);
        int pi = prof_begin(h, K_DYSON);
        dyson_bgj_t<true><<<nblocks, BGJ_THREADS, 0, h->stream>>>(a);
        prof_end(h, pi);
        QS_CUDA(h, cudaGetLastError());
        return 0;
    }
    if (variant == DYSON_BLOCKED && use_blocked(N)) {
        size_t sm = (size_t)swz_units(N) * sizeof(zc);
        QS_CUDA(h, smem_cap((const void *)dyson_bgj));
        a.ws = nullptr;
        int pi = prof_begin(h, K_DYSON);
        dyson_bgj<<<nblocks, BGJ_THREADS, sm, h->stream>>>(a);
        prof_end(h, pi);
        QS_CUDA(h, cudaGetLastError());
        return 0;
    }
    int thr = dyson_threads(N);
    size_t sm = 0;
    if (dyson_fits(N)) {
        sm = dyson_smem(N);
        QS_CUDA(h, smem_cap((const void *)dyson_gj));
        a.ws = nullptr;
    } else {
        nblocks = std::min<int>(nblocks, (int)h->ws_slots);
        a.ws = h->d_Gws;
    }
    int pi = prof_begin(h, K_DYSON);
    dyson_gj<<<nblocks, thr, sm, h->stream>>>(a);
    prof_end(h, pi);
    QS_CUDA(h, cudaGetLastError());
    return 0;
}

int invert_batched_dev(cudaStream_t st, int N, int batch, zc *d_A, int *d_info, zc *d_ws, int ws_slots) {
    DysonArgs a{};
    a.N = N;
    a.iw0 = 0;
    a.iw1 = batch;
    a.Ain = d_A;
    a.out_mode = 1;
    a.Gout = d_A;
    a.info = d_info;
    a.info_each = d_info + 1;
    int thr = dyson_threads(N);
    int nb = std::min(batch, 148 * 8);
    size_t sm = 0;
    if (use_blocked(N)) {
        sm = (size_t)swz_units(N) * sizeof(zc);
        cudaError_t e = smem_cap((const void *)dyson_bgj);
        if (e != cudaSuccess) return -(int)e;
        count_launch();
        dyson_bgj<<<nb, BGJ_THREADS, sm, st>>>(a);
        e = cudaGetLastError();
        return e == cudaSuccess ? 0 : -(int)e;
    }
    if (use_blocked_gm(N) && d_ws && ws_slots > 0) {
        a.ws = d_ws;
        nb = std::min(std::min(nb, 148), ws_slots);
        count_launch();
        dyson_bgj_t<true><<<nb, BGJ_THREADS, 0, st>>>(a);
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? 0 : -(int)e;
    }
    if (dyson_fits(N)) {
        sm = dyson_smem(N);
        cudaError_t e = smem_cap((const void *)dyson_gj);
        if (e != cudaSuccess) return -(int)e;
    } else {
        a.ws = d_ws;
        nb = std::min(nb, ws_slots);
    }
    count_launch();
    dyson_gj<<<nb, thr, sm, st>>>(a);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : -(int)e;
}

// Batched inversion with every matrix in the given global workspace (ws_slots matrices
// of N x N complex, reused round-robin by the blocks), whatever N is.
int invert_batched_ws(cudaStream_t st, int N, int batch, zc *d_A, int *d_min_info, int *d_info_each, zc *d_ws,
                      int ws_slots) {
    DysonArgs a{};
    a.N = N;
    a.iw0 = 0;
    a.iw1 = batch;
    a.Ain = d_A;
    a.out_mode = 1;
    a.Gout = d_A;
    a.info = d_min_info;
    a.info_each = d_info_each;
    a.ws = d_ws;
    int nb = std::min(std::min(batch, 148 * 8), ws_slots);
    if (nb < 1) return -1;
    count_launch();
    dyson_gj<<<nb, dyson_threads(N), 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : -(int)e;
}

// sweep(mode) over all energies (src/scf.f90:280-290).
//   M_INIT2 / M_SCF2: output into d_out (SCF vector, DL); M_SCF2 subtracts d_x.
//   M_SCF1 / M_FINAL: per-energy arrays of the handle.
int sweep(qs_handle *h, int mode, double V, bool use_sigma, double *d_out, const double *d_x, bool fp32) {
    const int N = h->Norb, nA = h->nA, n = h->n;
    DysonArgs a{};
    a.N = N;
    a.nA = nA;
    a.Hemb = h->d_Hemb;
    a.Sig1 = h->d_Sig1;
    a.SigR = h->d_SigR;
    a.pos = h->d_pos;
    a.act = h->d_act;
    a.omega = h->d_omega;
    a.use_sigma = use_sigma;
    a.order2 = (h->order == 2);
    a.info = h->d_info;
    int rc;
    if (mode == M_INIT2 || mode == M_SCF2) {
        a.iw0 = 0;
        a.iw1 = n;
        a.out_mode = 0;
        a.Gout = h->d_G;
        {
            int cand[3], nc = 0;
            if (use_blocked(N) || (use_blocked_gm(N) && h->d_Gws)) cand[nc++] = DYSON_BLOCKED;
            if (use_bgj_ws(N) && h->d_Gws) cand[nc++] = DYSON_BLOCKED2;
            cand[nc++] = DYSON_UNBLOCKED;
            rc = tune_launch(h, TUNE_DYSON, tune_key(N, n), cand, nc, nc > 1 ? cand[0] : DYSON_UNBLOCKED,
                             [&](int v) { return launch_dyson(h, a, std::min(n, 148 * 16), v); });
            if (rc) return rc;
        }
        KeldyshArgs k{};
        k.nA = nA;
        k.n = n;
        k.nblk = h->nblk;
        k.G = h->d_G;
        k.SigL = (use_sigma && h->order == 2) ? h->d_SigL : nullptr;
        k.GamLs = h->d_GamLs;
        k.GamRs = h->d_GamRs;
        k.omega = h->d_omega;
        k.V = V;
        k.mu = h->mu;
        k.beta = h->beta;
        k.out = d_out;
        k.xsub = (mode == M_SCF2) ? d_x : nullptr;
        k.gRd = h->d_gRd;
        k.gLd = h->d_gLd;
        k.Tws = h->d_T;
        k.err = h->d_info + 1;
        k.cidx = h->d_kd_cidx;
        k.nc = (h->nS == nA) ? h->kd_nc : -1;
        const int nb = (int)std::min<size_t>(h->T_slots, (size_t)n);
        const int nbt = std::min(n, 148);
        auto launch_k = [&](int v) -> int {
            int pi;
            if (v == KELDYSH_TF32) return launch_keldysh_tf32(h, k);
            if (v == KELDYSH_TC) {
                QS_CUDA(h, smem_cap((const void *)keldysh_tc));
                pi = prof_begin(h, K_KELDYSH);
                keldysh_tc<<<nbt, 256, KD_SMEM, h->stream>>>(k);
            } else {
                pi = prof_begin(h, K_KELDYSH);
                keldysh_scf2<<<nb, 256, 0, h->stream>>>(k);
            }
            prof_end(h, pi);
            QS_CUDA(h, cudaGetLastError());
            return 0;
        };
        const bool tc_ok = nA >= 32 && nA <= KD_MP && h->T_slots >= (size_t)(2 * nbt);
        const int fallback = (tc_ok && nA >= 48) ? KELDYSH_TC : KELDYSH_CUDA;
        // the FP32 phase of a QS_PREC_MIXED solve: the 3xTF32 kernel on the fifth-generation
        // tensor cores is a candidate too, kept only where it is the fastest
        if (fp32 && mode == M_SCF2 && keldysh_tf32_fits(nA)) {
            int c3[3], nc = 0;
            c3[nc++] = KELDYSH_TF32;
            if (tc_ok) c3[nc++] = KELDYSH_TC;
            c3[nc++] = KELDYSH_CUDA;
            return tune_launch(h, TUNE_KELDYSH32, tune_key(nA, n), c3, nc, fallback, launch_k);
        }
        const int cand[2] = {KELDYSH_TC, KELDYSH_CUDA};
        return tune_launch(h, TUNE_KELDYSH, tune_key(nA, n), tc_ok ? cand : cand + 1, tc_ok ? 2 : 1, fallback,
                           launch_k);
    }
    // chunked full inversion + per-energy outputs
    const int Mrows = (mode == M_FINAL) ? N : nA;
    for (int iw0 = 0; iw0 < n; iw0 += (int)h->G_chunk) {
        int iw1 = std::min(n, iw0 + (int)h->G_chunk);
        a.iw0 = iw0;
        a.iw1 = iw1;
        a.out_mode = 1;
        a.Gout = h->d_G;
        if ((rc = launch_dyson(h, a, std::min(iw1 - iw0, 148 * 16), DYSON_BLOCKED))) return rc;
        FinalArgs f{};
        f.N = N;
        f.nS = h->nS;
        f.nA = nA;
        f.nCL = h->nCL;
        f.N_sites = h->N_sites;
        f.N_atoms = h->N_atoms;
        f.iw0 = iw0;
        f.iw1 = iw1;
        f.mode = mode;
        f.G = h->d_G;
        f.sup = h->d_sup;
        f.act = h->d_act;
        f.pos = h->d_pos;
        f.cl = h->d_cl;
        f.site_int = h->d_site_int;
        f.atom_first = h->d_atom_first;
        f.atom_norb = h->d_atom_norb;
        f.atom_off = h->d_atom_off;
        f.GamLs = h->d_GamLs;
        f.GamRs = h->d_GamRs;
        f.GamLcl = h->d_GamLcl;
        f.SigL = (use_sigma && h->order == 2) ? h->d_SigL : nullptr;
        f.omega = h->d_omega;
        f.V = V;
        f.mu = h->mu;
        f.beta = h->beta;
        f.Tws = h->d_T;
        f.dosd = h->d_dosd;
        f.trU = h->d_trU;
        f.trD = h->d_trD;
        f.onsL = h->d_onsL;
        f.atomL = h->has_atomL ? h->d_atomL : nullptr;
        f.atomL_ld = h->has_atomL ? h->atom_off.back() : 0;
        f.gRd = h->d_gRd;
        f.gLd = h->d_gLd;
        size_t per = (size_t)Mrows * h->nS;
        int nb = (int)std::min<size_t>(std::min<size_t>(h->T_bytes / (sizeof(zc) * std::max<size_t>(per, 1)), 148 * 8),
                                       (size_t)(iw1 - iw0));
        nb = std::max(nb, 1);
        int pi = prof_begin(h, K_FINAL);
        final_outputs<<<nb, 256, 0, h->stream>>>(f);
        prof_end(h, pi);
        QS_CUDA(h, cudaGetLastError());
    }
    return 0;
}

}  // namespace qs
