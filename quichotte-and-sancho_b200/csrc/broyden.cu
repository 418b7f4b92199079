// broyden.cu -- modified Broyden mixing (D.D. Johnson, PRB 38, 12807 (1988)) on device
// vectors: broyden_solve (common/broyden_mixing.f90:51-184) with its history in HBM.
//
// Every O(n) step is an FP64 device reduction or update; the host sees only the scalars
// it needs each step (max|F|, rms|F|, ||dF||, the nh x nh Gram column and dF^T F) and
// solves the nh x nh system (nh <= nhist) as the reference's dposv does. One pass of
// hist_update writes the new history column pair AND accumulates its Gram column and
// dF^T F against the whole history, so each history column is read once per step for the
// dots and once for the x update.
//
// x, xold, F, Fold are rotated by pointer swaps instead of the reference's copies
// (xold = x, Fold = F), so the state after a step is the reference's.
#include <algorithm>
#include <cmath>

#include "qs_common.cuh"

namespace qs {

constexpr int RED_BLOCKS = 1184;  // 148 SMs x 8
constexpr int RED_THREADS = 256;
constexpr int MAXH = 32;           // largest history length handled by the fused kernels

static int red_blocks(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>(RED_BLOCKS, (n + RED_THREADS - 1) / RED_THREADS)); }

// block reduction of NV doubles (sum), result in lane 0 of warp 0 via shared memory
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *sh /* [NV][RED_THREADS/32] */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[k * 32 + wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double x = threadIdx.x < nw ? sh[k * 32 + threadIdx.x] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            v[k] = x;
        }
    }
    __syncthreads();
}

// partials[b] = (max |F|, sum F^2, sum (F-Fold)^2)
__global__ void __launch_bounds__(256) vec_norms(const double *__restrict__ F, const double *__restrict__ Fold, int64_t n,
                                                 double *__restrict__ part) {
    __shared__ double sh[3 * 32];
    double mx = 0.0, v[2] = {0.0, 0.0};
    const int64_t n2 = n / 2;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n2; q += stride) {
        double2 f = *(const double2 *)(F + 2 * q);
        mx = fmax(mx, fmax(fabs(f.x), fabs(f.y)));
        v[0] = fma(f.x, f.x, v[0]);
        v[0] = fma(f.y, f.y, v[0]);
        if (Fold) {
            double2 o = *(const double2 *)(Fold + 2 * q);
            double d0 = f.x - o.x, d1 = f.y - o.y;
            v[1] = fma(d0, d0, v[1]);
            v[1] = fma(d1, d1, v[1]);
        }
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        double f = F[n - 1];
        mx = fmax(mx, fabs(f));
        v[0] = fma(f, f, v[0]);
        if (Fold) {
            double d = f - Fold[n - 1];
            v[1] = fma(d, d, v[1]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) sh[64 + (threadIdx.x >> 5)] = mx;
    block_sum<2>(v, sh);
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmax(m, sh[64 + w]);
        part[3 * blockIdx.x + 0] = m;
        part[3 * blockIdx.x + 1] = v[0];
        part[3 * blockIdx.x + 2] = v[1];
    }
}

// New history pair in slot `slot` plus the Gram column and dF^T F over nh <= NH columns
// (common/broyden_mixing.f90:103-138,150-156). Single-precision history stores
// real(dF/||dF||) and real(alpha dF/||dF|| + dx/||dF||); every dot accumulates in FP64.
// Each thread handles groups of 4 consecutive elements (vector loads); n % 4 elements at
// the end are handled one by one. History columns are ld = broyden_ld(n) elements apart (n
// rounded up to a multiple of 4), so every column starts on a 16-byte boundary.
template <typename HT> struct V4;
template <> struct V4<float> { using t = float4; };
template <> struct V4<double> { using t = double4; };

__device__ __forceinline__ double4 ld4(const double *p) {
    double2 a = *(const double2 *)p, b = *(const double2 *)(p + 2);
    return double4{a.x, a.y, b.x, b.y};
}
__device__ __forceinline__ void st4(double *p, double4 v) {
    *(double2 *)p = double2{v.x, v.y};
    *(double2 *)(p + 2) = double2{v.z, v.w};
}
template <typename HT> __device__ __forceinline__ void hld4(const HT *p, double (&o)[4]);
template <> __device__ __forceinline__ void hld4<float>(const float *p, double (&o)[4]) {
    float4 v = *(const float4 *)p;
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
template <> __device__ __forceinline__ void hld4<double>(const double *p, double (&o)[4]) {
    double4 v = ld4(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
template <typename HT> __device__ __forceinline__ void hst4(HT *p, const HT (&v)[4]);
template <> __device__ __forceinline__ void hst4<float>(float *p, const float (&v)[4]) {
    *(float4 *)p = float4{v[0], v[1], v[2], v[3]};
}
template <> __device__ __forceinline__ void hst4<double>(double *p, const double (&v)[4]) {
    st4(p, double4{v[0], v[1], v[2], v[3]});
}

template <typename HT>
__device__ __forceinline__ void hist_elem(double f, double fo, double xx, double xo, double fnorm, double rf, double alpha,
                                          HT &dnew, HT &unew) {
    double d = f - fo, dx = xx - xo;
    if (sizeof(HT) == 4) {
        dnew = (HT)(d * rf);
        unew = (HT)(alpha * d * rf + dx * rf);
    } else {  // double history: dF = (F - Fold)/fnorm, U = alpha dF + (x - xold)/fnorm
        double dd = d / fnorm;
        dnew = (HT)dd;
        unew = (HT)(alpha * dd + dx / fnorm);
    }
}

// Four elements per thread (16-byte accesses). The NH column loads of a step are issued
// together, before the dots that use them, so that a step keeps all its loads in flight;
// the 2 NH FP64 accumulators and those loads need more than 128 registers a thread for
// NH >= 8, so the long-history forms run one block of 8 warps per SM (still ~80 KB of loads
// in flight per SM, above what HBM latency asks for).
template <typename HT, int E> struct HV;
template <> struct HV<float, 4> { using t = float4; };
template <> struct HV<double, 4> { using t = double4; };
template <> struct HV<float, 2> { using t = float2; };
template <> struct HV<double, 2> { using t = double2; };
template <int E> __device__ __forceinline__ void ldE(const double *p, double (&o)[E]) {
    if constexpr (E == 4) {
        double4 v = ld4(p);
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    } else {
        double2 v = *(const double2 *)p;
        o[0] = v.x; o[1] = v.y;
    }
}
template <typename HT, int E> __device__ __forceinline__ void hldE(const HT *p, double (&o)[E]) {
    if constexpr (E == 4) {
        hld4<HT>(p, o);
    } else if constexpr (sizeof(HT) == 4) {
        float2 v = *(const float2 *)p;
        o[0] = v.x; o[1] = v.y;
    } else {
        double2 v = *(const double2 *)p;
        o[0] = v.x; o[1] = v.y;
    }
}
template <typename HT, int E> __device__ __forceinline__ void hstE(HT *p, const HT (&v)[E]) {
    if constexpr (E == 4) {
        hst4<HT>(p, v);
    } else if constexpr (sizeof(HT) == 4) {
        *(float2 *)p = float2{v[0], v[1]};
    } else {
        *(double2 *)p = double2{v[0], v[1]};
    }
}

template <typename HT, int NH, int E = 4>
__global__ void __launch_bounds__(256, NH >= 8 ? 1 : 2) hist_update(const double *__restrict__ F, const double *__restrict__ Fold,
                                                      const double *__restrict__ x, const double *__restrict__ xold,
                                                      int64_t n, int64_t ld, double fnorm, double alpha,
                                                      HT *__restrict__ dF, HT *__restrict__ U, int slot, int nh,
                                                      int store, double *__restrict__ part) {
    __shared__ double sh[2 * NH * 8];
    double g[NH], c[NH];
#pragma unroll
    for (int k = 0; k < NH; k++) { g[k] = 0.0; c[k] = 0.0; }
    const double rf = 1.0 / fnorm;
    const int64_t nE = n / E;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nE + (n - E * nE); q += stride) {
        const bool vec = q < nE;
        const int64_t i0 = vec ? E * q : E * nE + (q - nE);
        const int cnt = vec ? E : 1;
        double f[E], dn[E];
        HT dnew[E] = {}, unew[E];
        if (vec) {
            ldE<E>(F + i0, f);
        } else {
            f[0] = F[i0];
        }
        if (store) {
            double fo[E], xx[E], xo[E];
            if (vec) {
                ldE<E>(Fold + i0, fo);
                ldE<E>(x + i0, xx);
                ldE<E>(xold + i0, xo);
            } else {
                fo[0] = Fold[i0]; xx[0] = x[i0]; xo[0] = xold[i0];
            }
#pragma unroll
            for (int e = 0; e < E; e++)
                if (e < cnt) hist_elem<HT>(f[e], fo[e], xx[e], xo[e], fnorm, rf, alpha, dnew[e], unew[e]);
            if (vec) {
                hstE<HT, E>(dF + (int64_t)slot * ld + i0, dnew);
                hstE<HT, E>(U + (int64_t)slot * ld + i0, unew);
            } else {
                dF[(int64_t)slot * ld + i0] = dnew[0];
                U[(int64_t)slot * ld + i0] = unew[0];
            }
        }
#pragma unroll
        for (int e = 0; e < E; e++) dn[e] = (double)dnew[e];
        // all column loads of the step first (independent, in flight together; kept in the
        // history's own type until used), then the dots
        typename HV<HT, E>::t dk[NH];
#pragma unroll
        for (int k = 0; k < NH; k++) {
            if (k < nh && !(store && k == slot)) {
                if (vec) {
                    dk[k] = *(const typename HV<HT, E>::t *)(dF + (int64_t)k * ld + i0);
                } else {
                    HT *d = (HT *)&dk[k];
                    d[0] = dF[(int64_t)k * ld + i0];
                }
            }
        }
#pragma unroll
        for (int k = 0; k < NH; k++) {
            if (k < nh) {
                const HT *d = (const HT *)&dk[k];
#pragma unroll
                for (int e = 0; e < E; e++)
                    if (e < cnt) {
                        const double v = (store && k == slot) ? dn[e] : (double)d[e];
                        g[k] = fma(v, dn[e], g[k]);
                        c[k] = fma(v, f[e], c[k]);
                    }
            }
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NH; k++) {
        double a = g[k], b = c[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if (lane == 0) {
            sh[(2 * k) * 8 + wid] = a;
            sh[(2 * k + 1) * 8 + wid] = b;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 2 * nh; t += blockDim.x) {
        double s2 = 0.0;
        for (int w = 0; w < nw; w++) s2 += sh[t * 8 + w];
        part[(int64_t)blockIdx.x * 2 * MAXH + t] = s2;
    }
}

// The same step for long histories (NH = 16, 32) with the columns split over SPL = NH / 8
// adjacent threads: the threads of a group share their four elements (their F, Fold, x,
// xold loads are the same transactions) and each keeps the dots of 8 columns, so a thread
// needs 16 accumulators and 8 column loads, two 8-warp blocks fit on an SM, and each
// thread's loads of a step are all in flight together.
template <typename HT, int NH>
__global__ void __launch_bounds__(256, 2) hist_update_split(const double *__restrict__ F, const double *__restrict__ Fold,
                                                            const double *__restrict__ x,
                                                            const double *__restrict__ xold, int64_t n, int64_t ld,
                                                            double fnorm, double alpha, HT *__restrict__ dF,
                                                            HT *__restrict__ U, int slot, int nh, int store,
                                                            double *__restrict__ part) {
    constexpr int CPT = 8, SPL = NH / CPT, E = 4;
    __shared__ double sh[2 * NH * 8];
    const int h = threadIdx.x % SPL;  // this thread's column block: columns h CPT .. h CPT + 7
    double g[CPT], c[CPT];
#pragma unroll
    for (int k = 0; k < CPT; k++) { g[k] = 0.0; c[k] = 0.0; }
    const double rf = 1.0 / fnorm;
    const int64_t nE = n / E;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x / SPL;
    for (int64_t q = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / SPL; q < nE + (n - E * nE); q += stride) {
        const bool vec = q < nE;
        const int64_t i0 = vec ? E * q : E * nE + (q - nE);
        const int cnt = vec ? E : 1;
        double f[E], dn[E];
        HT dnew[E] = {}, unew[E];
        if (vec) {
            ldE<E>(F + i0, f);
        } else {
            f[0] = F[i0];
        }
        if (store) {
            double fo[E], xx[E], xo[E];
            if (vec) {
                ldE<E>(Fold + i0, fo);
                ldE<E>(x + i0, xx);
                ldE<E>(xold + i0, xo);
            } else {
                fo[0] = Fold[i0]; xx[0] = x[i0]; xo[0] = xold[i0];
            }
#pragma unroll
            for (int e = 0; e < E; e++)
                if (e < cnt) hist_elem<HT>(f[e], fo[e], xx[e], xo[e], fnorm, rf, alpha, dnew[e], unew[e]);
            if (h == 0) {
                if (vec) {
                    hstE<HT, E>(dF + (int64_t)slot * ld + i0, dnew);
                    hstE<HT, E>(U + (int64_t)slot * ld + i0, unew);
                } else {
                    dF[(int64_t)slot * ld + i0] = dnew[0];
                    U[(int64_t)slot * ld + i0] = unew[0];
                }
            }
        }
#pragma unroll
        for (int e = 0; e < E; e++) dn[e] = (double)dnew[e];
        typename HV<HT, E>::t dk[CPT];
#pragma unroll
        for (int kk = 0; kk < CPT; kk++) {
            const int k = h * CPT + kk;
            if (k < nh && !(store && k == slot)) {
                if (vec) {
                    dk[kk] = *(const typename HV<HT, E>::t *)(dF + (int64_t)k * ld + i0);
                } else {
                    HT *d = (HT *)&dk[kk];
                    d[0] = dF[(int64_t)k * ld + i0];
                }
            }
        }
#pragma unroll
        for (int kk = 0; kk < CPT; kk++) {
            const int k = h * CPT + kk;
            if (k < nh) {
                const HT *d = (const HT *)&dk[kk];
#pragma unroll
                for (int e = 0; e < E; e++)
                    if (e < cnt) {
                        const double v = (store && k == slot) ? dn[e] : (double)d[e];
                        g[kk] = fma(v, dn[e], g[kk]);
                        c[kk] = fma(v, f[e], c[kk]);
                    }
            }
        }
    }
    // sums over the warp's lanes of the same column block (lanes h, h + SPL, ...), then over
    // the block's warps
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int kk = 0; kk < CPT; kk++) {
        double a = g[kk], b = c[kk];
#pragma unroll
        for (int o = 16; o >= SPL; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if (lane < SPL) {
            const int k = lane * CPT + kk;
            sh[(2 * k) * 8 + wid] = a;
            sh[(2 * k + 1) * 8 + wid] = b;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 2 * nh; t += blockDim.x) {
        double s2 = 0.0;
        for (int w = 0; w < nw; w++) s2 += sh[t * 8 + w];
        part[(int64_t)blockIdx.x * 2 * MAXH + t] = s2;
    }
}

template <typename HT>
static void launch_hist(int nb, cudaStream_t st, const double *F, const double *Fold, const double *x, const double *xold,
                        int64_t n, double fnorm, double alpha, HT *dF, HT *U, int slot, int nh, int store, double *part) {
    const int64_t ld = broyden_ld(n);
    if (nh <= 4)
        hist_update<HT, 4><<<nb, RED_THREADS, 0, st>>>(F, Fold, x, xold, n, ld, fnorm, alpha, dF, U, slot, nh, store, part);
    else if (nh <= 8)
        hist_update<HT, 8><<<nb, RED_THREADS, 0, st>>>(F, Fold, x, xold, n, ld, fnorm, alpha, dF, U, slot, nh, store, part);
    else if (nh <= 16)
        hist_update_split<HT, 16><<<nb, RED_THREADS, 0, st>>>(F, Fold, x, xold, n, ld, fnorm, alpha, dF, U, slot, nh,
                                                               store, part);
    else
        hist_update_split<HT, 32><<<nb, RED_THREADS, 0, st>>>(F, Fold, x, xold, n, ld, fnorm, alpha, dF, U, slot, nh,
                                                               store, part);
}

// x_new = x + alpha F - sum_k gamma_k U_k   (common/broyden_mixing.f90:165-178), the
// gamma terms subtracted one by one in k order as the reference's loop does
template <typename HT>
__global__ void __launch_bounds__(256) x_update(const double *__restrict__ x, const double *__restrict__ F,
                                                const HT *__restrict__ U, const double *__restrict__ gam, int nh,
                                                double alpha, int64_t n, int64_t ld, double *__restrict__ xnew) {
    __shared__ double gs[MAXH];
    if (threadIdx.x < nh) gs[threadIdx.x] = gam[threadIdx.x];
    __syncthreads();
    const int64_t n4 = n / 4;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n4; q += stride) {
        const int64_t i0 = 4 * q;
        double4 xv = ld4(x + i0), fv = ld4(F + i0);
        double r[4] = {xv.x + alpha * fv.x, xv.y + alpha * fv.y, xv.z + alpha * fv.z, xv.w + alpha * fv.w};
        for (int k = 0; k < nh; k++) {
            double u[4];
            hld4<HT>(U + (int64_t)k * ld + i0, u);
#pragma unroll
            for (int e = 0; e < 4; e++) r[e] -= u[e] * gs[k];
        }
        st4(xnew + i0, double4{r[0], r[1], r[2], r[3]});
    }
    for (int64_t i = 4 * n4 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
        double xi = x[i] + alpha * F[i];
        for (int k = 0; k < nh; k++) xi -= (double)U[(int64_t)k * ld + i] * gs[k];
        xnew[i] = xi;
    }
}

// deterministic sum of per-block partials: out[j] = op_b part[b*stride + j]
__global__ void part_reduce(const double *__restrict__ part, int nb, int stride, int nv, int max_first,
                            double *__restrict__ out) {
    int j = threadIdx.x;
    if (j >= nv) return;
    double s = 0.0;
    for (int b = 0; b < nb; b++) {
        double v = part[(int64_t)b * stride + j];
        s = (max_first && j == 0) ? fmax(s, v) : s + v;
    }
    out[j] = s;
}

// Cholesky solve of the nh x nh system (w0^2 I + dF^T dF) gamma = dF^T F, as dposv('U').
// Returns 0 or the LAPACK-style info (> 0: not positive definite). A pivot fails only when
// it is <= 0, as in the OpenBLAS dpotrf the reference links (its unblocked factorisation
// tests ajj <= 0): a NaN pivot passes and the NaN reaches gamma, so a non-finite Gram matrix
// does not reset the history there either.
static int chol_solve(int nh, const std::vector<double> &A0, int lda, std::vector<double> &b) {
    std::vector<double> U((size_t)nh * nh, 0.0);
    for (int j = 0; j < nh; j++) {
        double s = A0[j + (size_t)j * lda];
        for (int k = 0; k < j; k++) s -= U[k + (size_t)j * nh] * U[k + (size_t)j * nh];
        if (s <= 0.0) return j + 1;
        double ujj = std::sqrt(s);
        U[j + (size_t)j * nh] = ujj;
        for (int i = j + 1; i < nh; i++) {
            double t = A0[j + (size_t)i * lda];
            for (int k = 0; k < j; k++) t -= U[k + (size_t)j * nh] * U[k + (size_t)i * nh];
            U[j + (size_t)i * nh] = t / ujj;
        }
    }
    for (int i = 0; i < nh; i++) {  // U^T y = b
        double s = b[i];
        for (int k = 0; k < i; k++) s -= U[k + (size_t)i * nh] * b[k];
        b[i] = s / U[i + (size_t)i * nh];
    }
    for (int i = nh - 1; i >= 0; i--) {  // U x = y
        double s = b[i];
        for (int k = i + 1; k < nh; k++) s -= U[i + (size_t)k * nh] * b[k];
        b[i] = s / U[i + (size_t)i * nh];
    }
    return 0;
}

int broyden_solve_dev(qs_handle *h, BroydenResidual &res, double *&d_x, double *&d_F, double *&d_Fold, double *&d_xold,
                      void *d_hdF, void *d_hU, int64_t n, double alpha_mix, int nhist, int maxscf, double tolf, bool sp,
                      BroydenOut &out) {
    const double w0 = 0.01;  // Johnson's regulariser
    if (nhist > MAXH) {
        h->err = "nhist larger than " + std::to_string(MAXH) + " is not supported";
        return -1;
    }
    const int lda = std::max(nhist, 1);
    std::vector<double> gram((size_t)lda * lda, 0.0), a((size_t)lda * lda), cvec(lda);
    const int nb = red_blocks(n);
    double *part = h->d_red, *fin = h->d_red + (size_t)RED_BLOCKS * 2 * MAXH;
    double *gam = fin + 2 * MAXH;
    std::vector<double> hv(2 * MAXH + 4);
    int nstored = 0, nh = 0;
    out = BroydenOut{};
    out.fmax = HUGE_VAL;
    cudaStream_t st = h->stream;
    for (int its = 1; its <= maxscf; its++) {
        out.n_iter = its;
        bool abort = false;
        int rc = res(d_x, d_F, abort);
        if (rc) return rc;
        if (abort) {
            out.aborted = true;
            break;
        }
        // max|F|, ||F||, ||F - Fold||
        const bool want_dn = its > 1 && nhist > 0;
        int pi = prof_begin(h, K_BROYDEN);
        vec_norms<<<nb, RED_THREADS, 0, st>>>(d_F, want_dn ? d_Fold : nullptr, n, part);
        prof_end(h, pi);
        count_launch();
        part_reduce<<<1, 32, 0, st>>>(part, nb, 3, 3, 1, fin);
        QS_CUDA(h, cudaGetLastError());
        QS_CUDA(h, cudaMemcpyAsync(hv.data(), fin, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
        QS_CUDA(h, cudaStreamSynchronize(st));
        double fmax = hv[0], rms = std::sqrt(hv[1]) / std::sqrt((double)n), fnorm = std::sqrt(hv[2]);
        out.fmax = fmax;
        out.log.push_back({its, fmax, rms, std::min(nstored, nhist)});
        if (fmax < tolf) {
            out.converged = true;
            break;
        }
        // history pair, Gram column, dF^T F. A residual that changed precision (the FP32
        // phase of a mixed solve ending) starts a new history: the stored pairs model the
        // other residual function
        if (res.precision_changed()) {
            nstored = 0;
            nh = 0;
        }
        bool store = want_dn && fnorm > 0.0 && !res.precision_changed();
        int slot = want_dn ? nstored % nhist : 0;
        int nh_new = store ? std::min(nstored + 1, nhist) : std::min(nstored, nhist);
        if (nh_new > 0 || store) {
            int pj = prof_begin(h, K_BROYDEN);
            if (sp)
                launch_hist<float>(nb, st, d_F, d_Fold, d_x, d_xold, n, store ? fnorm : 1.0, alpha_mix, (float *)d_hdF,
                                   (float *)d_hU, slot, nh_new, store, part);
            else
                launch_hist<double>(nb, st, d_F, d_Fold, d_x, d_xold, n, store ? fnorm : 1.0, alpha_mix, (double *)d_hdF,
                                    (double *)d_hU, slot, nh_new, store, part);
            prof_end(h, pj);
            count_launch();
            part_reduce<<<1, 2 * MAXH, 0, st>>>(part, nb, 2 * MAXH, 2 * nh_new, 0, fin);
            QS_CUDA(h, cudaGetLastError());
            QS_CUDA(h, cudaMemcpyAsync(hv.data(), fin, 2 * nh_new * sizeof(double), cudaMemcpyDeviceToHost, st));
            QS_CUDA(h, cudaStreamSynchronize(st));
        }
        if (store) {
            nstored++;
            for (int k = 0; k < nh_new; k++) {
                gram[k + (size_t)slot * lda] = hv[2 * k];
                gram[slot + (size_t)k * lda] = hv[2 * k];
            }
        }
        nh = std::min(nstored, nhist);
        for (int k = 0; k < nh; k++) cvec[k] = hv[2 * k + 1];
        // gamma = (w0^2 I + dF^T dF)^-1 dF^T F
        if (nh > 0) {
            for (int j = 0; j < nh; j++)
                for (int i = 0; i < nh; i++) a[i + (size_t)j * lda] = gram[i + (size_t)j * lda];
            for (int i = 0; i < nh; i++) a[i + (size_t)i * lda] += w0 * w0;
            std::vector<double> b(cvec.begin(), cvec.begin() + nh);
            if (chol_solve(nh, a, lda, b) != 0) {
                nstored = 0;  // WARNING: Broyden history ill-conditioned, resetting
                nh = 0;
                out.n_resets++;
            } else {
                QS_CUDA(h, cudaMemcpyAsync(gam, b.data(), nh * sizeof(double), cudaMemcpyHostToDevice, st));
            }
        }
        // x_new into the xold buffer, then rotate: xold <- x, x <- x_new, Fold <- F
        int pk = prof_begin(h, K_BROYDEN);
        if (sp)
            x_update<float><<<nb, RED_THREADS, 0, st>>>(d_x, d_F, (const float *)d_hU, gam, nh, alpha_mix, n, broyden_ld(n), d_xold);
        else
            x_update<double><<<nb, RED_THREADS, 0, st>>>(d_x, d_F, (const double *)d_hU, gam, nh, alpha_mix, n, broyden_ld(n), d_xold);
        prof_end(h, pk);
        QS_CUDA(h, cudaGetLastError());
        std::swap(d_x, d_xold);
        std::swap(d_F, d_Fold);
    }
    return 0;
}

int vec_maxabs(qs_handle *h, const double *d_v, int64_t n, double &mx) {
    const int nb = red_blocks(n);
    double *part = h->d_red, *fin = h->d_red + (size_t)RED_BLOCKS * 2 * MAXH;
    int pi = prof_begin(h, K_BROYDEN);
    vec_norms<<<nb, RED_THREADS, 0, h->stream>>>(d_v, nullptr, n, part);
    prof_end(h, pi);
    count_launch();
    part_reduce<<<1, 32, 0, h->stream>>>(part, nb, 3, 3, 1, fin);
    QS_CUDA(h, cudaGetLastError());
    double hv[3];
    QS_CUDA(h, cudaMemcpyAsync(hv, fin, 3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    QS_CUDA(h, cudaStreamSynchronize(h->stream));
    mx = hv[0];
    return 0;
}

size_t broyden_red_len() { return (size_t)RED_BLOCKS * 2 * MAXH + 4 * MAXH; }

}  // namespace qs
