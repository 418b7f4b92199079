// fft.cuh -- mixed-radix (2,3,4,5,7,8) Stockham FFTs of short sequences held in shared
// memory, one warp per sequence.
//
// Conventions are FFTW's, as the reference uses them (src/self_energies.f90:102-103,129,
// 205,208): sign = -1 is the forward transform sum_j x_j exp(-2 pi i jk/L), sign = +1 the
// backward one, both unnormalised.
//
// One pass of radix R over a sequence of length L with Ns = product of the radices already
// applied (autosort Stockham, decimation in time):
//   for j in [0, L/R):  k = j mod Ns
//     v_r = x[j + r L/R] * exp(sign 2 pi i r k / (Ns R)),   r = 0..R-1
//     v   = DFT_R(v)
//     y[(j / Ns) Ns R + k + r Ns] = v_r
// After the last pass the result is in natural order. The passes alternate between the
// sequence and a scratch sequence of the warp (out of place), so only __syncwarp is needed
// between them, never a block barrier.
//
// Shared-memory index padding: element p of a sequence lives at p + p/8 (one spare complex
// every 8), which spreads the strided accesses of the early passes over all banks.
//
// Twiddles come from a table twL[m] = exp(-2 pi i m / L), m < L, that the calling kernel
// keeps in shared memory (L1 holds little next to the sequence buffers, and a global table
// read at stride Nf/L would miss it on every access).
#pragma once
#include "qs_common.cuh"

namespace qs {

__host__ __device__ __forceinline__ int pidx(int p) { return p + (p >> 3); }
__host__ __device__ __forceinline__ int padded_len(int L) { return L + (L >> 3) + 1; }

// twiddle W^m from a table for the given sign
template <typename T> __device__ __forceinline__ cplx<T> twid(const cplx<T> *tw, int m, int sign) {
    return sign < 0 ? tw[m] : conj(tw[m]);
}

// an FP64 twiddle at the kernel's element type
template <typename T> __device__ __forceinline__ cplx<T> cvt(zc v) { return cplx<T>{(T)v.x, (T)v.y}; }

// The shared-memory twiddle table of a length-L transform. Power-of-two lengths 64/128/256:
// the twiddles of each pass with Ns > 1 laid out [r][k] (W_L^{r k L/(Ns R)} at r Ns + k,
// pass Ns = 8 first, then Ns = 64), so that the lanes of a pass read consecutive entries;
// other lengths: twL[m] = W_L^m.
__host__ __device__ __forceinline__ int fft_table_len(int L) {
    return L == 64 ? 64 : (L == 128 ? 192 : (L == 256 ? 320 : L));
}
// fill it from the FP64 table of W_Nf (tw[m * tws] = W_L^m), all threads of the block
template <typename T> __device__ void fft_table_fill(cplx<T> *tbl, int L, const zc *__restrict__ tw, int tws) {
    if (L == 64 || L == 128 || L == 256) {
        for (int idx = threadIdx.x; idx < 64; idx += blockDim.x) {
            const int r = idx >> 3, k = idx & 7;
            tbl[idx] = cvt<T>(tw[(size_t)(r * k * (L / 64)) * tws]);
        }
        for (int idx = threadIdx.x; idx < L; idx += blockDim.x) {  // (L / 64) x 64
            const int r = idx >> 6, k = idx & 63;
            if (L > 64) tbl[64 + idx] = cvt<T>(tw[(size_t)(r * k) * tws]);
        }
    } else {
        for (int m = threadIdx.x; m < L; m += blockDim.x) tbl[m] = cvt<T>(tw[(size_t)m * tws]);
    }
}

// multiply by sign*i
template <typename T> __device__ __forceinline__ cplx<T> mul_si(cplx<T> a, int sign) {
    return sign < 0 ? cplx<T>{a.y, -a.x} : cplx<T>{-a.y, a.x};
}

template <typename T>
__device__ __forceinline__ void bfly4(cplx<T> &a0, cplx<T> &a1, cplx<T> &a2, cplx<T> &a3, int sign) {
    cplx<T> s02 = a0 + a2, d02 = a0 - a2, s13 = a1 + a3, d13 = mul_si(a1 - a3, sign);
    a0 = s02 + s13;
    a2 = s02 - s13;
    a1 = d02 + d13;
    a3 = d02 - d13;
}

// DFT of R points in registers
template <typename T, int R>
__device__ __forceinline__ void dft(cplx<T> (&v)[R], int sign, const cplx<T> *twL, int L) {
    if constexpr (R == 2) {
        cplx<T> a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    } else if constexpr (R == 4) {
        bfly4(v[0], v[1], v[2], v[3], sign);
    } else if constexpr (R == 8) {
        cplx<T> e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
        cplx<T> o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
        bfly4(e0, e1, e2, e3, sign);
        bfly4(o0, o1, o2, o3, sign);
        const T h = (T)0.70710678118654752440084436210484903928;
        // W8^1 = (1 + sign i)/sqrt2 ; W8^2 = sign i ; W8^3 = (-1 + sign i)/sqrt2
        cplx<T> t1 = cplx<T>{h * (o1.x - (T)sign * o1.y), h * (o1.y + (T)sign * o1.x)};
        cplx<T> t2 = mul_si(o2, sign);
        cplx<T> t3 = cplx<T>{h * (-o3.x - (T)sign * o3.y), h * (-o3.y + (T)sign * o3.x)};
        v[0] = e0 + o0;
        v[4] = e0 - o0;
        v[1] = e1 + t1;
        v[5] = e1 - t1;
        v[2] = e2 + t2;
        v[6] = e2 - t2;
        v[3] = e3 + t3;
        v[7] = e3 - t3;
    } else {  // 3, 5, 7: direct DFT with table constants W_R^m = W_L^{m L/R}
        cplx<T> o[R];
        const int st = L / R;
#pragma unroll
        for (int q = 0; q < R; q++) {
            cplx<T> s = v[0];
#pragma unroll
            for (int r = 1; r < R; r++) {
                const int m = (r * q) % R;
                if (m == 0) s = s + v[r];
                else {
                    cplx<T> w = sign < 0 ? twL[m * st] : conj(twL[m * st]);
                    cfma(s, v[r], w);
                }
            }
            o[q] = s;
        }
#pragma unroll
        for (int q = 0; q < R; q++) v[q] = o[q];
    }
}

// one radix-R pass of a warp, src -> dst (both padded); butterflies are processed one at a
// time per lane, so only R values are live in registers
template <typename T, int R>
__device__ __forceinline__ void warp_pass(const cplx<T> *src, cplx<T> *dst, int L, int Ns, int sign,
                                          const cplx<T> *twL) {
    const int lane = threadIdx.x & 31;
    const int nR = L / R;
    const int ang = L / (Ns * R);
    for (int j = lane; j < nR; j += 32) {
        cplx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = src[pidx(j + r * nR)];
        const int k = j % Ns;
        if (k) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                const int m = r * k * ang;  // < R Ns ang = L
                v[r] = v[r] * (sign < 0 ? twL[m] : conj(twL[m]));
            }
        }
        dft<T, R>(v, sign, twL, L);
        const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) dst[pidx(idxD + r * Ns)] = v[r];
    }
    __syncwarp();
}

// the whole transform of one padded sequence s by one warp, with the warp's own scratch
// sequence and the length-L twiddle table twL; the result is left in s
template <typename T>
__device__ void warp_fft(cplx<T> *s, cplx<T> *scratch, const FftLen &P, int sign, const cplx<T> *twL) {
    cplx<T> *a = s, *b = scratch;
    const int L = P.L;
    int Ns = 1;
    unsigned code = P.code;
    for (int p = 0; p < P.nrad; p++) {
        const int R = code & 15u;
        code >>= 4;
        switch (R) {
            case 2: warp_pass<T, 2>(a, b, L, Ns, sign, twL); break;
            case 3: warp_pass<T, 3>(a, b, L, Ns, sign, twL); break;
            case 4: warp_pass<T, 4>(a, b, L, Ns, sign, twL); break;
            case 5: warp_pass<T, 5>(a, b, L, Ns, sign, twL); break;
            case 7: warp_pass<T, 7>(a, b, L, Ns, sign, twL); break;
            default: warp_pass<T, 8>(a, b, L, Ns, sign, twL); break;
        }
        cplx<T> *t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    if (a != s) {
        const int lane = threadIdx.x & 31;
        for (int j = lane; j < L; j += 32) s[pidx(j)] = a[pidx(j)];
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------
// Power-of-two lengths L = 64, 128, 256 with compile-time passes: the warp transforms
// P = 256 / L sequences at once (sequence q at s + q ps, q < nvalid), every lane holding 8
// complex values per pass, in place (all loads of a pass precede its stores; no scratch).
// Passes: radix 8 (Ns = 1), radix 8 (Ns = 8), then radix L / 64 (Ns = 64) when L > 64.
// ---------------------------------------------------------------------------------
template <typename T, int L, int R, int Ns>
__device__ __forceinline__ void pow2_pass(cplx<T> *s, int ps, int nvalid, int sign, const cplx<T> *twL) {
    static_assert(Ns == 1 || Ns == 8 || Ns == 64, "the passes of warp_fft_pow2");
    constexpr int nR = L / R;  // butterflies per sequence
    constexpr int U = 8 / R;   // butterflies per lane
    const int lane = threadIdx.x & 31;
    cplx<T> v[U][R];
#pragma unroll
    for (int u = 0; u < U; u++) {
        const int b = lane + 32 * u, sq = b / nR, j = b % nR;
        const cplx<T> *x = s + sq * ps;
#pragma unroll
        for (int r = 0; r < R; r++) v[u][r] = (sq < nvalid) ? x[pidx(j + r * nR)] : cplx<T>{0, 0};
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < U; u++) {
        const int b = lane + 32 * u, sq = b / nR, j = b % nR;
        const int k = j % Ns;
        if (Ns > 1 && k) {
            constexpr int off = (Ns == 8) ? 0 : 64;  // this pass's part of the table ([r][k])
#pragma unroll
            for (int r = 1; r < R; r++) v[u][r] = v[u][r] * twid(twL, off + r * Ns + k, sign);
        }
        dft<T, R>(v[u], sign, twL, L);
        cplx<T> *x = s + sq * ps;
        const int idxD = (j / Ns) * Ns * R + k;
        if (sq < nvalid) {
#pragma unroll
            for (int r = 0; r < R; r++) x[pidx(idxD + r * Ns)] = v[u][r];
        }
    }
    __syncwarp();
}

template <typename T, int L>
__device__ __forceinline__ void warp_fft_pow2(cplx<T> *s, int ps, int nvalid, int sign, const cplx<T> *twL) {
    static_assert(L == 64 || L == 128 || L == 256, "power-of-two lengths 64..256");
    pow2_pass<T, L, 8, 1>(s, ps, nvalid, sign, twL);
    pow2_pass<T, L, 8, 8>(s, ps, nvalid, sign, twL);
    if constexpr (L > 64) pow2_pass<T, L, L / 64, 64>(s, ps, nvalid, sign, twL);
}

// number of sequences one warp transforms per call for length L (1 on the generic path)
__host__ __device__ __forceinline__ int fft_group(int L) { return (L == 64 || L == 128 || L == 256) ? 256 / L : 1; }

// Transform the group of up to fft_group(L) sequences at s + q ps (q < nvalid) by the
// calling warp with the table of fft_table_fill; scratch is used by the generic path (one
// sequence per call).
template <typename T>
__device__ __forceinline__ void warp_fft_group(cplx<T> *s, int ps, int nvalid, cplx<T> *scratch, const FftLen &P,
                                               int sign, const cplx<T> *twL) {
    switch (P.L) {
        case 64: warp_fft_pow2<T, 64>(s, ps, nvalid, sign, twL); break;
        case 128: warp_fft_pow2<T, 128>(s, ps, nvalid, sign, twL); break;
        case 256: warp_fft_pow2<T, 256>(s, ps, nvalid, sign, twL); break;
        default: warp_fft(s, scratch, P, sign, twL); break;
    }
}

}  // namespace qs
