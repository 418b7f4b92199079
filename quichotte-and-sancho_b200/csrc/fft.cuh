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
// After the last pass the result is in natural order. A pass is done in place: every lane
// first loads all inputs of its butterflies into registers, the warp synchronises, then
// the outputs are written. Only __syncwarp is needed, never a block barrier.
//
// Shared-memory index padding: element p of a sequence lives at p + p/8 (one spare complex
// every 8), which spreads the strided accesses of the early passes over all banks.
#pragma once
#include "qs_common.cuh"

namespace qs {

__host__ __device__ __forceinline__ int pidx(int p) { return p + (p >> 3); }
__host__ __device__ __forceinline__ int padded_len(int L) { return L + (L >> 3) + 1; }

// twiddle W_Nf^m (m in [0, Nf)) for the given sign
template <typename T>
__device__ __forceinline__ cplx<T> twid(const cplx<T> *__restrict__ tw, int m, int sign) {
    return sign < 0 ? tw[m] : conj(tw[m]);
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
__device__ __forceinline__ void dft(cplx<T> (&v)[R], int sign, const cplx<T> *__restrict__ tw, int Nf) {
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
    } else {  // 3, 5, 7: direct DFT with table constants W_R^m = W_Nf^{m Nf/R}
        cplx<T> o[R];
        const int st = Nf / R;
#pragma unroll
        for (int q = 0; q < R; q++) {
            cplx<T> s = v[0];
#pragma unroll
            for (int r = 1; r < R; r++) {
                const int m = (r * q) % R;
                if (m == 0) s = s + v[r];
                else {
                    cplx<T> w = sign < 0 ? tw[m * st] : conj(tw[m * st]);
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
                                          const cplx<T> *__restrict__ tw, int Nf) {
    const int lane = threadIdx.x & 31;
    const int nR = L / R;
    const int tws = Nf / L;
    const int ang = L / (Ns * R);
    for (int j = lane; j < nR; j += 32) {
        cplx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = src[pidx(j + r * nR)];
        const int k = j % Ns;
        if (k) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                const int m = (r * k * ang) * tws;
                v[r] = v[r] * (sign < 0 ? tw[m] : conj(tw[m]));
            }
        }
        dft<T, R>(v, sign, tw, Nf);
        const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) dst[pidx(idxD + r * Ns)] = v[r];
    }
    __syncwarp();
}

// the whole transform of one padded sequence s by one warp, with the warp's own scratch
// sequence; the result is left in s
template <typename T>
__device__ void warp_fft(cplx<T> *s, cplx<T> *scratch, const FftLen &P, int sign, const cplx<T> *__restrict__ tw,
                         int Nf) {
    cplx<T> *a = s, *b = scratch;
    const int L = P.L;
    int Ns = 1;
    unsigned code = P.code;
    for (int p = 0; p < P.nrad; p++) {
        const int R = code & 15u;
        code >>= 4;
        switch (R) {
            case 2: warp_pass<T, 2>(a, b, L, Ns, sign, tw, Nf); break;
            case 3: warp_pass<T, 3>(a, b, L, Ns, sign, tw, Nf); break;
            case 4: warp_pass<T, 4>(a, b, L, Ns, sign, tw, Nf); break;
            case 5: warp_pass<T, 5>(a, b, L, Ns, sign, tw, Nf); break;
            case 7: warp_pass<T, 7>(a, b, L, Ns, sign, tw, Nf); break;
            default: warp_pass<T, 8>(a, b, L, Ns, sign, tw, Nf); break;
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

}  // namespace qs
