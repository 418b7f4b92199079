// fft.cuh -- mixed-radix (2,3,4,5,7,8) Stockham FFT of many short sequences held in
// shared memory, cooperatively by one thread block.
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
// After the last pass the result is in natural order.
#pragma once
#include "qs_common.cuh"

namespace qs {

// twiddle W_Nf^m (m in [0, Nf)) for the given sign
template <typename T>
__device__ __forceinline__ cplx<T> twid(const cplx<T> *__restrict__ tw, int m, int sign) {
    cplx<T> w = tw[m];
    return sign < 0 ? w : conj(w);
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

template <typename T>
__device__ __forceinline__ void butterfly(cplx<T> *v, int R, int sign, const cplx<T> *__restrict__ tw, int Nf) {
    if (R == 2) {
        cplx<T> a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    } else if (R == 4) {
        bfly4(v[0], v[1], v[2], v[3], sign);
    } else if (R == 8) {
        // even / odd radix-4 halves, then the radix-2 combination with W8^q
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
    } else {  // 3, 5, 7: direct DFT with table twiddles W_R^m = W_Nf^{m Nf/R}
        cplx<T> o[7];
        int st = Nf / R;
        for (int q = 0; q < R; q++) {
            cplx<T> s = v[0];
            for (int r = 1; r < R; r++) {
                int m = (r * q) % R;
                if (m == 0) s = s + v[r];
                else cfma(s, v[r], twid(tw, m * st, sign));
            }
            o[q] = s;
        }
        for (int q = 0; q < R; q++) v[q] = o[q];
    }
}

// FFT of nseq sequences of length P.L stored contiguously in buf (sequence s at s*L).
// tmp has the same size. Returns the buffer that holds the result. Ends with a barrier.
template <typename T>
__device__ cplx<T> *smem_fft(cplx<T> *buf, cplx<T> *tmp, int nseq, const FftLen &P, int sign,
                             const cplx<T> *__restrict__ tw, int Nf) {
    const int L = P.L;
    const int tws = Nf / L;
    cplx<T> *a = buf, *b = tmp;
    int Ns = 1;
    for (int p = 0; p < P.nrad; p++) {
        const int R = P.rad[p];
        const int nR = L / R;
        const int total = nseq * nR;
        const int ang = L / (Ns * R);
        for (int t = threadIdx.x; t < total; t += blockDim.x) {
            int s = t / nR, j = t - s * nR;
            const cplx<T> *src = a + (size_t)s * L;
            cplx<T> *dst = b + (size_t)s * L;
            int k = j % Ns;
            cplx<T> v[8];
#pragma unroll
            for (int r = 0; r < 8; r++)
                if (r < R) {
                    v[r] = src[j + r * nR];
                    if (r && k) v[r] = v[r] * twid(tw, (r * k * ang) * tws, sign);
                }
            butterfly(v, R, sign, tw, Nf);
            int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < 8; r++)
                if (r < R) dst[idxD + r * Ns] = v[r];
        }
        __syncthreads();
        cplx<T> *t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    return a;
}

}  // namespace qs
