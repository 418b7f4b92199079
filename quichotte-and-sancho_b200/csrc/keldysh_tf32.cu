// keldysh_tf32.cu -- the Keldysh step of the FP32 phase of a QS_PREC_MIXED solve on the
// fifth-generation tensor cores: G^< = G^r SL G^r^dagger (src/scf.f90:333-355) with
// SL = i (f_L Gamma_L + f_R Gamma_R) + Sigma2^<, written into the SCF residual as
// F = pack(G_out) - x (src/scf.f90:158-188; pack_gf common/linear_algebra.f90:155-191).
//
// One CTA of 16 warps per SM walks the energies. Both complex products (T = G SL, then
// L = T G^dagger) run as tcgen05.mma of kind tf32 with FP32 accumulators in tensor memory:
// each operand x is split into two TF32 parts x = hi + lo (round to nearest), and each real
// product a b is formed as a_hi b_hi + a_hi b_lo + a_lo b_hi ("3xTF32"), which keeps close
// to FP32 accuracy; a complex product is four real ones (the -Im Im term through the
// instruction's A-negate bit), so 12 MMAs of 128 x 128 x 8 per k-step of 8.
//   * Operands are padded to 128 and staged in 16-wide k chunks into shared memory in the
//     tensor core's K-major core-matrix layout (tcgen05.cuh), double-buffered: the chunk
//     after the next is staged while the tensor core works on the current one, and a
//     buffer is refilled only once the mbarrier signalled by tcgen05.commit says the MMAs
//     that read it completed. Every thread stages one (row, k-quad) of each operand: the
//     G^r columns are read with consecutive rows on consecutive lanes, the SL rows (Sigma2^<
//     is column-major, SL(k, n) at k + n nA) with four consecutive k per lane, so that all
//     loads are coalesced, and 16 warps keep enough of them in flight to cover the latency
//     of the global reads (the conversion and split run on the CUDA cores).
//   * TMEM holds T (columns 0-255: real, imaginary) and L (256-511). The second product reads
//     T back from TMEM (tcgen05.ld), splits it and stages it as its A operand.
//   * The epilogue reads L from TMEM (lane = row; the four warps of a lane quarter take
//     different 32-column blocks), writes the upper triangle of G^< minus x into F, the
//     diagonal into gLd, and copies G^r - x (FP64) into the G^r part of F.
// The G^r part of F is exact (FP64 from the Dyson kernel); the G^< part carries the
// rounding of the FP32 products (relative ~1e-7), which the FP32 phase tolerates (the
// residual switches to the FP64 kernels before max|F| approaches that level).
//
// Every wait on an mbarrier is bounded; a wait that gives up sets *err, the CTA waits (again
// bounded) for its MMAs in flight, frees its tensor memory and returns.
#include <cstdint>

#include "qs_common.cuh"
#include "tcgen05.cuh"

namespace qs {
namespace {

using namespace tc;

constexpr int KT_M = 128;                  // padded order: M = N = K = 128
constexpr int KT_KC = 16;                  // k per staged chunk
constexpr int KT_NQ = KT_KC / 4;           // 16-byte k-quads per row of a chunk
constexpr int KT_NCH = KT_M / KT_KC;       // chunks per product
constexpr int KT_TILE = KT_M * KT_KC * 4;  // one 128 x 16 TF32 tile: 8 KB
constexpr int KT_BUF = 8 * KT_TILE;        // A (re hi, re lo, im hi, im lo) + B (the same)
constexpr int KT_SMEM = 2 * KT_BUF;        // two buffers: 128 KB
constexpr int KT_THREADS = 512;  // 16 warps: 4 lane quarters x 4
constexpr uint32_t KT_TMEM_COLS = 512;     // T re, T im, L re, L im: 128 columns each

// one 4-element k-quad of row r (real and imaginary parts) split into the 4 tiles of a half
__device__ __forceinline__ void put_quad(unsigned char *half, int r, int q, const float (&re)[4], const float (&im)[4]) {
    float4 rh, rl, ih, il;
    split_tf32(re[0], rh.x, rl.x);
    split_tf32(re[1], rh.y, rl.y);
    split_tf32(re[2], rh.z, rl.z);
    split_tf32(re[3], rh.w, rl.w);
    split_tf32(im[0], ih.x, il.x);
    split_tf32(im[1], ih.y, il.y);
    split_tf32(im[2], ih.z, il.z);
    split_tf32(im[3], ih.w, il.w);
    const uint32_t o = cm_offset(r, 4 * q, KT_NQ);
    *(float4 *)(half + 0 * KT_TILE + o) = rh;
    *(float4 *)(half + 1 * KT_TILE + o) = rl;
    *(float4 *)(half + 2 * KT_TILE + o) = ih;
    *(float4 *)(half + 3 * KT_TILE + o) = il;
}

// the 24 MMAs of one staged chunk (two k-steps): D (re at d, im at d + 128) += A B
__device__ __forceinline__ void chunk_mmas(uint32_t bb, uint32_t d, bool first) {
    constexpr uint32_t i_pp = idesc_tf32(KT_M, KT_M, false, false), i_np = idesc_tf32(KT_M, KT_M, true, false);
    const uint32_t Dr = d, Di = d + KT_M;
#pragma unroll
    for (int s = 0; s < KT_KC / 8; s++) {
        auto A = [&](int t) { return smem_desc(bb + t * KT_TILE + 256 * s, 128, KT_NQ * 128); };
        auto B = [&](int t) { return smem_desc(bb + (4 + t) * KT_TILE + 256 * s, 128, KT_NQ * 128); };
        const uint32_t acc0 = (first && s == 0) ? 0u : 1u;
        mma_tf32(Dr, A(0), B(0), i_pp, acc0);  // + Re A Re B
        mma_tf32(Dr, A(0), B(1), i_pp, 1);
        mma_tf32(Dr, A(1), B(0), i_pp, 1);
        mma_tf32(Dr, A(2), B(2), i_np, 1);     // - Im A Im B
        mma_tf32(Dr, A(2), B(3), i_np, 1);
        mma_tf32(Dr, A(3), B(2), i_np, 1);
        mma_tf32(Di, A(0), B(2), i_pp, acc0);  // + Re A Im B
        mma_tf32(Di, A(0), B(3), i_pp, 1);
        mma_tf32(Di, A(1), B(2), i_pp, 1);
        mma_tf32(Di, A(2), B(0), i_pp, 1);     // + Im A Re B
        mma_tf32(Di, A(2), B(1), i_pp, 1);
        mma_tf32(Di, A(3), B(0), i_pp, 1);
    }
}

__global__ void __launch_bounds__(KT_THREADS, 1) keldysh_tf32(KeldyshArgs a) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ uint64_t bar[2];
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nA = a.nA, nfull = nA * nA;
    if (warp == 0) {
        tmem_alloc(&tslot, KT_TMEM_COLS);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tm = tslot, tT = tm, tL = tm + 2 * KT_M;
    const uint32_t sbase = smem_u32(sm);
    const uint32_t lanes = (uint32_t)(32 * (warp & 3)) << 16;  // this warp's TMEM lane quarter
    const int64_t offL = 2 * (int64_t)nfull, offD = offL + (int64_t)nA * (nA - 1);
    int g = 0;  // chunks staged so far: buffer g & 1, mbarrier phase g >> 1
    bool ok = true;
    // wait (block-uniformly) until the MMAs of chunk gg have completed
    auto wait_chunk = [&](int gg) -> bool {
        const bool w = gg < 0 || mbar_wait(&bar[gg & 1], (gg >> 1) & 1);
        return !__syncthreads_or(!w);
    };
    for (int iw = blockIdx.x; iw < a.n && ok; iw += gridDim.x) {
        const zc *G = a.G + (size_t)iw * nfull;
        const double w = a.omega[iw];
        const double fL = fermi_d(w, a.V, a.mu, a.beta), fR = fermi_d(w, 0.0, a.mu, a.beta);
        const zc *SL2 = a.SigL ? a.SigL + (size_t)iw * nfull : nullptr;
        // ---- T = G SL: thread (m = tid % 128, quad tid / 128) stages A = G(m, k), thread
        // (n = tid / 4, quad tid % 4) stages B = SL(k, n)
        for (int c = 0; c < KT_NCH; c++, g++) {
            if (!(ok = wait_chunk(g - 2))) break;
            unsigned char *buf = sm + (g & 1) * KT_BUF;
            {
                const int m = tid & (KT_M - 1), q = tid >> 7;
                float re[4], im[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int k = KT_KC * c + 4 * q + e;
                    const zc gv = (m < nA && k < nA) ? G[m + (size_t)k * nA] : zc{0, 0};
                    re[e] = (float)gv.x;
                    im[e] = (float)gv.y;
                }
                put_quad(buf, m, q, re, im);
            }
            {
                const int n = tid >> 2, q = tid & 3;
                float re[4], im[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int k = KT_KC * c + 4 * q + e;
                    zc s{0, 0};
                    if (n < nA && k < nA) {  // SL(k, n) = i (fL GamL_s + fR GamR_s) / hbar + Sigma2^<  (src/scf.f90:333-336)
                        const size_t idx = k + (size_t)n * nA;
                        const zc gl = a.GamLs[idx], gr = a.GamRs[idx];
                        const zc s2 = SL2 ? SL2[idx] : zc{0, 0};
                        s = zc{-(fL * gl.y + fR * gr.y) + s2.x, fL * gl.x + fR * gr.x + s2.y};
                    }
                    re[e] = (float)s.x;
                    im[e] = (float)s.y;
                }
                put_quad(buf + 4 * KT_TILE, n, q, re, im);
            }
            fence_async_smem();
            __syncthreads();
            if (tid == 0) {
                fence_after_sync();
                chunk_mmas(sbase + (g & 1) * KT_BUF, tT, c == 0);
                mma_commit(&bar[g & 1]);
            }
        }
        if (!ok || !(ok = wait_chunk(g - 1))) break;  // T complete
        fence_after_sync();
        // ---- L = T G^dagger: warps 0-3 stage A = T from tensor memory (row = TMEM lane),
        // thread (n = tid % 128, quad tid / 128) stages B(k, n) = conj G(n, k)
        for (int c = 0; c < KT_NCH; c++, g++) {
            if (!(ok = wait_chunk(g - 2))) break;
            unsigned char *buf = sm + (g & 1) * KT_BUF;
            if (warp < 4) {
                float tr[16], ti[16];
                tmem_ld16(tT + lanes + KT_KC * c, tr);
                tmem_ld16(tT + lanes + KT_M + KT_KC * c, ti);
                const int r = 32 * warp + lane;
#pragma unroll
                for (int q = 0; q < KT_NQ; q++) {
                    const float re[4] = {tr[4 * q], tr[4 * q + 1], tr[4 * q + 2], tr[4 * q + 3]};
                    const float im[4] = {ti[4 * q], ti[4 * q + 1], ti[4 * q + 2], ti[4 * q + 3]};
                    put_quad(buf, r, q, re, im);
                }
            }
            {
                const int n = tid & (KT_M - 1), q = tid >> 7;
                float bre[4], bim[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int k = KT_KC * c + 4 * q + e;
                    const zc gv = (n < nA && k < nA) ? G[n + (size_t)k * nA] : zc{0, 0};  // B(k, n) = conj G(n, k)
                    bre[e] = (float)gv.x;
                    bim[e] = -(float)gv.y;
                }
                put_quad(buf + 4 * KT_TILE, n, q, bre, bim);
            }
            fence_async_smem();
            __syncthreads();
            if (tid == 0) {
                fence_after_sync();
                chunk_mmas(sbase + (g & 1) * KT_BUF, tL, c == 0);
                mma_commit(&bar[g & 1]);
            }
        }
        if (!ok || !(ok = wait_chunk(g - 1))) break;  // L complete
        fence_after_sync();
        // ---- epilogue: the upper triangle of G^< and its diagonal, then G^r, minus x
        double *blk = a.out + (size_t)iw * a.nblk;
        const double *xb = a.xsub ? a.xsub + (size_t)iw * a.nblk : nullptr;
        const int r = 32 * (warp & 3) + lane;
        for (int j = warp >> 2; 32 * j < nA; j += KT_THREADS / 128) {  // warp-uniform
            float lr[32], li[32];
            tmem_ld32(tL + lanes + 32 * j, lr);
            tmem_ld32(tL + lanes + KT_M + 32 * j, li);
#pragma unroll 4
            for (int i = 0; i < 32; i++) {
                const int c = 32 * j + i;
                if (c >= nA || r > c) continue;
                if (r < c) {
                    const int64_t o = offL + 2 * ((int64_t)c * (c - 1) / 2 + r);
                    blk[o] = xb ? (double)lr[i] - xb[o] : (double)lr[i];
                    blk[o + 1] = xb ? (double)li[i] - xb[o + 1] : (double)li[i];
                } else {
                    blk[offD + r] = xb ? (double)li[i] - xb[offD + r] : (double)li[i];
                    if (a.gLd) a.gLd[(size_t)iw * nA + r] = zc{(double)lr[i], (double)li[i]};
                }
            }
        }
        for (int idx = tid; idx < nfull; idx += KT_THREADS) {
            const zc gv = G[idx];
            blk[2 * idx] = xb ? gv.x - xb[2 * idx] : gv.x;
            blk[2 * idx + 1] = xb ? gv.y - xb[2 * idx + 1] : gv.y;
        }
        if (a.gRd)
            for (int i = tid; i < nA; i += KT_THREADS) a.gRd[(size_t)iw * nA + i] = G[i + (size_t)i * nA];
        fence_before_sync();
        __syncthreads();  // TMEM reads done before the next energy's MMAs overwrite it
    }
    if (!ok) {
        if (tid == 0 && a.err) atomicExch(a.err, 1);
        if (g > 0) mbar_wait(&bar[(g - 1) & 1], ((g - 1) >> 1) & 1);  // MMAs in flight (bounded)
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (warp == 0) tmem_dealloc(tm, KT_TMEM_COLS);
}

}  // namespace

bool keldysh_tf32_fits(int nA) { return nA >= 32 && nA <= KT_M; }

int launch_keldysh_tf32(qs_handle *h, const KeldyshArgs &k) {
    if (!keldysh_tf32_fits(k.nA)) return -1;
    QS_CUDA(h, cudaFuncSetAttribute(keldysh_tf32, cudaFuncAttributeMaxDynamicSharedMemorySize, KT_SMEM));
    const int nb = std::min(k.n, 148);
    int pi = prof_begin(h, K_KELDYSH);
    keldysh_tf32<<<nb, KT_THREADS, KT_SMEM, h->stream>>>(k);
    prof_end(h, pi);
    QS_CUDA(h, cudaGetLastError());
    return 0;
}

}  // namespace qs
