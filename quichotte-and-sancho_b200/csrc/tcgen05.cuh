// tcgen05.cuh -- Blackwell (sm_100a) fifth-generation tensor-core primitives, as inline PTX:
// tensor-memory (TMEM) allocation, shared-memory matrix descriptors, tcgen05.mma of kind
// tf32 with FP32 accumulators in TMEM, completion through an mbarrier, and TMEM -> register
// loads for the epilogue.
//
// Operand layout used throughout (the canonical K-major, no-swizzle layout of the tensor
// core): an R x K tile of 32-bit elements is a grid of "core matrices" of 8 rows x 4
// elements (16 bytes a row, 128 bytes each, rows contiguous). Core matrix (g, q) -- rows
// 8g..8g+7, elements 4q..4q+3 -- starts at byte ((g * NQ) + q) * 128 with NQ = K / 4:
//   element (r, k) at byte ((r >> 3) * NQ + (k >> 2)) * 128 + (r & 7) * 16 + (k & 3) * 4.
// The descriptor of the k-step s (elements 8s..8s+7) starts at byte 256 s, with the leading
// (K-direction) core-matrix offset 128 bytes and the stride (row-direction) offset NQ * 128.
//
// Every wait on an mbarrier is bounded (a poll count and a 2 s clock limit): it gives up and
// reports it, so that a kernel can record an error, free its TMEM and return.
#pragma once

#include <cstdint>

namespace qs {
namespace tc {

constexpr uint32_t QS_TC_SPIN_LIMIT = 1u << 24;
constexpr uint64_t QS_TC_WAIT_NS = 2000000000ull;  // 2 s

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// ---- TMEM allocation (one full warp executes these) ----
__device__ __forceinline__ void tmem_alloc(uint32_t *slot_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot_smem)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---- mbarrier ----
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// bounded wait for the phase with the given parity to complete: gives up after
// QS_TC_SPIN_LIMIT polls or QS_TC_WAIT_NS nanoseconds, whichever comes first; false if so
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 0; it < QS_TC_SPIN_LIMIT; it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 255) == 255 && global_ns() - t0 > QS_TC_WAIT_NS) return false;
    }
    return false;
}

// ---- MMA ----
// shared-memory matrix descriptor, K-major, no swizzle (byte offsets are multiples of 16)
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
    return d;
}
// instruction descriptor: kind::tf32, FP32 accumulator, both operands K-major, M x N
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, bool neg_a, bool neg_b) {
    return (1u << 4)                          // D format: F32
           | (2u << 7) | (2u << 10)           // A, B format: TF32
           | ((neg_a ? 1u : 0u) << 13) | ((neg_b ? 1u : 0u) << 14)
           | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// D[tmem] (+)= A[desc] B[desc]^T; issued by one thread
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// the mbarrier receives one arrival when every MMA issued before by this thread completed
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// ---- TMEM -> registers: 32 lanes (this warp's quarter) x 32 consecutive 32-bit columns ----
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// ---- TMEM -> registers: 32 lanes x 16 consecutive 32-bit columns ----
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// ---- TF32 splitting: x = hi + lo with hi, lo representable in TF32 (round to nearest) ----
__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}
__device__ __forceinline__ void split_tf32(float x, float &hi, float &lo) {
    hi = to_tf32(x);
    lo = to_tf32(x - hi);
}

// byte offset of element (r, k) in the K-major core-matrix layout with NQ = K / 4
__host__ __device__ __forceinline__ uint32_t cm_offset(int r, int k, int NQ) {
    return (uint32_t)((((r >> 3) * NQ + (k >> 2)) << 7) + ((r & 7) << 4) + ((k & 3) << 2));
}

}  // namespace tc
}  // namespace qs
