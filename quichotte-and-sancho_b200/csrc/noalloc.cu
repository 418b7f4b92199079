// noalloc.cu -- qs_invert_batched_noalloc: the batched Dyson inversion for callers that
// cannot allocate GPU memory.
//
// Who needs it: a caller whose device memory is all handed out by someone else, e.g. a
// solver embedded in a larger GPU application that owns a fixed memory pool or arena and
// forbids allocations behind its back, or a latency-critical loop that cannot afford the
// device-wide synchronisation cudaMalloc/cudaFree may cause. Such a caller already holds
// its matrices and outputs in device memory and only needs the inversion itself.
//
// The Gauss-Jordan kernel normally keeps each matrix in shared memory and falls back to a
// global workspace that qs_create / qs_invert_batched allocate. Here the workspace is the
// file-scope array below instead: QS_NOALLOC_SCRATCH_BYTES (16 MiB) on every GPU that loads
// this library, held until the process exits. Every matrix goes through it, whatever N.
// Its device address is looked up on every call (cudaGetSymbolAddress with the caller's
// device current), so a context that was destroyed and created again (cudaDeviceReset)
// never leaves a stale address behind; host code never uses the symbol itself. The first
// call on a device may load the module there, so it should come before any stream capture.
#include <climits>
#include <cstdio>

#include "qs_common.cuh"

namespace {

constexpr size_t QS_NOALLOC_SCRATCH_BYTES = 16u << 20;  // 16 MiB
constexpr size_t QS_NOALLOC_HEADER = 256;               // first bytes: the min-info word
constexpr int QS_NOALLOC_MAX_N = 512;                   // the kernel's limit (>= 3 slots of 512^2 fit)

static __device__ __align__(256) unsigned char g_noalloc_scratch[QS_NOALLOC_SCRATCH_BYTES];

// device address of the scratch array in the current context of the current device
int scratch_address(void **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return -(int)e;
    if (p == nullptr) return -1;
    *out = p;
    return 0;
}

}  // namespace

extern "C" int qs_invert_batched_noalloc(int N, int batch, double *A, int *info, void *stream) {
    if (N < 1 || N > QS_NOALLOC_MAX_N || batch < 0) {
        std::fprintf(stderr,
                     "qs_invert_batched_noalloc: N = %d, batch = %d rejected: needs 1 <= N <= %d and batch >= 0 "
                     "(scratch %zu bytes per GPU)\n",
                     N, batch, QS_NOALLOC_MAX_N, QS_NOALLOC_SCRATCH_BYTES);
        return QS_ERR_NOALLOC_LIMIT;
    }
    if (batch == 0) return 0;
    if (!A || !info) return -1;
    void *base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    const size_t per = (size_t)N * N * sizeof(qs::zc);
    const int slots = (int)((QS_NOALLOC_SCRATCH_BYTES - QS_NOALLOC_HEADER) / per);
    if (slots < 1) return QS_ERR_NOALLOC_LIMIT;
    cudaStream_t st = (cudaStream_t)stream;
    int *d_min = (int *)base;
    qs::zc *ws = (qs::zc *)((unsigned char *)base + QS_NOALLOC_HEADER);
    // the scratch keeps the previous call's contents: the outputs that must start at zero
    // (info) and the min-info word are reset here; the workspace is overwritten per matrix
    cudaError_t e = cudaMemsetAsync(info, 0, sizeof(int) * (size_t)batch, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_min, 0x7f, sizeof(int), st);
    if (e != cudaSuccess) return -(int)e;
    return qs::invert_batched_ws(st, N, batch, (qs::zc *)A, d_min, info, ws, slots);
}
