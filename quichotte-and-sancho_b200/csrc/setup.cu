// setup.cu -- the dense linear algebra of the model set-up, on the device.
//
//   qs_hermitian_eigensystem  hermitian_eigensystem (common/linear_algebra.f90:32-56, LAPACK
//                             zheev) over a batch of matrices of one size.
//   qs_hermitian_eigenvalues  the same without eigenvectors (zheev JOBZ = 'N'), which is all
//                             the energy grid needs (src/quichotte.f90:79-83): for N <= 160
//                             one block per matrix with the matrix in shared memory,
//                             Householder tridiagonalisation and Sturm multisection
//                             (tri_values below).
//   qs_dftb_lowdin            the dense part of build_hamiltonian_from_dftb_hs
//                             (src/hamiltonian.f90:625-640, 680-689): S^-1/2 from the
//                             eigenpairs of S (dsyev there), the SOC form on the spin-doubled
//                             basis and H = S^-1/2 Hao S^-1/2, made Hermitian.
//
// Eigenproblem: two-sided cyclic Jacobi in the round-robin (tournament) pair order, so the
// M/2 rotations of one round (M = N rounded up to even) act on disjoint index pairs and run
// at once. A round is two kernels:
//   jac_params   one thread per pair: the rotation that zeroes A(p,q), written as a pair
//                record and as two row records (the coefficients row p and row q take);
//   jac_rotate   each group of threads owns the two columns of one pair: it rotates them
//                (A J, and Z J for the eigenvectors), stages A J's two columns in shared
//                memory and applies the row rotations of all pairs to them (J^H A J).
// Every access is down a column, so A and Z stay column-major and coalesced. The M-1 rounds
// of a sweep and the convergence test are one CUDA graph, replayed once per sweep; the host
// reads one counter per sweep. A matrix is converged when its off-diagonal weight is at
// rounding level, sum_{i!=j} |a_ij|^2 <= (N eps)^2 sum |a_ij|^2; then every eigenvalue is
// within about N eps ||A||_F of the exact one, the accuracy class of zheev. Each matrix is
// first scaled by an exact power of two (jac_scale), so the sums of squares stay in range.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "qs_common.cuh"

namespace qs {
namespace {

// Work buffers of the set-up come from a memory pool of their own per device that keeps up
// to 4 GiB of freed memory mapped between calls (the default pool returns it at every
// synchronisation, so each call of a large size mapped its buffers again, at a cost that
// varied from call to call). It stays apart from the default pool that the solver handles use,
// whose free memory the serving loop's admission reads.
cudaError_t setup_alloc(void **p, size_t bytes, cudaStream_t st) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = pools.find(dev);
        if (it == pools.end()) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            if ((e = cudaMemPoolCreate(&pool, &props)) != cudaSuccess) return e;
            uint64_t keep = 4ull << 30;
            if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return e;
            pools[dev] = pool;
        } else {
            pool = it->second;
        }
    }
    return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

constexpr int JAC_MAX_N = 2048;
constexpr int JAC_MAX_SWEEPS = 60;
constexpr int JAC_THREADS = 256;

struct __align__(16) JacPair {
    double c, s, phx, phy;  // rotation: c, s and the phase of A(p,q)
    double app, aqq;        // the pivot block's diagonal after the rotation
    int p, q;               // p < q; q >= N marks the idle slot of an odd N
};
struct __align__(16) JacRow {
    double c, bx, by;  // A''(j,k) = c A'(j,k) + (bx + i by) A'(partner,k)
    int partner;
};

// index pair of slot i in round r of the round-robin order over M (even) indices
__device__ __forceinline__ void jac_slot(int M, int r, int i, int &p, int &q) {
    if (i == 0) {
        p = r;
        q = M - 1;
    } else {
        p = (r + i) % (M - 1);
        q = (r - i + (M - 1)) % (M - 1);
    }
    if (p > q) {
        int t = p;
        p = q;
        q = t;
    }
}

__global__ void jac_init(int N, int64_t total, zc *__restrict__ A, zc *__restrict__ Z) {
    const int64_t nn = (int64_t)N * N;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t % nn;
        const int i = (int)(e % N), j = (int)(e / N);
        Z[t] = zc{i == j ? 1.0 : 0.0, 0.0};
        if (i == j) A[t].y = 0.0;  // the diagonal of a Hermitian matrix is real
    }
}

// Scale matrix b by 2^-e[b] so that its largest |Re| or |Im| lies in [1, 2): exact, and the
// sums of squares of the convergence test neither overflow nor underflow (LAPACK scales
// likewise). The eigenvalues are scaled back by 2^e[b]; the eigenvectors do not change.
// One block per matrix.
__global__ void jac_scale(int N, zc *__restrict__ A, int *__restrict__ expo) {
    const int b = blockIdx.x;
    zc *a = A + (int64_t)b * N * N;
    double m = 0.0;
    for (int64_t e = threadIdx.x; e < (int64_t)N * N; e += blockDim.x) m = fmax(m, fmax(fabs(a[e].x), fabs(a[e].y)));
    __shared__ double sm[32];
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    m = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmax(m, sm[w]);
    const int ex = (m > 0.0 && m < INFINITY) ? ilogb(m) : 0;  // NaN or Inf: left to the test
    if (threadIdx.x == 0) expo[b] = ex;
    if (ex == 0) return;
    for (int64_t e = threadIdx.x; e < (int64_t)N * N; e += blockDim.x) {
        a[e].x = ldexp(a[e].x, -ex);
        a[e].y = ldexp(a[e].y, -ex);
    }
}

// done[b]: 0 active, 1 converged, 2 not finite (stops; reported as not converged).
// One block per matrix; counts the active matrices into *active.
__global__ void jac_check(int N, const zc *__restrict__ A, int *__restrict__ done, int *__restrict__ active) {
    const int b = blockIdx.x;
    if (done[b]) return;
    const zc *a = A + (int64_t)b * N * N;
    double off = 0.0, tot = 0.0;
    for (int64_t e = threadIdx.x; e < (int64_t)N * N; e += blockDim.x) {
        const zc v = a[e];
        const double w = v.x * v.x + v.y * v.y;
        tot += w;
        if (e % N != e / N) off += w;
    }
    __shared__ double so[32], st[32];
    for (int o = 16; o; o >>= 1) {
        off += __shfl_xor_sync(0xffffffffu, off, o);
        tot += __shfl_xor_sync(0xffffffffu, tot, o);
    }
    if ((threadIdx.x & 31) == 0) {
        so[threadIdx.x >> 5] = off;
        st[threadIdx.x >> 5] = tot;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        off = 0.0;
        tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            off += so[w];
            tot += st[w];
        }
        const double ne = (double)N * 2.220446049250313e-16;
        int d = 0;
        if (!(off < INFINITY) || !(tot < INFINITY)) d = 2;  // NaN or Inf entries
        else if (off <= ne * ne * tot) d = 1;
        done[b] = d;
        if (d == 0) atomicAdd(active, 1);
    }
}

__global__ void jac_params(int N, int M, int r, int batch, const zc *__restrict__ A, const int *__restrict__ done,
                           JacPair *__restrict__ pairs, JacRow *__restrict__ rows) {
    const int S = M / 2;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= S * batch) return;
    const int b = t / S, i = t - b * S;
    if (done[b]) return;
    int p, q;
    jac_slot(M, r, i, p, q);
    const zc *a = A + (int64_t)b * N * N;
    JacPair P;
    P.p = p;
    P.q = q;
    P.c = 1.0;
    P.s = 0.0;
    P.phx = 1.0;
    P.phy = 0.0;
    JacRow *R = rows + (int64_t)b * M;
    if (q >= N) {  // p has no partner among these rotations (odd N)
        P.app = a[p + (int64_t)p * N].x;
        P.aqq = 0.0;
        pairs[t] = P;
        R[p] = JacRow{1.0, 0.0, 0.0, p};
        return;
    }
    const double app = a[p + (int64_t)p * N].x, aqq = a[q + (int64_t)q * N].x;
    const zc apq = a[p + (int64_t)q * N];
    const double mag = hypot(apq.x, apq.y);
    P.app = app;
    P.aqq = aqq;
    if (mag > 0.0) {
        // R = [[c, s], [-s, c]] diagonalises [[app, mag], [mag, aqq]]: t = tan(theta) is the
        // smaller root of t^2 + 2 tau t - 1 = 0, tau = (aqq - app) / (2 mag)
        const double tau = (aqq - app) / (2.0 * mag);
        const double tt = fabs(tau) > 1e150 ? 0.5 / tau : copysign(1.0, tau) / (fabs(tau) + sqrt(1.0 + tau * tau));
        const double c = 1.0 / sqrt(1.0 + tt * tt);
        P.c = c;
        P.s = tt * c;
        P.phx = apq.x / mag;
        P.phy = apq.y / mag;
        P.app = app - tt * mag;
        P.aqq = aqq + tt * mag;
    }
    pairs[t] = P;
    // J = [[c, s ph], [-s conj(ph), c]] on (p, q);  J^H rows: p <- c p - s ph q, q <- c q + s conj(ph) p
    R[p] = JacRow{P.c, -P.s * P.phx, -P.s * P.phy, q};
    R[q] = JacRow{P.c, P.s * P.phx, -P.s * P.phy, p};
}

// grid (ceil(S / groups), batch), JAC_THREADS threads in groups of G; shared: groups x 2N complex
__global__ void __launch_bounds__(JAC_THREADS) jac_rotate(int N, int M, int G, zc *__restrict__ A, zc *__restrict__ Z,
                                                           const int *__restrict__ done,
                                                           const JacPair *__restrict__ pairs,
                                                           const JacRow *__restrict__ rows) {
    extern __shared__ zc jsm[];
    const int S = M / 2, groups = JAC_THREADS / G;
    const int b = blockIdx.y;
    if (done[b]) return;
    const int gi = threadIdx.x / G, lt = threadIdx.x - gi * G;
    const int slot = blockIdx.x * groups + gi;
    const bool have = slot < S;
    zc *a = A + (int64_t)b * N * N, *z = Z + (int64_t)b * N * N;
    zc *cp = jsm + (int64_t)gi * 2 * N, *cq = cp + N;
    JacPair P{};
    if (have) P = pairs[(int64_t)b * S + slot];
    const bool two = have && P.q < N;
    // A J and Z J on columns p, q:  p' = c p - s conj(ph) q,  q' = c q + s ph p
    const zc wp = zc{-P.s * P.phx, P.s * P.phy}, wq = zc{P.s * P.phx, P.s * P.phy};
    if (have) {
        zc *ap = a + (int64_t)P.p * N, *aq = a + (int64_t)P.q * N;
        zc *zp = z + (int64_t)P.p * N, *zq = z + (int64_t)P.q * N;
        for (int j = lt; j < N; j += G) {
            if (two) {
                const zc x = ap[j], y = aq[j];
                zc u = P.c * x, v = P.c * y;
                cfma(u, wp, y);
                cfma(v, wq, x);
                cp[j] = u;
                cq[j] = v;
                const zc zx = zp[j], zy = zq[j];
                zc zu = P.c * zx, zv = P.c * zy;
                cfma(zu, wp, zy);
                cfma(zv, wq, zx);
                zp[j] = zu;
                zq[j] = zv;
            } else {
                cp[j] = ap[j];
            }
        }
    }
    __syncthreads();
    if (!have) return;
    // J^H (A J) on the staged columns, every row j with its own pair's coefficients
    const JacRow *R = rows + (int64_t)b * M;
    zc *ap = a + (int64_t)P.p * N, *aq = a + (int64_t)P.q * N;
    for (int j = lt; j < N; j += G) {
        const JacRow w = R[j];
        const zc bw = zc{w.bx, w.by};
        zc u = w.c * cp[j];
        cfma(u, bw, cp[w.partner]);
        if (j == P.p) u = zc{P.app, 0.0};
        else if (two && j == P.q) u = zc{0.0, 0.0};
        ap[j] = u;
        if (two) {
            zc v = w.c * cq[j];
            cfma(v, bw, cq[w.partner]);
            if (j == P.q) v = zc{P.aqq, 0.0};
            else if (j == P.p) v = zc{0.0, 0.0};
            aq[j] = v;
        }
    }
}

// eigenvalues ascending (ties and non-finite values in index order, NaN last) and the rank of
// every diagonal entry; one block per matrix
__global__ void jac_sort(int N, const zc *__restrict__ A, const int *__restrict__ expo, double *__restrict__ E,
                         int *__restrict__ rank) {
    extern __shared__ double dk[];
    const int b = blockIdx.x;
    const zc *a = A + (int64_t)b * N * N;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const double d = a[i + (int64_t)i * N].x;
        dk[i] = d;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const double di = dk[i];
        const double ki = isnan(di) ? INFINITY : di;
        const bool ni = isnan(di);
        int k = 0;
        for (int j = 0; j < N; j++) {
            const double dj = dk[j];
            const bool nj = isnan(dj);
            const double kj = nj ? INFINITY : dj;
            // order: (key, NaN after finite/inf, index)
            const bool before = kj < ki || (kj == ki && (nj < ni || (nj == ni && j < i)));
            k += before;
        }
        rank[(int64_t)b * N + i] = k;
        E[(int64_t)b * N + k] = ldexp(di, expo[b]);
    }
}

__global__ void jac_permute(int N, int64_t total, const zc *__restrict__ Z, const int *__restrict__ rank,
                            zc *__restrict__ V) {
    const int64_t nn = (int64_t)N * N;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = t / nn, e = t - b * nn;
        const int i = (int)(e % N), j = (int)(e / N);
        V[b * nn + i + (int64_t)rank[b * N + j] * N] = Z[t];
    }
}

int grid_for(int64_t total) { return (int)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 148 * 16)); }

// Jacobi on `batch` matrices of order N in dA (device, overwritten: eigenvectors in the
// columns, ascending), eigenvalues into dE. dinfo[b] = 0, or 1 for a matrix that did not
// converge (or held non-finite entries). dW: N*N*batch complex workspace (the rotated
// eigenvectors). Runs on `st`; returns a CUDA error code.
cudaError_t eigh_dev(cudaStream_t st, int N, int batch, zc *dA, double *dE, int *dinfo, zc *dW) {
    const int M = N + (N & 1), S = M / 2;
    const int64_t total = (int64_t)N * N * batch;
    int *dflag = nullptr, *dact = nullptr, *drank = nullptr, *dexpo = nullptr;
    JacPair *dpairs = nullptr;
    JacRow *drows = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaError_t e;
    int G = 32;
    while (G < N && G < JAC_THREADS) G *= 2;
    const int groups = JAC_THREADS / G;
    const size_t smem = sizeof(zc) * 2 * (size_t)N * groups;
    const dim3 rgrid((S + groups - 1) / groups, batch);
    const int pgrid = (S * batch + 127) / 128;
    int active = 0, sweeps = 0;
    std::vector<int> hflag(batch);
#define JAC_TRY(x)                          \
    do {                                    \
        if ((e = (x)) != cudaSuccess) goto out; \
    } while (0)
    JAC_TRY(setup_alloc((void **)&dflag, sizeof(int) * (2 * batch + 1), st));
    dact = dflag + batch;
    dexpo = dact + 1;
    JAC_TRY(setup_alloc((void **)&drank, sizeof(int) * (size_t)N * batch, st));
    JAC_TRY(setup_alloc((void **)&dpairs, sizeof(JacPair) * (size_t)S * batch, st));
    JAC_TRY(setup_alloc((void **)&drows, sizeof(JacRow) * (size_t)M * batch, st));
    JAC_TRY(smem_cap((const void *)jac_rotate));
    JAC_TRY(smem_cap((const void *)jac_sort));
    JAC_TRY(cudaMemsetAsync(dflag, 0, sizeof(int) * (batch + 1), st));
    jac_init<<<grid_for(total), 256, 0, st>>>(N, total, dA, dW);
    count_launch();
    jac_scale<<<batch, 256, 0, st>>>(N, dA, dexpo);
    count_launch();
    jac_check<<<batch, 256, 0, st>>>(N, dA, dflag, dact);
    count_launch();
    JAC_TRY(cudaGetLastError());
    JAC_TRY(cudaMemcpyAsync(&active, dact, sizeof(int), cudaMemcpyDeviceToHost, st));
    JAC_TRY(cudaStreamSynchronize(st));
    if (active > 0) {
        // one sweep: M-1 rounds, then the convergence test of every matrix still active
        JAC_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        for (int r = 0; r < M - 1; r++) {
            jac_params<<<pgrid, 128, 0, st>>>(N, M, r, batch, dA, dflag, dpairs, drows);
            jac_rotate<<<rgrid, JAC_THREADS, smem, st>>>(N, M, G, dA, dW, dflag, dpairs, drows);
        }
        cudaMemsetAsync(dact, 0, sizeof(int), st);
        jac_check<<<batch, 256, 0, st>>>(N, dA, dflag, dact);
        e = cudaStreamEndCapture(st, &graph);
        if (e != cudaSuccess) goto out;
        JAC_TRY(cudaGraphInstantiate(&exec, graph, 0));
        while (active > 0 && sweeps < JAC_MAX_SWEEPS) {
            JAC_TRY(cudaGraphLaunch(exec, st));
            for (int k = 0; k < 2 * (M - 1) + 1; k++) count_launch();
            JAC_TRY(cudaMemcpyAsync(&active, dact, sizeof(int), cudaMemcpyDeviceToHost, st));
            JAC_TRY(cudaStreamSynchronize(st));
            sweeps++;
        }
    }
    jac_sort<<<batch, 256, sizeof(double) * N, st>>>(N, dA, dexpo, dE, drank);
    count_launch();
    jac_permute<<<grid_for(total), 256, 0, st>>>(N, total, dW, drank, dA);
    count_launch();
    JAC_TRY(cudaGetLastError());
    JAC_TRY(cudaMemcpyAsync(hflag.data(), dflag, sizeof(int) * batch, cudaMemcpyDeviceToHost, st));
    JAC_TRY(cudaStreamSynchronize(st));
    for (int b = 0; b < batch; b++) hflag[b] = hflag[b] == 1 ? 0 : 1;
    JAC_TRY(cudaMemcpyAsync(dinfo, hflag.data(), sizeof(int) * batch, cudaMemcpyHostToDevice, st));
    JAC_TRY(cudaStreamSynchronize(st));
out:
#undef JAC_TRY
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        cudaStreamCaptureStatus cs;
        if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(st, &g);
            if (g) cudaGraphDestroy(g);
        }
    }
    if (dflag) cudaFreeAsync(dflag, st);
    if (drank) cudaFreeAsync(drank, st);
    if (dpairs) cudaFreeAsync(dpairs, st);
    if (drows) cudaFreeAsync(drows, st);
    cudaStreamSynchronize(st);
    return e;
}

// ---- eigenvalues only: one block per matrix, the matrix in shared memory ----
// Two phases, both inside one launch:
//  1. Householder reduction to a real tridiagonal matrix, with zhetd2's reflectors
//     H = I - tau v v^H (v(1) = 1, beta real, tau and v as zlarfg forms them) applied as
//     A22 <- A22 - v w^H - w v^H, w = p - (tau/2)(p^H v) v, p = tau A22 v. The lower triangle
//     is packed by columns, (i, j) with i >= j at col(j) + i - j, so N <= 160 fits one
//     block's shared memory; the trailing matrix-vector product runs as G x m thread
//     partials (no atomics, a fixed summation order), the rank-2 update one warp per column,
//     and warp 0 forms the next reflector as soon as its column is updated (four block
//     barriers per column). Shared-memory bandwidth bounds this phase: every step reads the
//     trailing matrix twice (Hermitian, one triangle stored) and updates it once.
//  2. The eigenvalues of the tridiagonal matrix (d, e^2) by Sturm counts (tv_count): one count
//     per thread at 512 points of the Gershgorin interval brackets every eigenvalue, then
//     G threads per eigenvalue split its bracket into G + 1 parts per step until the bracket
//     is 2 eps ||T|| wide. A diagonal entry isolated by zero couplings is an eigenvalue as it
//     stands and is returned exactly (a diagonal matrix gives its own entries).
// Results are deterministic: every sum has a fixed order.
constexpr int TV_MAX_N = 160, TV_THREADS = 512, TV_WARPS = TV_THREADS / 32;

__device__ __forceinline__ int tv_col(int j, int N) { return j * N - j * (j - 1) / 2; }

// The number of eigenvalues of the tridiagonal (d, e2) below the shift s: the sign changes of
// the leading principal minors of T - s, p_0 = d_0 - s, p_i = (d_i - s) p_{i-1} - e_{i-1}^2 p_{i-2}
// (p_{-1} = 1), that is the negative pivots q_i = p_i / p_{i-1} of T - s = L D L^T, without a
// division per step. A minor that vanishes (exactly, or by underflow) is replaced by
// -2^-100 p_{i-1}, a negative pivot, as dstebz replaces a pivot |q| <= pivmin by -pivmin; the
// sign tests read the sign bits (integer operations). After every fourth step the pair
// (p_i, p_{i-1}) is rescaled by a power of two into 2^-300 .. 2^300 (exact, signs unchanged);
// with the matrix scaled to entries below 2, four steps stay far inside the double range. Per
// step this is one FMA on the dependence chain instead of a division (measured on B200: ~120
// cycles per step with 15 warps counting, against ~226 for the division form).
__device__ __forceinline__ int tv_count(const double *d, const double *e2, int N, double s) {
    double pc = d[0] - s, pm = 1.0;
    if (pc == 0.0) pc = -0x1p-100;
    int c = (int)((unsigned long long)__double_as_longlong(pc) >> 63);
    auto step = [&](double di, double ei) {
        double pn = fma(di - s, pc, -ei * pm);
        const double tiny = -0x1p-100 * pc;  // off the dependence chain
        if (pn == 0.0) pn = tiny;
        c += (int)((unsigned long long)(__double_as_longlong(pn) ^ __double_as_longlong(pc)) >> 63);
        pm = pc;
        pc = pn;
    };
    int i = 1;
    for (; i + 3 < N; i += 4) {
        const double d0 = d[i], d1 = d[i + 1], d2 = d[i + 2], d3 = d[i + 3];
        const double e0 = e2[i - 1], e1 = e2[i], f2 = e2[i + 1], f3 = e2[i + 2];
        step(d0, e0);
        step(d1, e1);
        step(d2, f2);
        step(d3, f3);
        const double mx = fmax(fabs(pc), fabs(pm));
        const double f = mx > 0x1p300 ? 0x1p-300 : (mx < 0x1p-300 ? 0x1p300 : 1.0);
        pc *= f;
        pm *= f;
    }
    for (; i < N; i++) step(d[i], e2[i - 1]);
    return c;
}

inline size_t tv_smem(int N) {
    return sizeof(zc) * ((size_t)N * (N + 1) / 2 + 3 * (size_t)N + TV_THREADS) + sizeof(double) * 3 * (size_t)N;
}

// reflector k (zlarfg on column k below the diagonal), by one warp: d_k, e_k^2, tau and scale, and
// v = (1, x / (alpha - beta)) into vk; tau = 0 when there is nothing to annihilate (H = I)
__device__ __forceinline__ void tv_reflector(const zc *L, int N, int k, double *d, double *e2, zc *tau_s, zc *vk) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, m = N - k - 1;
    const zc *col = L + tv_col(k, N);  // col[0] = L(k, k), col[1 + i] = L(k + 1 + i, k)
    double xn = 0.0;
    for (int i = 1 + lane; i < m; i += 32) xn += col[1 + i].x * col[1 + i].x + col[1 + i].y * col[1 + i].y;
    for (int o = 16; o; o >>= 1) xn += __shfl_xor_sync(FULL, xn, o);
    xn = __shfl_sync(FULL, xn, 0);  // one value for every lane
    const zc al = col[1];
    zc t{0.0, 0.0}, sc{0.0, 0.0};
    double ee = al.x * al.x + al.y * al.y;
    if (!(m == 1 || (xn == 0.0 && al.y == 0.0))) {
        const double beta = -copysign(sqrt(ee + xn), al.x);
        const double zx = al.x - beta, zz = zx * zx + al.y * al.y;  // |alpha - beta|^2 >= beta^2 > 0
        const double rb = 1.0 / beta, rz = 1.0 / zz;
        t = zc{(beta - al.x) * rb, -al.y * rb};
        sc = zc{zx * rz, -al.y * rz};  // 1 / (alpha - beta)
        ee = beta * beta;
        for (int i = lane; i < m; i += 32) vk[i] = (i == 0) ? zc{1.0, 0.0} : col[1 + i] * sc;
    }
    if (lane == 0) {
        d[k] = col[0].x;
        e2[k] = ee;
        *tau_s = t;
    }
}

__global__ void __launch_bounds__(TV_THREADS, 1) tri_values(int N, const zc *__restrict__ A, double *__restrict__ E,
                                                        int *__restrict__ info) {
    extern __shared__ __align__(16) unsigned char tv_raw[];
    const int np = N * (N + 1) / 2;
    zc *L = (zc *)tv_raw;    // packed lower triangle
    zc *v = L + np;          // the reflectors k and k + 1 (two buffers)
    zc *w = v + 2 * N;       // w of the rank-2 update
    zc *part = w + N;        // the matrix-vector partials; the 512 Sturm counts of the bracketing pass
    double *d = (double *)(part + TV_THREADS), *e2 = d + N, *ev = e2 + N;
    __shared__ double red[TV_WARPS][2];
    __shared__ zc tau_s[2];
    __shared__ double glo_s, ghi_s, piv_s, tol_s;
    __shared__ int ex_s, bad_s;
    const unsigned FULL = 0xffffffffu;
    const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const zc *a = A + (int64_t)b * N * N;
    // L(j, i) = conj(A(i, j)) from the upper triangle (i < j), the diagonal's real part
    {
        double m = 0.0;
        int bad = 0;
        for (int e = tid; e < N * N; e += TV_THREADS) {
            const int i = e % N, j = e / N;
            if (i > j) continue;
            const zc x = a[e];
            const zc y = (i == j) ? zc{x.x, 0.0} : zc{x.x, -x.y};
            L[tv_col(i, N) + j - i] = y;
            bad |= !(isfinite(y.x) && isfinite(y.y));
            m = fmax(m, fmax(fabs(y.x), fabs(y.y)));
        }
        for (int o = 16; o; o >>= 1) {
            m = fmax(m, __shfl_xor_sync(FULL, m, o));
            bad |= __shfl_xor_sync(FULL, bad, o);
        }
        if (lane == 0) {
            red[warp][0] = m;
            red[warp][1] = bad;
        }
        __syncthreads();
        if (tid == 0) {
            double mm = 0.0;
            int bb = 0;
            for (int q = 0; q < TV_WARPS; q++) {
                mm = fmax(mm, red[q][0]);
                bb |= red[q][1] != 0.0;
            }
            // scale by 2^-ex so that the largest |Re| or |Im| lies in [1, 2), as LAPACK scales
            ex_s = (mm > 0.0 && mm < INFINITY) ? ilogb(mm) : 0;
            bad_s = bb;
            info[b] = bb;  // non-finite entries: info = 1, no eigenvalues
        }
        __syncthreads();
        if (bad_s) {
            for (int i = tid; i < N; i += TV_THREADS) E[(int64_t)b * N + i] = NAN;
            return;
        }
        if (ex_s != 0)
            for (int e = tid; e < np; e += TV_THREADS) L[e] = zc{ldexp(L[e].x, -ex_s), ldexp(L[e].y, -ex_s)};
        __syncthreads();
    }
    // phase 1: reflector k annihilates column k below the subdiagonal. Warp 0 forms reflector
    // k + 1 as soon as it has updated column k + 1, while the other warps finish the update of
    // step k (v and tau alternate between two buffers).
    if (warp == 0 && N > 1) tv_reflector(L, N, 0, d, e2, &tau_s[0], v);
    __syncthreads();
    for (int k = 0; k + 1 < N; k++) {
        const int s = k + 1, m = N - s;
        const zc t = tau_s[k & 1];
        const zc *vk = v + (k & 1) * N;
        zc *vn = v + ((k + 1) & 1) * N;
        const bool next = k + 2 < N;  // reflector k + 1 exists
        if (t.x == 0.0 && t.y == 0.0) {
            if (warp == 0 && next) tv_reflector(L, N, k + 1, d, e2, &tau_s[(k + 1) & 1], vn);
            __syncthreads();
            continue;
        }
        // partials of A22 v: thread (g, i) sums the columns j = g (mod G) of row i
        const int G = min(16, TV_THREADS / m);
        if (tid < G * m) {
            const int i = tid % m, g = tid / m, I = s + i;
            zc a0{0.0, 0.0}, a1{0.0, 0.0};  // two accumulators: shorter dependence chains
            int j = g;
            for (; j + G <= i; j += 2 * G) {  // row i of the lower part
                cfma(a0, L[tv_col(s + j, N) + i - j], vk[j]);
                cfma(a1, L[tv_col(s + j + G, N) + i - j - G], vk[j + G]);
            }
            if (j <= i) {
                cfma(a0, L[tv_col(s + j, N) + i - j], vk[j]);
                j += G;
            }
            const zc *ci = L + tv_col(I, N) - i;  // ci[j] = L(s + j, I), j > i
            for (; j + G < m; j += 2 * G) {
                cfma(a0, conj(ci[j]), vk[j]);
                cfma(a1, conj(ci[j + G]), vk[j + G]);
            }
            if (j < m) cfma(a0, conj(ci[j]), vk[j]);
            part[g * m + i] = a0 + a1;
        }
        __syncthreads();
        // p = tau A22 v, the dot p^H v, w = p - (tau / 2)(p^H v) v
        zc p{0.0, 0.0};
        double dx = 0.0, dy = 0.0;
        if (tid < m) {
            zc acc = part[tid];
            for (int g = 1; g < G; g++) acc = acc + part[g * m + tid];
            p = t * acc;
            const zc vi = vk[tid];
            dx = p.x * vi.x + p.y * vi.y;
            dy = p.x * vi.y - p.y * vi.x;
        }
        for (int o = 16; o; o >>= 1) {
            dx += __shfl_xor_sync(FULL, dx, o);
            dy += __shfl_xor_sync(FULL, dy, o);
        }
        if (lane == 0) {
            red[warp][0] = dx;
            red[warp][1] = dy;
        }
        __syncthreads();
        if (tid < m) {
            double rx[TV_WARPS], ry[TV_WARPS];  // pairwise sum of the warps' parts
#pragma unroll
            for (int q = 0; q < TV_WARPS; q++) {
                rx[q] = red[q][0];
                ry[q] = red[q][1];
            }
#pragma unroll
            for (int h = TV_WARPS / 2; h; h >>= 1)
#pragma unroll
                for (int q = 0; q < h; q++) {
                    rx[q] += rx[q + h];
                    ry[q] += ry[q + h];
                }
            const zc aw{-0.5 * (t.x * rx[0] - t.y * ry[0]), -0.5 * (t.x * ry[0] + t.y * rx[0])};
            w[tid] = p + aw * vk[tid];
        }
        __syncthreads();
        // A22 -= v w^H + w v^H on the lower triangle, one warp per column, the diagonal kept real;
        // warp 0 updates column k + 1 alone and forms its reflector, warps 1.. the other columns
        for (int j = warp; j < m; j += (warp == 0 ? m : TV_WARPS - 1)) {
            zc *cj = L + tv_col(s + j, N) - j;  // cj[i] = L(s + i, s + j), i >= j
            const zc vj = conj(vk[j]), wj = conj(w[j]);
#pragma unroll 2
            for (int i = j + lane; i < m; i += 32) {
                zc x = cj[i] - vk[i] * wj - w[i] * vj;
                if (i == j) x.y = 0.0;
                cj[i] = x;
            }
            if (j == 0 && next) {  // column k + 1 is final: its reflector
                __syncwarp();
                tv_reflector(L, N, k + 1, d, e2, &tau_s[(k + 1) & 1], vn);
            }
        }
        __syncthreads();
    }
    if (tid == 0) d[N - 1] = L[tv_col(N - 1, N)].x;
    __syncthreads();
    // phase 2: Gershgorin interval, pivmin (dstebz: the underflow threshold x max(1, max e^2))
    if (warp == 0) {
        double lo = INFINITY, hi = -INFINITY, me = 0.0;
        for (int i = lane; i < N; i += 32) {
            const double r = (i > 0 ? sqrt(e2[i - 1]) : 0.0) + (i + 1 < N ? sqrt(e2[i]) : 0.0);
            lo = fmin(lo, d[i] - r);
            hi = fmax(hi, d[i] + r);
            if (i + 1 < N) me = fmax(me, e2[i]);
        }
        for (int o = 16; o; o >>= 1) {
            lo = fmin(lo, __shfl_xor_sync(FULL, lo, o));
            hi = fmax(hi, __shfl_xor_sync(FULL, hi, o));
            me = fmax(me, __shfl_xor_sync(FULL, me, o));
        }
        if (lane == 0) {
            const double eps = 2.220446049250313e-16, tn = fmax(fabs(lo), fabs(hi));
            const double pv = 2.2250738585072014e-308 * fmax(1.0, me);
            const double widen = 2.0 * N * eps * tn + 2.0 * pv;
            glo_s = lo - widen;
            ghi_s = hi + widen;
            piv_s = pv;
            tol_s = 2.0 * eps * tn + 4.0 * pv;
        }
    }
    __syncthreads();
    const double glo = glo_s, ghi = ghi_s, pv = piv_s, tol = tol_s;
    // one count per thread at 512 points of the Gershgorin interval brackets every eigenvalue;
    // then G threads per eigenvalue (32 / G eigenvalues per warp) split its bracket into G + 1
    // parts per step
    int *cnt = (int *)part;
    const double step0 = (ghi - glo) / (TV_THREADS + 1);
    cnt[tid] = tv_count(d, e2, N, glo + step0 * (tid + 1));
    __syncthreads();
    int G = 32;
    while (G > 1 && TV_WARPS * (32 / G) < N) G--;
    const int per = 32 / G, slot = lane / G, r = lane % G;
    const int kk = warp * per + slot;
    const bool own = slot < per && kk < N;
    const int k = own ? kk : N - 1;
    double lo = glo, hi = ghi;
    for (int q = 0; q < TV_THREADS; q++) {
        const double sq = glo + step0 * (q + 1);
        if (cnt[q] <= k) lo = fmax(lo, sq);
        else hi = fmin(hi, sq);
    }
    // the same number of steps for every group (the shuffles need all lanes)
    int iters = 0;
    for (double wd = step0; wd > tol && iters < 80; wd /= (G + 1)) iters++;
    const int base = min(slot * G, 32 - G);
    for (int it = 0; it < iters; it++) {
        const double sg = lo + (hi - lo) * (double)(r + 1) / (double)(G + 1);
        const int c = tv_count(d, e2, N, sg);
        double nlo = lo, nhi = hi;
        for (int q = 0; q < G; q++) {
            const double sq = __shfl_sync(FULL, sg, base + q);
            const int cq = __shfl_sync(FULL, c, base + q);
            if (cq <= k) nlo = fmax(nlo, sq);
            else nhi = fmin(nhi, sq);
        }
        lo = nlo;
        hi = nhi;
    }
    if (own && r == 0) {
        // an isolated diagonal entry within the tolerance is the eigenvalue itself (the pivmin
        // guard counts s = d_i as above d_i, so the bracket may end a pivmin short of it)
        const double mid = 0.5 * (lo + hi);
        double lam = mid, best = tol;
        for (int i = 0; i < N; i++)
            if ((i == 0 || e2[i - 1] == 0.0) && (i + 1 == N || e2[i] == 0.0) && fabs(d[i] - mid) <= best) {
                best = fabs(d[i] - mid);
                lam = d[i];
            }
        ev[k] = lam;
    }
    __syncthreads();
    // ascending order (brackets of nearly equal eigenvalues may overlap)
    for (int i = tid; i < N; i += TV_THREADS) {
        const double x = ev[i];
        int rank = 0;
        for (int j = 0; j < N; j++) rank += ev[j] < x || (ev[j] == x && j < i);
        E[(int64_t)b * N + rank] = ldexp(x, ex_s);
    }
}

// ---- Loewdin transform ----

// C = alpha A op(B) + beta C, complex FP64, column-major, op(B) = B or B^H; 64x64 tiles of C,
// 256 threads with a 4x4 block each (the set-up's few products; not on the SCF path)
constexpr int GT = 64, GK = 8;
__global__ void __launch_bounds__(256) zgemm_small(int m, int n, int k, const zc *__restrict__ A, int lda,
                                                  const zc *__restrict__ B, int ldb, bool conjB, zc *__restrict__ C,
                                                  int ldc, double alpha, double beta) {
    __shared__ zc As[GK][GT + 1], Bs[GK][GT + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int i0 = blockIdx.x * GT, j0 = blockIdx.y * GT;
    zc acc[4][4] = {};
    for (int k0 = 0; k0 < k; k0 += GK) {
        for (int e = threadIdx.x; e < GK * GT; e += 256) {
            {  // A(i0 + ii, k0 + kk): ii fastest, down a column
                const int kk = e / GT, ii = e % GT, gi = i0 + ii, gk = k0 + kk;
                As[kk][ii] = (gi < m && gk < k) ? A[gi + (int64_t)gk * lda] : zc{0.0, 0.0};
            }
            if (conjB) {  // B^H(k, j) = conj(B(j, k)): j fastest
                const int kk = e / GT, jj = e % GT, gj = j0 + jj, gk = k0 + kk;
                Bs[kk][jj] = (gj < n && gk < k) ? conj(B[gj + (int64_t)gk * ldb]) : zc{0.0, 0.0};
            } else {      // B(k, j): k fastest
                const int kk = e % GK, jj = e / GK, gj = j0 + jj, gk = k0 + kk;
                Bs[kk][jj] = (gj < n && gk < k) ? B[gk + (int64_t)gj * ldb] : zc{0.0, 0.0};
            }
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; kk++) {
            zc av[4], bv[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                av[u] = As[kk][tx + 16 * u];
                bv[u] = Bs[kk][ty + 16 * u];
            }
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int v = 0; v < 4; v++) cfma(acc[u][v], av[u], bv[v]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const int gi = i0 + tx + 16 * u, gj = j0 + ty + 16 * v;
            if (gi < m && gj < n) {
                zc *c = C + gi + (int64_t)gj * ldc;
                const zc old = beta == 0.0 ? zc{0.0, 0.0} : beta * *c;
                *c = old + alpha * acc[u][v];
            }
        }
}

void zgemm(cudaStream_t st, int m, int n, int k, const zc *A, int lda, const zc *B, int ldb, bool conjB, zc *C,
           int ldc, double alpha, double beta) {
    dim3 grid((m + GT - 1) / GT, (n + GT - 1) / GT);
    zgemm_small<<<grid, 256, 0, st>>>(m, n, k, A, lda, B, ldb, conjB, C, ldc, alpha, beta);
    count_launch();
}

// W(:,k) = Z(:,k) / ev_k^(1/4) (src/hamiltonian.f90:636-639), and the minimum eigenvalue
__global__ void lowdin_scale(int N, const double *__restrict__ ev, zc *__restrict__ Z) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N * N; t += gridDim.x * blockDim.x) {
        const int k = t / N;
        const double f = 1.0 / sqrt(sqrt(ev[k]));
        Z[t] = f * Z[t];
    }
}

// S^-1/2 for N <= 160 without eigenvectors: the coupled Newton-Schulz iteration (Higham,
// Functions of Matrices, 2008, sec. 6.7) on A = S / ev_max, whose eigenvalues lie in (0, 1]:
//   T = (3 I - Z Y) / 2,  Y <- Y T,  Z <- T Z,   Y0 = A, Z0 = I,   Z -> A^-1/2,
// so S^-1/2 = Z / sqrt(ev_max), the same matrix function that U diag(ev^-1/2) U^T forms in the
// reference (src/hamiltonian.f90:627-640). Every iterate is a polynomial in A, so each
// eigenvalue follows the scalar map and the smallest one converges last: the host runs that
// scalar map for ev_min / ev_max to fix the number of steps.
__global__ void ns_init(int N, double c, const zc *__restrict__ S, zc *__restrict__ Y, zc *__restrict__ Z) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N * N; t += gridDim.x * blockDim.x) {
        Y[t] = c * S[t];
        Z[t] = zc{(t % N == t / N) ? 1.0 : 0.0, 0.0};
    }
}
__global__ void ns_shift(int N, zc *__restrict__ T) {  // T <- (3 I - T) / 2
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N * N; t += gridDim.x * blockDim.x)
        T[t] = zc{(t % N == t / N ? 1.5 : 0.0) - 0.5 * T[t].x, -0.5 * T[t].y};
}
// Smh = f (Z + Z^T) / 2, real (S is real); one thread per pair i <= j, so Smh may be Z
__global__ void ns_final(int N, double f, const zc *Z, zc *Smh) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N * N; t += gridDim.x * blockDim.x) {
        const int i = t % N, j = t / N;
        if (i > j) continue;
        const double v = 0.5 * f * (Z[i + (int64_t)j * N].x + Z[j + (int64_t)i * N].x);
        Smh[i + (int64_t)j * N] = zc{v, 0.0};
        Smh[j + (int64_t)i * N] = zc{v, 0.0};
    }
}
static int ns_steps(double r) {  // r = ev_min / ev_max in (0, 1]
    double y = r, z = 1.0;
    int k = 0;
    while (k < 200) {
        const double t = 0.5 * (3.0 - z * y);
        y *= t;
        z *= t;
        k++;
        if (std::fabs(z * y - 1.0) <= 4e-16) break;
    }
    return k + 1;  // one more step: the error squares
}

// X2(2i+s, 2j+s) = X(i,j) (spin doubling, spin fastest; src/hamiltonian.f90:672-680)
__global__ void spin_double(int N, const zc *__restrict__ X, zc *__restrict__ X2) {
    const int No = 2 * N;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < No * No; t += gridDim.x * blockDim.x) {
        const int r = t % No, c = t / No;
        X2[t] = (r & 1) == (c & 1) ? X[(r >> 1) + (int64_t)(c >> 1) * N] : zc{0.0, 0.0};
    }
}

// y += a x
__global__ void zaxpy_k(int64_t n, double a, const zc *__restrict__ x, zc *__restrict__ y) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        y[t] = y[t] + a * x[t];
}

__global__ void real_to_complex(int64_t n, const double *__restrict__ x, zc *__restrict__ z) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        z[t] = zc{x[t], 0.0};
}

// H = (Hn + Hn^H) / 2 (src/hamiltonian.f90:689)
__global__ void hermitize(int n, const zc *__restrict__ Hn, zc *__restrict__ H) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n * n; t += gridDim.x * blockDim.x) {
        const int i = t % n, j = t / n;
        H[t] = 0.5 * (Hn[t] + conj(Hn[j + (int64_t)i * n]));
    }
}

// makes `device` current for the scope of a call (device < 0: leaves the current one)
struct DeviceScope {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceScope(int device) {
        if (device < 0) return;
        if ((err = cudaGetDevice(&prev)) == cudaSuccess) err = cudaSetDevice(device);
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace
}  // namespace qs

using namespace qs;

extern "C" {

int qs_hermitian_eigensystem(int N, int batch, double *A, double *E, int *info, int device) {
    if (N < 1 || N > JAC_MAX_N || batch < 0 || batch > 65535 || (batch > 0 && (!A || !E))) return -1;
    if (batch == 0) return 0;
    DeviceScope ds(device);
    if (ds.err != cudaSuccess) return -(int)ds.err;
    const size_t nn = (size_t)N * N * batch;
    cudaStream_t st = nullptr;
    zc *dA = nullptr, *dW = nullptr;
    double *dE = nullptr;
    int *dinfo = nullptr;
    std::vector<int> hinfo(batch, 0);
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return -(int)e;
    if ((e = setup_alloc((void **)&dA, sizeof(zc) * nn, st)) == cudaSuccess &&
        (e = setup_alloc((void **)&dW, sizeof(zc) * nn, st)) == cudaSuccess &&
        (e = setup_alloc((void **)&dE, sizeof(double) * (size_t)N * batch, st)) == cudaSuccess &&
        (e = setup_alloc((void **)&dinfo, sizeof(int) * batch, st)) == cudaSuccess &&
        (e = cudaMemcpyAsync(dA, A, sizeof(zc) * nn, cudaMemcpyHostToDevice, st)) == cudaSuccess &&
        (e = eigh_dev(st, N, batch, dA, dE, dinfo, dW)) == cudaSuccess &&
        (e = cudaMemcpyAsync(A, dA, sizeof(zc) * nn, cudaMemcpyDeviceToHost, st)) == cudaSuccess &&
        (e = cudaMemcpyAsync(E, dE, sizeof(double) * (size_t)N * batch, cudaMemcpyDeviceToHost, st)) == cudaSuccess &&
        (e = cudaMemcpyAsync(hinfo.data(), dinfo, sizeof(int) * batch, cudaMemcpyDeviceToHost, st)) == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (dA) cudaFreeAsync(dA, st);
    if (dW) cudaFreeAsync(dW, st);
    if (dE) cudaFreeAsync(dE, st);
    if (dinfo) cudaFreeAsync(dinfo, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (e != cudaSuccess) return -(int)e;
    int bad = 0;
    for (int b = 0; b < batch; b++) {
        if (info) info[b] = hinfo[b];
        bad |= hinfo[b];
    }
    return bad ? 1 : 0;
}

// N <= 160: one buffer [A | E | info], one launch of tri_values and one copy back, on the
// calling thread's stream (the program calls this once, for the energy grid)
static int eigenvalues_small(int N, int batch, const double *A, double *E, int *info) {
    cudaStream_t st = cudaStreamPerThread;
    const size_t bA = sizeof(zc) * (size_t)N * N * batch, bE = sizeof(double) * (size_t)N * batch;
    const size_t bI = sizeof(int) * (size_t)batch;
    std::vector<unsigned char> back(bE + bI);
    unsigned char *buf = nullptr;
    cudaError_t e = setup_alloc((void **)&buf, bA + bE + bI, st);
    if (e != cudaSuccess) return -(int)e;
    if ((e = cudaMemcpyAsync(buf, A, bA, cudaMemcpyHostToDevice, st)) == cudaSuccess &&
        (e = smem_cap((const void *)tri_values)) == cudaSuccess) {
        tri_values<<<batch, TV_THREADS, tv_smem(N), st>>>(N, (const zc *)buf, (double *)(buf + bA), (int *)(buf + bA + bE));
        count_launch();
        if ((e = cudaGetLastError()) == cudaSuccess &&
            (e = cudaMemcpyAsync(back.data(), buf + bA, bE + bI, cudaMemcpyDeviceToHost, st)) == cudaSuccess)
            e = cudaStreamSynchronize(st);
    }
    cudaFreeAsync(buf, st);
    if (e != cudaSuccess) {
        cudaStreamSynchronize(st);
        return -(int)e;
    }
    std::memcpy(E, back.data(), bE);
    int bad = 0;
    for (int b = 0; b < batch; b++) {
        int v;
        std::memcpy(&v, back.data() + bE + sizeof(int) * b, sizeof(int));
        if (info) info[b] = v;
        bad |= v;
    }
    return bad ? 1 : 0;
}

int qs_hermitian_eigenvalues(int N, int batch, const double *A, double *E, int *info, int device) {
    if (N < 1 || N > JAC_MAX_N || batch < 0 || batch > 65535 || (batch > 0 && (!A || !E))) return -1;
    if (batch == 0) return 0;
    DeviceScope ds(device);
    if (ds.err != cudaSuccess) return -(int)ds.err;
    if (N <= TV_MAX_N) return eigenvalues_small(N, batch, A, E, info);
    const size_t nn = (size_t)N * N * batch;
    cudaStream_t st = nullptr;
    zc *dA = nullptr, *dW = nullptr;
    double *dE = nullptr;
    int *dinfo = nullptr;
    std::vector<int> hinfo(batch, 0);
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return -(int)e;
    if ((e = setup_alloc((void **)&dA, sizeof(zc) * nn, st)) == cudaSuccess &&
        (e = setup_alloc((void **)&dW, sizeof(zc) * nn, st)) == cudaSuccess &&
        (e = setup_alloc((void **)&dE, sizeof(double) * (size_t)N * batch, st)) == cudaSuccess &&
        (e = setup_alloc((void **)&dinfo, sizeof(int) * batch, st)) == cudaSuccess &&
        (e = cudaMemcpyAsync(dA, A, sizeof(zc) * nn, cudaMemcpyHostToDevice, st)) == cudaSuccess) {
        e = eigh_dev(st, N, batch, dA, dE, dinfo, dW);  // the eigenvectors are not used
        if (e == cudaSuccess &&
            (e = cudaMemcpyAsync(E, dE, sizeof(double) * (size_t)N * batch, cudaMemcpyDeviceToHost, st)) == cudaSuccess &&
            (e = cudaMemcpyAsync(hinfo.data(), dinfo, sizeof(int) * batch, cudaMemcpyDeviceToHost, st)) == cudaSuccess)
            e = cudaStreamSynchronize(st);
    }
    if (dA) cudaFreeAsync(dA, st);
    if (dW) cudaFreeAsync(dW, st);
    if (dE) cudaFreeAsync(dE, st);
    if (dinfo) cudaFreeAsync(dinfo, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (e != cudaSuccess) return -(int)e;
    int bad = 0;
    for (int b = 0; b < batch; b++) {
        if (info) info[b] = hinfo[b];
        bad |= hinfo[b];
    }
    return bad ? 1 : 0;
}

int qs_dftb_lowdin(int N, const double *S, const double *H0, const double *Lam, int soc_dual, double *H,
                   double *evmin, int device) {
    if (N < 1 || N > JAC_MAX_N || !S || !H0 || !Lam || !H) return -1;
    DeviceScope ds(device);
    if (ds.err != cudaSuccess) return -(int)ds.err;
    const int No = 2 * N;
    const size_t n1 = (size_t)N * N, n2 = (size_t)No * No;
    cudaStream_t st = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return -(int)e;
    zc *buf = nullptr;
    double *dR = nullptr;
    int *dinfo = nullptr;
    int rc = 0, hinfo = 0;
    std::vector<double> ev(N);
    const int gb = 148 * 8;
#define LOW_TRY(x)                          \
    do {                                    \
        if ((e = (x)) != cudaSuccess) goto out; \
    } while (0)
    // n1 blocks: S then its eigenvectors, the eigensolver's workspace, S^-1/2;
    // n2 blocks: Sm2, Lam, Hao, T, Hn.  dR: S, H0 (real), the eigenvalues of S
    LOW_TRY(setup_alloc((void **)&buf, sizeof(zc) * (3 * n1 + 5 * n2), st));
    LOW_TRY(setup_alloc((void **)&dR, sizeof(double) * (2 * n1 + N), st));
    LOW_TRY(setup_alloc((void **)&dinfo, sizeof(int), st));
    {
        zc *dS = buf, *dW = buf + n1, *dSmh = buf + 2 * n1;
        zc *dSm2 = buf + 3 * n1, *dLam = dSm2 + n2, *dHao = dLam + n2, *dT = dHao + n2, *dHn = dT + n2;
        double *dE = dR + 2 * n1;
        LOW_TRY(cudaMemcpyAsync(dR, S, sizeof(double) * n1, cudaMemcpyHostToDevice, st));
        LOW_TRY(cudaMemcpyAsync(dR + n1, H0, sizeof(double) * n1, cudaMemcpyHostToDevice, st));
        LOW_TRY(cudaMemcpyAsync(dLam, Lam, sizeof(zc) * n2, cudaMemcpyHostToDevice, st));
        // S^-1/2 = U diag(ev^-1/2) U^T (src/hamiltonian.f90:627-640): for N <= 160 the
        // eigenvalues by tri_values and the matrix function by Newton-Schulz, above by the
        // Jacobi eigenpairs
        const bool small = N <= TV_MAX_N;
        real_to_complex<<<gb, 256, 0, st>>>((int64_t)n1, dR, dS);
        count_launch();
        if (small) {
            LOW_TRY(smem_cap((const void *)tri_values));
            tri_values<<<1, TV_THREADS, tv_smem(N), st>>>(N, dS, dE, dinfo);
            count_launch();
            LOW_TRY(cudaGetLastError());
        } else {
            LOW_TRY(eigh_dev(st, N, 1, dS, dE, dinfo, dW));
        }
        LOW_TRY(cudaMemcpyAsync(ev.data(), dE, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
        LOW_TRY(cudaMemcpyAsync(&hinfo, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st));
        LOW_TRY(cudaStreamSynchronize(st));
        double mn = ev[0];
        for (int k = 1; k < N; k++) mn = std::fmin(mn, ev[k]);
        if (evmin) *evmin = mn;
        if (hinfo || !(mn > 1e-8)) {  // eigensolver failure or S not positive definite: the reference stops
            rc = 1;
            goto out;
        }
        if (small) {
            double mx = ev[0];
            for (int k = 1; k < N; k++) mx = std::fmax(mx, ev[k]);
            const int steps = ns_steps(mn / mx);
            // Y, Z and their successors, T: work blocks not yet in use (Hn, T, Hao, W)
            zc *Y = dHn, *Yn = dT, *Z = dSmh, *Zn = dHao, *Tm = dW;
            ns_init<<<gb, 256, 0, st>>>(N, 1.0 / mx, dS, Y, Z);
            count_launch();
            for (int q = 0; q < steps; q++) {
                zgemm(st, N, N, N, Z, N, Y, N, false, Tm, N, 1.0, 0.0);
                ns_shift<<<gb, 256, 0, st>>>(N, Tm);
                count_launch();
                zgemm(st, N, N, N, Y, N, Tm, N, false, Yn, N, 1.0, 0.0);
                zgemm(st, N, N, N, Tm, N, Z, N, false, Zn, N, 1.0, 0.0);
                std::swap(Y, Yn);
                std::swap(Z, Zn);
            }
            ns_final<<<gb, 256, 0, st>>>(N, 1.0 / std::sqrt(mx), Z, dSmh);
            count_launch();
        } else {
            lowdin_scale<<<gb, 256, 0, st>>>(N, dE, dS);
            count_launch();
            zgemm(st, N, N, N, dS, N, dS, N, true, dSmh, N, 1.0, 0.0);  // W W^T, W real
        }
        spin_double<<<gb, 256, 0, st>>>(N, dSmh, dSm2);
        count_launch();
        // Hao = H0 spin-doubled, plus the SOC form (src/hamiltonian.f90:670-687)
        real_to_complex<<<gb, 256, 0, st>>>((int64_t)n1, dR + n1, dW);
        count_launch();
        spin_double<<<gb, 256, 0, st>>>(N, dW, dHao);
        count_launch();
        if (soc_dual) {
            real_to_complex<<<gb, 256, 0, st>>>((int64_t)n1, dR, dW);
            count_launch();
            spin_double<<<gb, 256, 0, st>>>(N, dW, dT);  // Sx2
            count_launch();
            zgemm(st, No, No, No, dT, No, dLam, No, false, dHao, No, 0.5, 1.0);
            zgemm(st, No, No, No, dLam, No, dT, No, false, dHao, No, 0.5, 1.0);
        } else {
            zaxpy_k<<<gb, 256, 0, st>>>((int64_t)n2, 1.0, dLam, dHao);
            count_launch();
        }
        // H = Sm2 (Hao Sm2), then (H + H^H) / 2 (src/hamiltonian.f90:688-689)
        zgemm(st, No, No, No, dHao, No, dSm2, No, false, dT, No, 1.0, 0.0);
        zgemm(st, No, No, No, dSm2, No, dT, No, false, dHn, No, 1.0, 0.0);
        hermitize<<<gb, 256, 0, st>>>(No, dHn, dHao);
        count_launch();
        LOW_TRY(cudaGetLastError());
        LOW_TRY(cudaMemcpyAsync(H, dHao, sizeof(zc) * n2, cudaMemcpyDeviceToHost, st));
        LOW_TRY(cudaStreamSynchronize(st));
    }
out:
#undef LOW_TRY
    if (buf) cudaFreeAsync(buf, st);
    if (dR) cudaFreeAsync(dR, st);
    if (dinfo) cudaFreeAsync(dinfo, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (e != cudaSuccess) return -(int)e;
    return rc;
}

}  // extern "C"
