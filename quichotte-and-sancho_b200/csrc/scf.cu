// scf.cu -- the self-consistent loop on the device and the C ABI of include/qsb200.h.
//
//   qs_create      setup_storage + scf_setup_sizes + sigma2_init (src/green_functions.f90:
//                  90-190, src/scf.f90:61-68, src/self_energies.f90:91-106), with every
//                  per-energy array allocated once in HBM (admission checked first)
//   qs_solve_scf   solve_scf (src/scf.f90:78-151): fresh or continued start, Broyden over
//                  the device residual, the final sweep and its sanity check
//   residual2      scf_residual2 (src/scf.f90:158-188): equal_time_lesser + Sigma1 on the
//                  device, sigma2_compute (FFT), sweep(M_SCF2) writing F = pack(G_out) - x
//   residual1      scf_residual1 (src/scf.f90:194-224) with its 8-number-per-site vector
#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "qs_common.cuh"

#include <atomic>

namespace qs {

size_t broyden_red_len();

static std::atomic<int64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(int64_t k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

int prof_begin(qs_handle *h, int fam, bool count) {
    if (count) count_launch();
    if (!h->prof_on) return -1;
    size_t i = h->prof_fam.size();
    if (2 * i + 2 > h->prof_ev.size()) {
        for (int k = 0; k < 64; k++) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return -1;
            h->prof_ev.push_back(e);
        }
    }
    h->prof_fam.push_back(fam);
    cudaEventRecord(h->prof_ev[2 * i], h->stream);
    return (int)i;
}
void prof_end(qs_handle *h, int idx) {
    if (idx < 0) return;
    cudaEventRecord(h->prof_ev[2 * idx + 1], h->stream);
}

int dalloc(qs_handle *h, void **p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    // stream-ordered: releasing a handle's memory does not synchronise the device, so
    // solves of other handles (the serving loop) keep running meanwhile
    cudaError_t e = cudaMallocAsync(p, bytes, h->stream);
    if (e != cudaSuccess) {
        h->err = "cudaMallocAsync of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e);
        *p = nullptr;
        return -2;
    }
    e = cudaMemsetAsync(*p, 0, bytes, h->stream);
    if (e != cudaSuccess) {
        h->err = cudaGetErrorString(e);
        return -(int)e;
    }
    h->allocs.push_back(*p);
    h->bytes_allocated += bytes;
    return 0;
}

void release_all(qs_handle *h) {
    for (void *p : h->allocs) cudaFreeAsync(p, h->stream);
    h->allocs.clear();
    cudaStreamSynchronize(h->stream);
}

// G^<(t=0) on the on-site blocks of the active sites from the SCF vector, then Sigma1
// (equal_time_lesser, src/green_functions.f90:192-213; sigma_first_order,
// src/self_energies.f90:45-72). One block per active site.
__global__ void glt0_sigma1(const double *__restrict__ x, int64_t nblk, int n, int nA, int N, const int *__restrict__ act,
                            const double *__restrict__ U, double pp, zc *__restrict__ Glt0, zc *__restrict__ Sig1) {
    __shared__ double sh[4][32];
    const int I = blockIdx.x, io = 2 * I;
    const int64_t offL = 2 * (int64_t)nA * nA, offD = offL + (int64_t)nA * (nA - 1);
    const int64_t o01 = offL + 2 * ((int64_t)(io + 1) * io / 2 + io);  // (io, io+1), strict upper
    double v[4] = {0, 0, 0, 0};
    for (int w = threadIdx.x; w < n; w += blockDim.x) {
        const double *b = x + (int64_t)w * nblk;
        v[0] += b[offD + io];
        v[1] += b[offD + io + 1];
        v[2] += b[o01];
        v[3] += b[o01 + 1];
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = 0; k < 4; k++) {
        double t = v[k];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (lane == 0) sh[k][wid] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s[4];
        for (int k = 0; k < 4; k++) {
            s[k] = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) s[k] += sh[k][w];
        }
        zc g00{0.0, s[0] * pp}, g11{0.0, s[1] * pp}, g01{s[2] * pp, s[3] * pp};
        zc g10 = -conj(g01);
        Glt0[4 * I + 0] = g00;
        Glt0[4 * I + 1] = g10;
        Glt0[4 * I + 2] = g01;
        Glt0[4 * I + 3] = g11;
        const int i0 = act[io];  // full index of the spin-up state
        const double u = U[i0];
        zc hart = g00 + g11;
        zc G[2][2] = {{g00, g01}, {g10, g11}};
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) {
                zc t = (a == b) ? G[a][b] - hart : G[a][b];
                Sig1[(i0 + a) + (size_t)(i0 + b) * N] = zc{-u * t.y, u * t.x};  // i hbar U t
            }
    }
}

int equal_time_lesser_sigma1(qs_handle *h, const double *d_x) {
    int pi = prof_begin(h, K_REDUCE);
    glt0_sigma1<<<h->nAs, 256, 0, h->stream>>>(d_x, h->nblk, h->n, h->nA, h->Norb, h->d_act, h->d_U,
                                                h->delta / (2.0 * PI), h->d_Glt0, h->d_Sig1);
    prof_end(h, pi);
    QS_CUDA(h, cudaGetLastError());
    return 0;
}

}  // namespace qs

using namespace qs;

// ------------------------------------------------------------------------------------
// host helpers
// ------------------------------------------------------------------------------------
namespace qs {

// check_diag_sanity (common/scf_checks.f90:59-91) from the per-state sums over energies:
// sumL[i] = sum_w G^<_ii(w), sumRim[i] = sum_w Im G^r_ii(w).
SanityOut check_diag_sanity(int nb, const std::vector<zc> &sumL, const std::vector<double> &sumRim, double delta,
                            const int *state_index) {
    SanityOut s;
    for (int i = 0; i < nb; i++) {
        int lab = state_index ? state_index[i] + 1 : i + 1;
        double nocc = 1.0 * (delta / (2.0 * PI)) * sumL[i].y;  // Re(-i hbar pp sum)
        double wsum = -1.0 * (delta / PI) * sumRim[i];
        if (!std::isfinite(nocc) || !std::isfinite(wsum)) {  // runaway only, as the reference returns here
            s.runaway = true;
            s.i_worst = lab;
            s.n_worst = nocc;
            s.w_worst = wsum;
            return s;
        }
        if (nocc < -1.0 || nocc > 2.0) s.runaway = true;
        if (nocc < -0.05 || nocc > 1.05 || wsum < 0.5) s.unphysical = true;
        if (std::fabs(nocc - 0.5) > std::fabs(s.n_worst - 0.5) || (wsum < s.w_worst && std::fabs(s.n_worst - 0.5) <= 0.55)) {
            s.i_worst = lab;
            s.n_worst = nocc;
            s.w_worst = wsum;
        }
    }
    if (s.runaway) s.unphysical = true;
    return s;
}

}  // namespace qs

namespace {

int read_info(qs_handle *h, int &info) {
    int hv[2];
    QS_CUDA(h, cudaMemcpyAsync(hv, h->d_info, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    QS_CUDA(h, cudaStreamSynchronize(h->stream));
    info = hv[0];
    if (hv[1] != 0) {  // a bounded tensor-core wait gave up (the kernel freed its TMEM and returned)
        h->err = "tensor-core Keldysh kernel: an mbarrier wait timed out";
        int z = 0;
        QS_CUDA(h, cudaMemcpyAsync(h->d_info + 1, &z, sizeof(int), cudaMemcpyHostToDevice, h->stream));
        QS_CUDA(h, cudaStreamSynchronize(h->stream));
        return -3;
    }
    if (info != INT_MAX) {
        h->err = "ERROR: ZGETRF failed (singular matrix?) at energy index " + std::to_string(info);
        int v = INT_MAX;
        QS_CUDA(h, cudaMemcpyAsync(h->d_info, &v, sizeof(int), cudaMemcpyHostToDevice, h->stream));
        return info;
    }
    return 0;
}

// the sanity of the active states from the sums over energies of the diagonals gRd, gLd
// already formed in the reduction scratch ([nA] gLd sums, then [nA] gRd sums)
int sweep_sanity_read(qs_handle *h, SanityOut &s) {
    zc *sums = (zc *)h->d_red;
    std::vector<zc> hs(2 * h->nA);
    QS_CUDA(h, cudaMemcpyAsync(hs.data(), sums, sizeof(zc) * 2 * h->nA, cudaMemcpyDeviceToHost, h->stream));
    int info, rc;
    if ((rc = read_info(h, info))) return rc;
    std::vector<zc> sl(hs.begin(), hs.begin() + h->nA);
    std::vector<double> sr(h->nA);
    for (int i = 0; i < h->nA; i++) sr[i] = hs[h->nA + i].y;
    s = check_diag_sanity(h->nA, sl, sr, h->delta, h->act.data());
    return 0;
}

// sums over energies of the diagonals gRd, gLd -> sanity of the active states
int sweep_sanity(qs_handle *h, SanityOut &s) {
    zc *sums = (zc *)h->d_red;  // [nA] gLd sums, then [nA] gRd sums
    int rc;
    if ((rc = sum_over_energies(h, h->d_gLd, h->nA, h->nA, h->n, sums))) return rc;
    if ((rc = sum_over_energies(h, h->d_gRd, h->nA, h->nA, h->n, sums + h->nA))) return rc;
    return sweep_sanity_read(h, s);
}

// order-1 vector: Re, Im of the 2x2 on-site block of G^<(t=0) of each interacting site
// (pack_nil / unpack_nil, src/scf.f90:226-255); G is Norb x Norb complex as double pairs.
void pack_nil(const qs_handle *h, const std::vector<double> &G, double *x) {
    int k = 0;
    const int N = h->Norb;
    for (int s = 0; s < h->N_sites; s++) {
        if (!h->site_int[s]) continue;
        for (int b = 2 * s; b <= 2 * s + 1; b++)
            for (int a = 2 * s; a <= 2 * s + 1; a++) {
                x[k] = G[2 * (a + (size_t)b * N)];
                x[k + 1] = G[2 * (a + (size_t)b * N) + 1];
                k += 2;
            }
    }
}
void unpack_nil(const qs_handle *h, const double *x, std::vector<double> &G) {
    std::fill(G.begin(), G.end(), 0.0);
    int k = 0;
    const int N = h->Norb;
    for (int s = 0; s < h->N_sites; s++) {
        if (!h->site_int[s]) continue;
        for (int b = 2 * s; b <= 2 * s + 1; b++)
            for (int a = 2 * s; a <= 2 * s + 1; a++) {
                G[2 * (a + (size_t)b * N)] = x[k];
                G[2 * (a + (size_t)b * N) + 1] = x[k + 1];
                k += 2;
            }
    }
}

// sigma_first_order on the host (order 1: G^<(t=0) lives on the host)
void sigma1_host(const qs_handle *h, const std::vector<double> &G, std::vector<double> &S) {
    const int N = h->Norb;
    std::fill(S.begin(), S.end(), 0.0);
    auto g = [&](int i, int j) { return zc{G[2 * (i + (size_t)j * N)], G[2 * (i + (size_t)j * N) + 1]}; };
    for (int i = 0; i < N; i += 2) {
        zc hart = g(i, i) + g(i + 1, i + 1);
        double u = h->U_site[i];
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) {
                zc t = (a == b) ? g(i + a, i + b) - hart : g(i + a, i + b);
                S[2 * ((i + a) + (size_t)(i + b) * N)] = -u * t.y;
                S[2 * ((i + a) + (size_t)(i + b) * N) + 1] = u * t.x;
            }
    }
}

// gather_onsite over a site mask from the device sums of onsL (4 per site)
void gather_onsite(const qs_handle *h, const std::vector<zc> &sums, const std::vector<char> &mask, std::vector<double> &G) {
    const double pp = h->delta / (2.0 * PI);
    const int N = h->Norb;
    for (int s = 0; s < h->N_sites; s++) {
        if (!mask[s]) continue;
        for (int b = 0; b < 2; b++)
            for (int a = 0; a < 2; a++) {
                zc v = sums[4 * s + a + 2 * b];
                G[2 * ((2 * s + a) + (size_t)(2 * s + b) * N)] = v.x * pp;
                G[2 * ((2 * s + a) + (size_t)(2 * s + b) * N) + 1] = v.y * pp;
            }
    }
}

int onsite_sums(qs_handle *h, std::vector<zc> &sums) {
    zc *d = (zc *)h->d_red;
    int rc;
    if ((rc = sum_over_energies(h, h->d_onsL, 4 * h->N_sites, 4 * h->N_sites, h->n, d))) return rc;
    sums.resize(4 * h->N_sites);
    QS_CUDA(h, cudaMemcpyAsync(sums.data(), d, sizeof(zc) * sums.size(), cudaMemcpyDeviceToHost, h->stream));
    QS_CUDA(h, cudaStreamSynchronize(h->stream));
    return 0;
}

// The order-2 residual F = pack(G_out[x]) - x. QS_PREC_MIXED: while max|F| is far above the
// FP32 noise floor, the steps form the second-order self-energies in FP32 (FFTs, 2x2
// algebra and spectra), and the Keldysh products run on the fastest of the 3xTF32
// tensor-core kernel (keldysh_tf32.cu) and the FP64 ones (autotuned). The FP32 transforms
// carry rounding relative to the largest spectra (|Sigma^r|, which on a fine grid is 10^3-10^4
// times |Sigma^<|), and the Dyson inverse amplifies it by its conditioning, so the floor of F
// depends on the model. The solve continues in FP64 once max|F| falls below mixed_switch =
// max(1e-5, 100 tolf), or once it has not improved for two steps (the FP32 floor reached,
// whatever its level: steps spent on it are wasted). An FP32 step whose max|F| is already
// below tolf is redone in FP64 first, so that it cannot end the solve: convergence
// (max|F| < tolf) is always decided on an FP64 residual, and the converged state meets the
// FP64 solve's criterion. At the first FP64 step the Broyden history restarts from the
// FP32 phase's iterate (precision_changed): its pairs model the FP32 residual function.
// The device work of one order-2 residual: G^<(t=0) and Sigma1, Sigma2, the sweep writing
// F = pack(G_out) - x, the sanity sums (no host synchronisation in between).
int residual2_launches(qs_handle *h, double V, const double *d_x, double *d_F, bool use32) {
    int rc;
    if ((rc = equal_time_lesser_sigma1(h, d_x))) return rc;
    if ((rc = sigma2_compute(h, d_x, use32))) return rc;
    if ((rc = sweep(h, M_SCF2, V, true, d_F, d_x, use32))) return rc;
    zc *sums = (zc *)h->d_red;
    if ((rc = sum_over_energies(h, h->d_gLd, h->nA, h->nA, h->n, sums))) return rc;
    if ((rc = sum_over_energies(h, h->d_gRd, h->nA, h->nA, h->n, sums + h->nA))) return rc;
    return 0;
}

// The FP64 residual's launches replayed from a CUDA graph: captured at the second evaluation
// of an (x, F, V) (the first one has made every autotuner decision of the sizes), replayed
// afterwards. Not with per-launch profiling on (its events are per launch) nor in the FP32
// phase; a capture that fails turns graphs off for the handle (eager launches, same results).
int residual2_graphed(qs_handle *h, double V, const double *d_x, double *d_F) {
    for (auto &g : h->graphs)
        if (g.exec && g.x == d_x && g.F == d_F && g.V == V) {
            QS_CUDA(h, cudaGraphLaunch(g.exec, h->stream));
            count_launches(g.launches);
            h->graph_replays++;
            return 0;
        }
    auto &g = h->graphs[h->graph_next];
    h->graph_next ^= 1;
    if (g.exec) {
        cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
    }
    const int64_t l0 = qs_kernel_launches();
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        h->graphs_off = true;
        return residual2_launches(h, V, d_x, d_F, false);
    }
    int rc = residual2_launches(h, V, d_x, d_F, false);
    cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    const int64_t captured = qs_kernel_launches() - l0;
    if (rc == 0 && e == cudaSuccess && graph) e = cudaGraphInstantiate(&g.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (rc != 0 || e != cudaSuccess || !g.exec) {
        cudaGetLastError();  // the failed capture leaves nothing behind on the stream
        g.exec = nullptr;
        h->graphs_off = true;
        h->err.clear();
        return residual2_launches(h, V, d_x, d_F, false);
    }
    g.x = d_x;
    g.F = d_F;
    g.V = V;
    g.launches = captured;
    QS_CUDA(h, cudaGraphLaunch(g.exec, h->stream));
    h->graph_replays++;
    return 0;
}

struct Residual2 : BroydenResidual {
    qs_handle *h;
    double V;
    int iter = 0;
    bool fp32 = false;  // this solve is still in its FP32 phase
    int n_mixed = 0;
    double best = HUGE_VAL;
    int since_best = 0;
    int last_prec = -1, cur_prec = -1;  // 1 = FP32 phase, 0 = FP64, of the last two evaluations
    int evals64 = 0;                    // FP64 evaluations of this solve (the first runs eagerly)
    bool precision_changed() const override { return last_prec >= 0 && last_prec != cur_prec; }
    int eval(const double *d_x, double *d_F, bool &abort, bool use32) {
        int rc;
        const bool graph = !use32 && !h->prof_on && !h->graphs_off && evals64 > 0;
        if (!use32) evals64++;
        if (graph) {
            if ((rc = residual2_graphed(h, V, d_x, d_F))) return rc;
        } else if ((rc = residual2_launches(h, V, d_x, d_F, use32))) {
            return rc;
        }
        SanityOut s;
        if ((rc = sweep_sanity_read(h, s))) return rc;
        abort = s.runaway;
        if (abort) QS_CUDA(h, cudaMemsetAsync(d_F, 0, sizeof(double) * h->n_vec, h->stream));
        return 0;
    }
    int operator()(const double *d_x, double *d_F, bool &abort) override {
        iter++;
        last_prec = cur_prec;
        cur_prec = fp32 ? 1 : 0;
        int rc;
        if (!fp32) return eval(d_x, d_F, abort, false);
        if ((rc = eval(d_x, d_F, abort, true))) return rc;
        if (abort) return 0;
        double fmax;
        if ((rc = vec_maxabs(h, d_F, h->n_vec, fmax))) return rc;
        if (fmax < best) {
            best = fmax;
            since_best = 0;
        } else {
            since_best++;
        }
        n_mixed++;
        if (fmax < h->mixed_switch || since_best >= 2) {
            fp32 = false;  // the next steps are FP64
            if (fmax < h->tolf) {  // never let an FP32 residual declare convergence: redo it
                n_mixed--;
                cur_prec = 0;
                return eval(d_x, d_F, abort, false);
            }
        }
        return 0;
    }
};

struct Residual1 : BroydenResidual {
    qs_handle *h;
    double V;
    int iter = 0;
    int operator()(const double *d_x, double *d_F, bool &abort) override {
        iter++;
        const int64_t nv = h->n_vec;
        std::vector<double> x(nv), F(nv);
        QS_CUDA(h, cudaMemcpyAsync(x.data(), d_x, sizeof(double) * nv, cudaMemcpyDeviceToHost, h->stream));
        QS_CUDA(h, cudaStreamSynchronize(h->stream));
        unpack_nil(h, x.data(), h->G_less_t0);
        sigma1_host(h, h->G_less_t0, h->Sig1);
        QS_CUDA(h, cudaMemcpyAsync(h->d_Sig1, h->Sig1.data(), sizeof(double) * h->Sig1.size(), cudaMemcpyHostToDevice, h->stream));
        int rc;
        if ((rc = sweep(h, M_SCF1, V, true, nullptr, nullptr))) return rc;
        SanityOut s;
        if ((rc = sweep_sanity(h, s))) return rc;
        abort = s.runaway;
        if (!abort) {
            std::vector<zc> sums;
            if ((rc = onsite_sums(h, sums))) return rc;
            std::vector<double> Gout((size_t)2 * h->Norb * h->Norb, 0.0);
            std::vector<char> mask(h->site_int.begin(), h->site_int.end());
            gather_onsite(h, sums, mask, Gout);
            pack_nil(h, Gout, F.data());
            for (int64_t i = 0; i < nv; i++) F[i] -= x[i];
        }
        QS_CUDA(h, cudaMemcpyAsync(d_F, F.data(), sizeof(double) * nv, cudaMemcpyHostToDevice, h->stream));
        QS_CUDA(h, cudaStreamSynchronize(h->stream));
        return 0;
    }
};

// final sweep + gather_onsite + gather_atoms + Current + final_sanity (src/scf.f90:134-140)
int final_sweep(qs_handle *h, double V, SanityOut &s) {
    int rc;
    if ((rc = sweep(h, M_FINAL, V, h->order >= 1, nullptr, nullptr))) return rc;
    const int N = h->Norb, ns4 = 4 * h->N_sites;
    const int nat = h->has_atomL ? h->atom_off.back() : 0;
    zc *d = (zc *)h->d_red;
    if ((rc = sum_over_energies(h, h->d_onsL, ns4, ns4, h->n, d))) return rc;
    if (nat && (rc = sum_over_energies(h, h->d_atomL, nat, nat, h->n, d + ns4))) return rc;
    double *dr = (double *)(d + ns4 + nat);
    if ((rc = sum_over_energies_real(h, h->d_dosd, N, N, h->n, dr))) return rc;
    if ((rc = sum_over_energies_real(h, h->d_trU, 1, 1, h->n, dr + N))) return rc;
    if ((rc = sum_over_energies_real(h, h->d_trD, 1, 1, h->n, dr + N + 1))) return rc;
    std::vector<zc> sums(ns4 + nat);
    std::vector<double> rs(N + 2);
    QS_CUDA(h, cudaMemcpyAsync(sums.data(), d, sizeof(zc) * sums.size(), cudaMemcpyDeviceToHost, h->stream));
    QS_CUDA(h, cudaMemcpyAsync(rs.data(), dr, sizeof(double) * rs.size(), cudaMemcpyDeviceToHost, h->stream));
    int info;
    if ((rc = read_info(h, info))) return rc;
    // G_less_obs: on-site blocks of every site, then the intra-atom blocks
    std::fill(h->G_less_obs.begin(), h->G_less_obs.end(), 0.0);
    std::vector<char> all(h->N_sites, 1);
    gather_onsite(h, sums, all, h->G_less_obs);
    if (nat) {
        const double pp = h->delta / (2.0 * PI);
        for (int at = 0; at < h->N_atoms; at++) {
            int m = 2 * h->atom_norb[at], lo = 2 * (h->atom_first[at] - 1);
            for (int b = 0; b < m; b++)
                for (int a = 0; a < m; a++) {
                    zc v = sums[ns4 + h->atom_off[at] + a + b * m];
                    h->G_less_obs[2 * ((lo + a) + (size_t)(lo + b) * N)] = v.x * pp;
                    h->G_less_obs[2 * ((lo + a) + (size_t)(lo + b) * N) + 1] = v.y * pp;
                }
        }
    }
    // Current (src/observables.f90:22-39)
    h->J_up = rs[N] * h->delta;
    h->J_down = rs[N + 1] * h->delta;
    // final_sanity (src/scf.f90:260-275): every state, G^<_ii from the on-site blocks
    std::vector<zc> sl(N);
    std::vector<double> sr(N);
    for (int i = 0; i < N; i++) {
        int st = i / 2, a = i % 2;
        sl[i] = sums[4 * st + a + 2 * a];
        sr[i] = rs[i];
    }
    s = check_diag_sanity(N, sl, sr, h->delta, nullptr);
    h->final_done = true;
    return 0;
}

void setup_storage(qs_handle *h) {
    const int N = h->Norb;
    h->site_int.assign(h->N_sites, 0);
    h->site_act.assign(h->N_sites, 0);
    h->pos.assign(N, -1);
    std::vector<char> conL(N, 0), conR(N, 0);
    for (int s = 0; s < h->N_sites; s++) h->site_int[s] = (h->order >= 1 && h->U_site[2 * s] != 0.0);
    h->n_int_sites = 0;
    for (int s = 0; s < h->N_sites; s++) h->n_int_sites += h->site_int[s];
    h->site_act = h->site_int;
    auto nz = [&](const std::vector<double> &G, int i, int j) {
        size_t k = 2 * (i + (size_t)j * N);
        return G[k] != 0.0 || G[k + 1] != 0.0;
    };
    for (int i = 0; i < N; i++) {
        bool l = false, r = false;
        for (int j = 0; j < N; j++) {
            l = l || nz(h->GammaL, i, j) || nz(h->GammaL, j, i);
            r = r || nz(h->GammaR, i, j) || nz(h->GammaR, j, i);
        }
        conL[i] = l;
        conR[i] = r;
        if (l || r) h->site_act[i / 2] = 1;
    }
    h->act.clear();
    for (int i = 0; i < N; i++)
        if (h->site_act[i / 2]) {
            h->pos[i] = (int)h->act.size();
            h->act.push_back(i);
        }
    h->nA = (int)h->act.size();
    h->asite.clear();
    for (int s = 0; s < h->N_sites; s++)
        if (h->site_act[s]) h->asite.push_back(s);
    h->nAs = (int)h->asite.size();
    h->cl.clear();
    for (int i = 0; i < N; i++)
        if (conL[i]) h->cl.push_back(i);
    h->nCL = (int)h->cl.size();
    h->sup.clear();
    if (h->order == 2) h->sup = h->act;
    else
        for (int i = 0; i < N; i++)
            if (conL[i] || conR[i]) h->sup.push_back(i);
    h->nS = (int)h->sup.size();
    int mx = 0;
    for (int v : h->atom_norb) mx = std::max(mx, v);
    h->has_atomL = mx > 1;
    h->atom_off.assign(h->N_atoms + 1, 0);
    for (int a = 0; a < h->N_atoms; a++) h->atom_off[a + 1] = h->atom_off[a] + (2 * h->atom_norb[a]) * (2 * h->atom_norb[a]);
    if (h->order == 1) h->n_vec = 8 * h->n_int_sites;
    else if (h->order == 2) h->n_vec = (int64_t)3 * h->nA * h->nA * h->n;
    else h->n_vec = 0;
    h->nblk = (int64_t)3 * h->nA * h->nA;
    h->G_less_t0.assign((size_t)2 * N * N, 0.0);
    h->G_less_obs.assign((size_t)2 * N * N, 0.0);
    h->Sig1.assign((size_t)2 * N * N, 0.0);
}

int good_fft_size_h(int nmin) {
    for (int n = nmin;; n++) {
        int m = n;
        for (int r : {2, 3, 5, 7})
            while (m % r == 0) m /= r;
        if (m == 1) return n;
    }
}

template <class T> int upload(qs_handle *h, T **d, const std::vector<T> &v) {
    int rc = dalloc(h, (void **)d, sizeof(T) * std::max<size_t>(v.size(), 1));
    if (rc) return rc;
    if (!v.empty()) QS_CUDA(h, cudaMemcpyAsync(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, h->stream));
    return 0;
}

}  // namespace

// ------------------------------------------------------------------------------------
// C ABI
// the host fields of a handle from the problem (no device work)
static int fill_host(qs_handle *h, const qs_problem *p) {
    h->Norb = p->Norb;
    h->N_sites = p->N_sites;
    h->N_atoms = p->N_atoms;
    h->order = p->order;
    h->n = p->n_omega;
    h->device = p->device;
    h->precision = p->precision;
    h->mu = p->mu;
    h->beta = p->beta;
    h->delta = p->delta;
    h->alpha_mix = p->alpha_mix;
    h->tolf = p->tolf;
    h->tolf_order1 = p->tolf_order1;
    h->mixed_switch = std::max(1e-5, 100.0 * p->tolf);
    h->nhist = p->nhist;
    h->maxscf = p->maxscf;
    h->single = p->single_history != 0;
    const int N = h->Norb;
    if (N > 512 || N < 2 || h->n < 1) {
        h->err = "qs_create: need 2 <= Norb <= 512 and n_omega >= 1";
        return -1;
    }
    const size_t nn = (size_t)N * N;
    h->H.assign(p->H, p->H + 2 * nn);
    h->GammaL.assign(p->GammaL, p->GammaL + 2 * nn);
    h->GammaR.assign(p->GammaR, p->GammaR + 2 * nn);
    h->U_site.assign(p->U_site, p->U_site + N);
    h->omega.assign(p->omega, p->omega + h->n);
    h->atom_norb.assign(p->atom_norb, p->atom_norb + p->N_atoms);
    h->atom_first.assign(p->atom_first, p->atom_first + p->N_atoms);
    if (h->precision != QS_PREC_FP64 && h->precision != QS_PREC_MIXED) {
        h->err = "qs_create: precision must be QS_PREC_FP64 or QS_PREC_MIXED";
        return -1;
    }
    if (h->nhist > 32 || h->nhist < 0) {
        h->err = "qs_create: nhist must be in 0..32";
        return -1;
    }
    return 0;
}

// device bytes a solve keeps (the allocations of qs_create), after setup_storage
static size_t handle_need(const qs_handle *h) {
    const int N = h->Norb, nA = h->nA, n = h->n;
    const size_t nn = (size_t)N * N, zc_ = sizeof(zc);
    const size_t hist_el = h->single ? 4 : 8;
    const int Nf = (h->order == 2) ? good_fft_size_h(2 * n - 1) : 0;
    size_t need = 0;
    need += nn * zc_ * 2 + (size_t)n * 8 * 1;                                // Hemb, Sig1, omega
    need += (size_t)n * (4 * h->N_sites * zc_ + N * 8 + 16);                // onsL, dosd, trU, trD
    if (h->has_atomL) need += (size_t)n * h->atom_off.back() * zc_;
    need += (size_t)n * std::max(nA, 1) * zc_ * 2;                           // gRd, gLd
    if (!dyson_fits_smem(N) || (N > 16 && N <= 256)) need += (size_t)148 * 2 * nn * zc_;  // Gauss-Jordan workspace
    if (h->order == 2) {
        size_t nY = (size_t)nA * nA + (size_t)nA * (nA + 1) / 2;
        need += (size_t)h->n_vec * 8 * 4;                                     // x, F, Fold, xold
        need += (size_t)broyden_ld(h->n_vec) * hist_el * 2 * h->nhist;                    // history
        need += (size_t)n * nA * nA * zc_ * 2;                                // SigR, SigL
        need += (nY + (size_t)2 * nA * nA) * Nf * zc_;                        // Y, V
    } else {
        const size_t G_chunk = std::max<size_t>(1, std::min<size_t>((size_t)n, (2ull << 30) / (nn * zc_)));
        need += G_chunk * nn * zc_;                                           // full-G chunk
        need += (size_t)148 * 4 * N * std::max(h->nS, 1) * zc_;               // sweep scratch
        const int64_t nv = std::max<int64_t>(h->n_vec, 1);
        if (h->order == 1) need += (size_t)nv * 8 * 4 + (size_t)broyden_ld(nv) * hist_el * 2 * h->nhist;
    }
    need += broyden_red_len() * 8 + (size_t)3 * h->nS * h->nS * zc_;        // reductions, Gamma blocks
    if (h->order == 2) {
        size_t nY = (size_t)nA * nA + (size_t)nA * (nA + 1) / 2;
        need += (size_t)Nf * zc_ + nY * 8 + (size_t)h->nAs * h->nAs * 16;      // twiddles, FFT tables
    }
    need += (size_t)1 << 20;  // index tables and the allocations' 256-byte granularity
    return need;
}

// ------------------------------------------------------------------------------------
extern "C" {

int qs_create(const qs_problem *p, qs_handle **out) {
    *out = nullptr;
    auto *h = new qs_handle();
    *out = h;
    int rc0 = fill_host(h, p);
    if (rc0) return rc0;
    QS_CUDA(h, cudaSetDevice(h->device));
    QS_CUDA(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    QS_CUDA(h, cudaEventCreate(&h->ev0));
    QS_CUDA(h, cudaEventCreate(&h->ev1));
    setup_storage(h);
    if (h->nCL > 32) {
        h->err = "qs_create: more than 32 left-contact states";
        return -1;
    }
    const int N = h->Norb;
    const size_t nn = (size_t)N * N;
    const int nA = h->nA, nS = h->nS, n = h->n;
    const int Nf = (h->order == 2) ? good_fft_size_h(2 * n - 1) : 0;
    const size_t zc_ = sizeof(zc);
    size_t hist_el = h->single ? 4 : 8;
    // ---- HBM admission: everything this solve keeps on the device
    size_t need = handle_need(h);
    size_t freeb = 0, totb = 0;
    QS_CUDA(h, cudaMemGetInfo(&freeb, &totb));
    if (need + (512ull << 20) > freeb) {
        h->err = "qs_create: HBM admission failed: the solve needs " + std::to_string(need >> 20) + " MiB, " +
                 std::to_string(freeb >> 20) + " MiB free";
        return -2;
    }

    // ---- model arrays: Hemb = -H + (i/2hbar)(GammaL + GammaR)  (src/scf.f90:92)
    std::vector<zc> Hemb(nn), GLs((size_t)nS * nS), GRs((size_t)nS * nS), GLcl((size_t)h->nCL * h->nCL);
    for (size_t k = 0; k < nn; k++) {
        double gr = h->GammaL[2 * k] + h->GammaR[2 * k], gi = h->GammaL[2 * k + 1] + h->GammaR[2 * k + 1];
        Hemb[k] = zc{-h->H[2 * k] - 0.5 * gi, -h->H[2 * k + 1] + 0.5 * gr};
    }
    for (int b = 0; b < nS; b++)
        for (int a = 0; a < nS; a++) {
            size_t k = h->sup[a] + (size_t)h->sup[b] * N;
            GLs[a + (size_t)b * nS] = zc{h->GammaL[2 * k], h->GammaL[2 * k + 1]};
            GRs[a + (size_t)b * nS] = zc{h->GammaR[2 * k], h->GammaR[2 * k + 1]};
        }
    for (int b = 0; b < h->nCL; b++)
        for (int a = 0; a < h->nCL; a++) {
            size_t k = h->cl[a] + (size_t)h->cl[b] * N;
            GLcl[a + (size_t)b * h->nCL] = zc{h->GammaL[2 * k], h->GammaL[2 * k + 1]};
        }
    std::vector<int> site_int(h->site_int.begin(), h->site_int.end());
    // the contact states: the rows and columns where the lead matrices are non-zero (the
    // Keldysh kernel adds their term to T = G Sigma2^< as a low-rank correction)
    std::vector<int> cidx;
    for (int k = 0; k < nS; k++) {
        bool nz = false;
        for (int j = 0; j < nS && !nz; j++) {
            const size_t kj = k + (size_t)j * nS, jk = j + (size_t)k * nS;
            nz = GLs[kj].x != 0.0 || GLs[kj].y != 0.0 || GRs[kj].x != 0.0 || GRs[kj].y != 0.0 || GLs[jk].x != 0.0 ||
                 GLs[jk].y != 0.0 || GRs[jk].x != 0.0 || GRs[jk].y != 0.0;
        }
        if (nz) cidx.push_back(k);
    }
    h->kd_nc = (int)cidx.size();
    if (cidx.empty()) cidx.push_back(0);
    int rc;
    if ((rc = upload(h, &h->d_kd_cidx, cidx))) return rc;
    if ((rc = upload(h, &h->d_Hemb, Hemb)) || (rc = dalloc(h, (void **)&h->d_Sig1, nn * zc_)) ||
        (rc = upload(h, &h->d_GamLs, GLs)) || (rc = upload(h, &h->d_GamRs, GRs)) || (rc = upload(h, &h->d_GamLcl, GLcl)) ||
        (rc = upload(h, &h->d_pos, h->pos)) || (rc = upload(h, &h->d_act, h->act)) || (rc = upload(h, &h->d_sup, h->sup)) ||
        (rc = upload(h, &h->d_cl, h->cl)) || (rc = upload(h, &h->d_atom_first, h->atom_first)) ||
        (rc = upload(h, &h->d_atom_norb, h->atom_norb)) || (rc = upload(h, &h->d_atom_off, h->atom_off)) ||
        (rc = upload(h, &h->d_site_int, site_int)) || (rc = upload(h, &h->d_omega, h->omega)) ||
        (rc = upload(h, &h->d_U, h->U_site)))
        return rc;
    // per-energy outputs
    if ((rc = dalloc(h, (void **)&h->d_onsL, (size_t)n * 4 * h->N_sites * zc_)) ||
        (rc = dalloc(h, (void **)&h->d_dosd, (size_t)n * N * 8)) || (rc = dalloc(h, (void **)&h->d_trU, (size_t)n * 8)) ||
        (rc = dalloc(h, (void **)&h->d_trD, (size_t)n * 8)) ||
        (rc = dalloc(h, (void **)&h->d_gRd, (size_t)n * std::max(nA, 1) * zc_)) ||
        (rc = dalloc(h, (void **)&h->d_gLd, (size_t)n * std::max(nA, 1) * zc_)) ||
        (rc = dalloc(h, (void **)&h->d_Glt0, (size_t)4 * std::max(h->nAs, 1) * zc_)))
        return rc;
    if (h->has_atomL && (rc = dalloc(h, (void **)&h->d_atomL, (size_t)n * h->atom_off.back() * zc_))) return rc;
    h->red_len = std::max<size_t>(broyden_red_len(), (size_t)2 * (4 * h->N_sites + h->atom_off.back() + 2 * N + 2 * nA + 8));
    if ((rc = dalloc(h, (void **)&h->d_red, h->red_len * 8))) return rc;
    if ((rc = dalloc(h, (void **)&h->d_info, sizeof(int) * 2))) return rc;
    int imax = INT_MAX;
    QS_CUDA(h, cudaMemcpyAsync(h->d_info, &imax, sizeof(int), cudaMemcpyHostToDevice, h->stream));
    // Gauss-Jordan workspace: for matrices that do not fit in shared memory, and for the
    // two-blocks-per-SM blocked variant (16 < N <= 256)
    if (!dyson_fits_smem(N) || (N > 16 && N <= 256)) {
        h->ws_slots = 148 * 2;
        if ((rc = dalloc(h, (void **)&h->d_Gws, h->ws_slots * nn * zc_))) return rc;
    }
    // order 2: SCF vectors, history, Sigma2 and the FFT; the sweep scratch aliases the
    // FFT intermediates (dead once Sigma2 is formed)
    const size_t Trows = (size_t)N * std::max(nS, 1);
    if (h->order == 2) {
        if ((rc = dalloc(h, (void **)&h->d_x, h->n_vec * 8)) || (rc = dalloc(h, (void **)&h->d_F, h->n_vec * 8)) ||
            (rc = dalloc(h, (void **)&h->d_Fold, h->n_vec * 8)) || (rc = dalloc(h, (void **)&h->d_xold, h->n_vec * 8)))
            return rc;
        if (h->nhist > 0 && ((rc = dalloc(h, &h->d_hdF, broyden_ld(h->n_vec) * hist_el * h->nhist)) ||
                             (rc = dalloc(h, &h->d_hU, broyden_ld(h->n_vec) * hist_el * h->nhist))))
            return rc;
        if ((rc = sigma2_setup(h))) return rc;
        h->d_G = h->d_Y;
        h->G_chunk = std::min<size_t>((size_t)n, (h->nY * (size_t)h->fft.Nf) / nn);
        h->d_T = h->d_V;
        h->T_bytes = h->nV * (size_t)h->fft.Nf * zc_;
        h->T_slots = std::min<size_t>(148 * 4, h->T_bytes / (std::max(Trows, (size_t)nA * nA) * zc_));
    } else {
        if (h->order == 1) {
            int64_t nv = std::max<int64_t>(h->n_vec, 1);
            if ((rc = dalloc(h, (void **)&h->d_x, nv * 8)) || (rc = dalloc(h, (void **)&h->d_F, nv * 8)) ||
                (rc = dalloc(h, (void **)&h->d_Fold, nv * 8)) || (rc = dalloc(h, (void **)&h->d_xold, nv * 8)))
                return rc;
            if (h->nhist > 0 && ((rc = dalloc(h, &h->d_hdF, broyden_ld(nv) * hist_el * h->nhist)) ||
                                 (rc = dalloc(h, &h->d_hU, broyden_ld(nv) * hist_el * h->nhist))))
                return rc;
        }
        h->G_chunk = std::max<size_t>(1, std::min<size_t>((size_t)n, (2ull << 30) / (nn * zc_)));
        if ((rc = dalloc(h, (void **)&h->d_G, h->G_chunk * nn * zc_))) return rc;
        h->T_slots = 148 * 4;
        h->T_bytes = h->T_slots * Trows * zc_;
        if ((rc = dalloc(h, (void **)&h->d_T, h->T_bytes))) return rc;
    }
    QS_CUDA(h, cudaStreamSynchronize(h->stream));
    return 0;
}

void qs_destroy(qs_handle *h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (auto &g : h->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    for (cudaEvent_t e : h->prof_ev) cudaEventDestroy(e);
    release_all(h);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

const char *qs_last_error(const qs_handle *h) { return h ? h->err.c_str() : "no handle"; }

int qs_estimate_bytes(const qs_problem *p, double *gib) {
    qs_handle h;
    int rc = fill_host(&h, p);
    if (rc) return rc;
    setup_storage(&h);
    *gib = (double)handle_need(&h) / (double)(1ull << 30);
    return 0;
}

double qs_device_bytes(const qs_handle *h) { return h ? (double)h->bytes_allocated / (double)(1ull << 30) : 0.0; }

int64_t qs_kernel_launches(void) { return g_launches.load(); }
int64_t qs_graph_replays(const qs_handle *h) { return h ? h->graph_replays : -1; }

int qs_profile(qs_handle *h, int enable, double *ms, int64_t *launches, int nfam) {
    QS_CUDA(h, cudaStreamSynchronize(h->stream));
    for (size_t i = 0; i < h->prof_fam.size(); i++) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, h->prof_ev[2 * i], h->prof_ev[2 * i + 1]) == cudaSuccess) {
            h->prof_ms[h->prof_fam[i]] += t;
            h->prof_count[h->prof_fam[i]] += 1;
        }
    }
    h->prof_fam.clear();
    for (int f = 0; f < K_NFAM && f < nfam; f++) {
        if (ms) ms[f] = h->prof_ms[f];
        if (launches) launches[f] = h->prof_count[f];
    }
    if (enable < 0 || enable != (int)h->prof_on) {  // reset the totals when switching
        for (int f = 0; f < K_NFAM; f++) {
            h->prof_ms[f] = 0;
            h->prof_count[f] = 0;
        }
    }
    if (enable >= 0) h->prof_on = enable != 0;
    return K_NFAM;
}
int64_t qs_vector_length(const qs_handle *h) { return h->n_vec; }
int qs_active_states(const qs_handle *h) { return h->nA; }
int qs_fft_length(const qs_handle *h) { return h->order == 2 ? h->fft.Nf : good_fft_size_h(2 * h->n - 1); }

int qs_solve_scf(qs_handle *h, double Volt, int fresh_start, qs_scf_result *res) {
    QS_CUDA(h, cudaSetDevice(h->device));
    QS_CUDA(h, cudaEventRecord(h->ev0, h->stream));
    BroydenOut bo;
    int rc = 0, n_mixed = 0;
    bool fresh = fresh_start || !h->have_x;
    if (h->order == 2) {
        if (fresh && (rc = sweep(h, M_INIT2, Volt, false, h->d_x, nullptr))) return rc;
        Residual2 r;
        r.h = h;
        r.V = Volt;
        // the FP32 phase runs on fresh starts only: a continued start is already within one or
        // two orders of magnitude of the FP32 floor, so its FP32 steps end on a stall after
        // three and save none of the FP64 tail (measured: 0.94x of the FP64 form over a
        // continued sweep with them, against a 16 % shorter median solve on fresh starts)
        r.fp32 = (h->precision == QS_PREC_MIXED) && fresh;
        rc = broyden_solve_dev(h, r, h->d_x, h->d_F, h->d_Fold, h->d_xold, h->d_hdF, h->d_hU, h->n_vec, h->alpha_mix,
                               h->nhist, h->maxscf, h->tolf, h->single, bo);
        if (rc) return rc;
        h->have_x = true;
        n_mixed = r.n_mixed;
    } else if (h->order == 1) {
        if (fresh) {
            // G^<(t=0) of the non-interacting system (src/scf.f90:103-108)
            std::fill(h->Sig1.begin(), h->Sig1.end(), 0.0);
            QS_CUDA(h, cudaMemsetAsync(h->d_Sig1, 0, sizeof(zc) * (size_t)h->Norb * h->Norb, h->stream));
            if ((rc = sweep(h, M_SCF1, Volt, false, nullptr, nullptr))) return rc;
            std::vector<zc> sums;
            if ((rc = onsite_sums(h, sums))) return rc;
            std::fill(h->G_less_t0.begin(), h->G_less_t0.end(), 0.0);
            std::vector<char> mask(h->site_int.begin(), h->site_int.end());
            gather_onsite(h, sums, mask, h->G_less_t0);
        }
        std::vector<double> x(std::max<int64_t>(h->n_vec, 1));
        pack_nil(h, h->G_less_t0, x.data());
        QS_CUDA(h, cudaMemcpyAsync(h->d_x, x.data(), sizeof(double) * h->n_vec, cudaMemcpyHostToDevice, h->stream));
        Residual1 r;
        r.h = h;
        r.V = Volt;
        rc = broyden_solve_dev(h, r, h->d_x, h->d_F, h->d_Fold, h->d_xold, h->d_hdF, h->d_hU, h->n_vec, h->alpha_mix,
                               h->nhist, h->maxscf, h->tolf_order1, h->single, bo);
        if (rc) return rc;
        h->have_x = true;
    } else {
        bo.log.push_back({1, 0.0, 0.0, 0});
        bo.n_iter = 1;
        bo.converged = true;
        bo.fmax = 0.0;
    }
    SanityOut s;
    if ((rc = final_sweep(h, Volt, s))) return rc;
    QS_CUDA(h, cudaEventRecord(h->ev1, h->stream));
    QS_CUDA(h, cudaEventSynchronize(h->ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    bool converged = bo.converged && !bo.aborted;
    if (converged && s.unphysical) converged = false;
    res->converged = converged;
    res->n_iter = bo.n_iter;
    res->fmax = bo.fmax;
    res->aborted = bo.aborted;
    res->runaway = s.runaway;
    res->unphysical = s.unphysical;
    res->i_worst = s.i_worst;
    res->n_worst = s.n_worst;
    res->w_worst = s.w_worst;
    res->n_resets = bo.n_resets;
    res->n_log = 0;
    for (auto &e : bo.log)
        if (res->log && res->n_log < res->log_cap) res->log[res->n_log++] = e;
    res->seconds = ms * 1e-3;
    res->n_mixed = n_mixed;
    return 0;
}

int qs_current(qs_handle *h, double, double *J_up, double *J_down) {
    if (!h->final_done) {
        h->err = "qs_current: no final sweep yet";
        return -1;
    }
    *J_up = h->J_up;
    *J_down = h->J_down;
    return 0;
}

int qs_get_observables(qs_handle *h, double *G_less_obs, double *dosd, double *trU, double *trD) {
    QS_CUDA(h, cudaSetDevice(h->device));
    if (G_less_obs) std::memcpy(G_less_obs, h->G_less_obs.data(), sizeof(double) * h->G_less_obs.size());
    if (dosd) QS_CUDA(h, cudaMemcpyAsync(dosd, h->d_dosd, sizeof(double) * (size_t)h->n * h->Norb, cudaMemcpyDeviceToHost, h->stream));
    if (trU) QS_CUDA(h, cudaMemcpyAsync(trU, h->d_trU, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->stream));
    if (trD) QS_CUDA(h, cudaMemcpyAsync(trD, h->d_trD, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->stream));
    QS_CUDA(h, cudaStreamSynchronize(h->stream));
    return 0;
}

int qs_initial_vector(qs_handle *h, double Volt, double *x) {
    QS_CUDA(h, cudaSetDevice(h->device));
    int rc;
    if (h->order == 2) {
        if ((rc = sweep(h, M_INIT2, Volt, false, h->d_x, nullptr))) return rc;
        if ((rc = convert_dl_to_ref(h->stream, h->nA, h->n, h->d_x, h->d_F))) return -rc;
        QS_CUDA(h, cudaMemcpyAsync(x, h->d_F, sizeof(double) * h->n_vec, cudaMemcpyDeviceToHost, h->stream));
        int info;
        return read_info(h, info);
    }
    if (h->order == 1) {
        QS_CUDA(h, cudaMemsetAsync(h->d_Sig1, 0, sizeof(zc) * (size_t)h->Norb * h->Norb, h->stream));
        if ((rc = sweep(h, M_SCF1, Volt, false, nullptr, nullptr))) return rc;
        std::vector<zc> sums;
        if ((rc = onsite_sums(h, sums))) return rc;
        std::vector<double> G((size_t)2 * h->Norb * h->Norb, 0.0);
        std::vector<char> mask(h->site_int.begin(), h->site_int.end());
        gather_onsite(h, sums, mask, G);
        pack_nil(h, G, x);
        int info;
        return read_info(h, info);
    }
    return 0;
}

int qs_residual(qs_handle *h, double Volt, const double *x, double *F, int *abort_flag) {
    QS_CUDA(h, cudaSetDevice(h->device));
    int rc;
    bool ab = false;
    if (h->order == 2) {
        // the reference-layout x goes through d_F as staging, then into d_x (device layout)
        QS_CUDA(h, cudaMemcpyAsync(h->d_F, x, sizeof(double) * h->n_vec, cudaMemcpyHostToDevice, h->stream));
        if ((rc = convert_ref_to_dl(h->stream, h->nA, h->n, h->d_F, h->d_x))) return -rc;
        Residual2 r;
        r.h = h;
        r.V = Volt;
        // a QS_PREC_MIXED handle evaluates the residual of its solves' FP32 phase
        if ((rc = r.eval(h->d_x, h->d_Fold, ab, h->precision == QS_PREC_MIXED))) return rc;
        if ((rc = convert_dl_to_ref(h->stream, h->nA, h->n, h->d_Fold, h->d_F))) return -rc;
        QS_CUDA(h, cudaMemcpyAsync(F, h->d_F, sizeof(double) * h->n_vec, cudaMemcpyDeviceToHost, h->stream));
        QS_CUDA(h, cudaStreamSynchronize(h->stream));
        h->have_x = false;
    } else if (h->order == 1) {
        QS_CUDA(h, cudaMemcpyAsync(h->d_x, x, sizeof(double) * h->n_vec, cudaMemcpyHostToDevice, h->stream));
        Residual1 r;
        r.h = h;
        r.V = Volt;
        if ((rc = r(h->d_x, h->d_F, ab))) return rc;
        QS_CUDA(h, cudaMemcpyAsync(F, h->d_F, sizeof(double) * h->n_vec, cudaMemcpyDeviceToHost, h->stream));
        QS_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    *abort_flag = ab;
    return 0;
}

int qs_self_energies(qs_handle *h, const double *x, double *SigR2, double *SigL2, double *Sig1) {
    if (h->order != 2) {
        h->err = "qs_self_energies: order 2 only";
        return -1;
    }
    QS_CUDA(h, cudaSetDevice(h->device));
    int rc;
    QS_CUDA(h, cudaMemcpyAsync(h->d_F, x, sizeof(double) * h->n_vec, cudaMemcpyHostToDevice, h->stream));
    if ((rc = convert_ref_to_dl(h->stream, h->nA, h->n, h->d_F, h->d_x))) return -rc;
    if ((rc = equal_time_lesser_sigma1(h, h->d_x))) return rc;
    if ((rc = sigma2_compute(h, h->d_x, h->precision == QS_PREC_MIXED))) return rc;
    const size_t bytes = sizeof(zc) * (size_t)h->n * h->nA * h->nA;
    if (SigR2) QS_CUDA(h, cudaMemcpyAsync(SigR2, h->d_SigR, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (SigL2) QS_CUDA(h, cudaMemcpyAsync(SigL2, h->d_SigL, bytes, cudaMemcpyDeviceToHost, h->stream));
    if (Sig1) QS_CUDA(h, cudaMemcpyAsync(Sig1, h->d_Sig1, sizeof(zc) * (size_t)h->Norb * h->Norb, cudaMemcpyDeviceToHost, h->stream));
    QS_CUDA(h, cudaStreamSynchronize(h->stream));
    h->have_x = false;
    return 0;
}

// ---- stand-alone entry points with their own device buffers ----
static int simple_fail(const char *what, cudaError_t e) {
    (void)what;
    return -(int)e;
}

int qs_invert_batched(int N, int batch, double *A, int *info, int precision) {
    if (N < 1 || N > 512 || batch < 0) return -1;
    if (precision != QS_PREC_FP64) return -1;
    if (batch == 0) return 0;
    zc *dA = nullptr, *ws = nullptr;
    int *dinfo = nullptr;
    size_t bytes = sizeof(zc) * (size_t)N * N * batch;
    cudaError_t e;
    if ((e = cudaMalloc(&dA, bytes)) != cudaSuccess) return simple_fail("malloc", e);
    if ((e = cudaMalloc(&dinfo, sizeof(int) * (batch + 1))) != cudaSuccess) { cudaFree(dA); return simple_fail("malloc", e); }
    int ws_slots = 0;
    if (!dyson_fits_smem(N)) {
        ws_slots = std::min(batch, 148 * 2);
        if ((e = cudaMalloc(&ws, sizeof(zc) * (size_t)N * N * ws_slots)) != cudaSuccess) {
            cudaFree(dA);
            cudaFree(dinfo);
            return simple_fail("malloc", e);
        }
    }
    int rc = 0;
    std::vector<int> hinfo(batch + 1, 0);
    hinfo[0] = INT_MAX;
    cudaMemcpy(dA, A, bytes, cudaMemcpyHostToDevice);
    cudaMemcpy(dinfo, hinfo.data(), sizeof(int) * (batch + 1), cudaMemcpyHostToDevice);
    rc = invert_batched_dev(0, N, batch, dA, dinfo, ws, ws_slots);
    if (rc == 0) {
        e = cudaMemcpy(A, dA, bytes, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(hinfo.data(), dinfo, sizeof(int) * (batch + 1), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = -(int)e;
    }
    if (rc == 0 && info)
        for (int b = 0; b < batch; b++) info[b] = hinfo[b + 1];
    cudaFree(dA);
    cudaFree(dinfo);
    if (ws) cudaFree(ws);
    if (rc == 0 && hinfo[0] != INT_MAX) rc = 1;
    return rc;
}

}  // extern "C"

// pack_gf / unpack_gf on the device (common/linear_algebra.f90:155-233)
namespace qs {
__global__ void pack_ref(int nb, int64_t Nw, const zc *__restrict__ Gr, const zc *__restrict__ Gl, double *__restrict__ out) {
    const int nf = nb * nb, nsu = (nf - nb) / 2;
    const int64_t blk = 2 * (int64_t)nf + 2 * nsu + nb;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < Nw * blk; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t w = t / blk;
        int e = (int)(t - w * blk);
        const zc *R = Gr + w * nf, *L = Gl + w * nf;
        double v;
        if (e < 2 * nf) {
            int part = e / nf, r = e % nf, i = r / nb, j = r % nb;
            v = part ? R[i + (size_t)j * nb].y : R[i + (size_t)j * nb].x;
        } else if (e < 2 * nf + nsu) {
            int r = e - 2 * nf, i = 0, acc = 0;
            while (acc + (nb - 1 - i) <= r) { acc += nb - 1 - i; i++; }
            int j = i + 1 + (r - acc);
            v = L[i + (size_t)j * nb].x;
        } else {
            int r = e - 2 * nf - nsu, i = 0, acc = 0;
            while (acc + (nb - i) <= r) { acc += nb - i; i++; }
            int j = i + (r - acc);
            v = L[i + (size_t)j * nb].y;
        }
        out[t] = v;
    }
}
__global__ void unpack_ref(int nb, int64_t Nw, const double *__restrict__ in, zc *__restrict__ Gr, zc *__restrict__ Gl) {
    const int nf = nb * nb, nsu = (nf - nb) / 2;
    const int64_t blk = 2 * (int64_t)nf + 2 * nsu + nb;
    // one thread per (w, i, j) element pair of G^r and G^<
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < Nw * nf; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t w = t / nf;
        int r = (int)(t - w * nf), i = r % nb, j = r / nb;
        const double *b = in + w * blk;
        Gr[w * nf + i + (size_t)j * nb] = zc{b[i * nb + j], b[nf + i * nb + j]};
        int p = i <= j ? i : j, q = i <= j ? j : i;  // upper element (p, q)
        // index of (p,q) in the row-major upper enumerations
        int up = p * nb - p * (p - 1) / 2 + (q - p);         // j >= i, includes the diagonal
        int sup = p * (nb - 1) - p * (p - 1) / 2 + (q - p - 1);  // j > i
        double re = (p == q) ? 0.0 : b[2 * nf + sup];
        double im = b[2 * nf + nsu + up];
        zc v{re, im};
        Gl[w * nf + i + (size_t)j * nb] = (i <= j) ? v : zc{-v.x, v.y};  // -conj(v)
    }
}
}  // namespace qs

extern "C" {
int qs_pack_gf(int nb, int Nw, const double *Gr, const double *Gl, double *out) {
    size_t nf = (size_t)nb * nb, blk = 3 * nf;
    zc *dR, *dL;
    double *dO;
    if (cudaMalloc(&dR, sizeof(zc) * nf * Nw) != cudaSuccess) return -2;
    cudaMalloc(&dL, sizeof(zc) * nf * Nw);
    cudaMalloc(&dO, sizeof(double) * blk * Nw);
    cudaMemcpy(dR, Gr, sizeof(zc) * nf * Nw, cudaMemcpyHostToDevice);
    cudaMemcpy(dL, Gl, sizeof(zc) * nf * Nw, cudaMemcpyHostToDevice);
    count_launch();
    pack_ref<<<1184, 256>>>(nb, Nw, dR, dL, dO);
    cudaError_t e = cudaMemcpy(out, dO, sizeof(double) * blk * Nw, cudaMemcpyDeviceToHost);
    cudaFree(dR);
    cudaFree(dL);
    cudaFree(dO);
    return e == cudaSuccess ? 0 : -(int)e;
}
int qs_unpack_gf(int nb, int Nw, const double *in, double *Gr, double *Gl) {
    size_t nf = (size_t)nb * nb, blk = 3 * nf;
    zc *dR, *dL;
    double *dI;
    if (cudaMalloc(&dR, sizeof(zc) * nf * Nw) != cudaSuccess) return -2;
    cudaMalloc(&dL, sizeof(zc) * nf * Nw);
    cudaMalloc(&dI, sizeof(double) * blk * Nw);
    cudaMemcpy(dI, in, sizeof(double) * blk * Nw, cudaMemcpyHostToDevice);
    count_launch();
    unpack_ref<<<1184, 256>>>(nb, Nw, dI, dR, dL);
    cudaError_t e = cudaMemcpy(Gr, dR, sizeof(zc) * nf * Nw, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(Gl, dL, sizeof(zc) * nf * Nw, cudaMemcpyDeviceToHost);
    cudaFree(dR);
    cudaFree(dL);
    cudaFree(dI);
    return e == cudaSuccess ? 0 : -(int)e;
}

// broyden_solve with a host residual: the Broyden state (x, F, history) is on the device
struct HostResidual : BroydenResidual {
    qs_residual_fn fn;
    void *ctx;
    qs_handle *h;
    int64_t n;
    std::vector<double> x, F;
    int operator()(const double *d_x, double *d_F, bool &abort) override {
        QS_CUDA(h, cudaMemcpyAsync(x.data(), d_x, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
        QS_CUDA(h, cudaStreamSynchronize(h->stream));
        int a = 0;
        fn(ctx, n, x.data(), F.data(), &a);
        abort = a != 0;
        QS_CUDA(h, cudaMemcpyAsync(d_F, F.data(), sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
        return 0;
    }
};

int qs_broyden_solve_host(qs_residual_fn residual, void *ctx, double *x, int64_t n, double alpha_mix, int nhist, int maxscf,
                          double tolf, int single_history, int *converged, int *n_iter, double *fmax, qs_scf_step *log,
                          int log_cap) {
    qs_handle h;
    if (n < 1 || nhist < 0 || nhist > 32) return -1;
    QS_CUDA((&h), cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
    int rc = 0;
    size_t hist_el = single_history ? 4 : 8;
    h.red_len = broyden_red_len();
    if ((rc = dalloc(&h, (void **)&h.d_x, n * 8)) || (rc = dalloc(&h, (void **)&h.d_F, n * 8)) ||
        (rc = dalloc(&h, (void **)&h.d_Fold, n * 8)) || (rc = dalloc(&h, (void **)&h.d_xold, n * 8)) ||
        (rc = dalloc(&h, (void **)&h.d_red, h.red_len * 8)) ||
        (nhist > 0 && ((rc = dalloc(&h, &h.d_hdF, broyden_ld(n) * hist_el * nhist)) || (rc = dalloc(&h, &h.d_hU, broyden_ld(n) * hist_el * nhist))))) {
    } else {
        cudaMemcpyAsync(h.d_x, x, sizeof(double) * n, cudaMemcpyHostToDevice, h.stream);
        HostResidual r;
        r.fn = residual;
        r.ctx = ctx;
        r.h = &h;
        r.n = n;
        r.x.resize(n);
        r.F.resize(n);
        BroydenOut bo;
        rc = broyden_solve_dev(&h, r, h.d_x, h.d_F, h.d_Fold, h.d_xold, h.d_hdF, h.d_hU, n, alpha_mix, nhist, maxscf, tolf,
                               single_history != 0, bo);
        if (rc == 0) {
            cudaMemcpyAsync(x, h.d_x, sizeof(double) * n, cudaMemcpyDeviceToHost, h.stream);
            cudaStreamSynchronize(h.stream);
            *converged = bo.converged;
            *n_iter = bo.n_iter;
            *fmax = bo.fmax;
            for (int i = 0; i < (int)bo.log.size() && i < log_cap; i++) log[i] = bo.log[i];
        }
    }
    release_all(&h);
    cudaStreamDestroy(h.stream);
    return rc;
}

}  // extern "C"
