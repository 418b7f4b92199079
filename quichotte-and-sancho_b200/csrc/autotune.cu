// autotune.cu -- a process-wide table of kernel-variant choices, filled by timing.
//
// Some steps have more than one kernel whose relative speed depends on the problem size
// (Dyson: blocked Gauss-Jordan on the FP64 tensor cores or the unblocked kernel; Keldysh:
// tensor-core or CUDA-core GEMMs). The first launch of a step at a size not yet in the table
// times every candidate on the handle's own inputs (CUDA events on its stream) and records
// the fastest; later launches at that size, from any handle of the process, use the
// recorded choice (each candidate timed twice, the faster run counting). Every candidate
// computes the same step; the chosen one is launched last,
// so the step's output is always the recorded variant's (bit-identical results whether or
// not this launch did the tuning).
#include <map>
#include <mutex>
#include <utility>

#include "qs_common.cuh"

namespace qs {

static std::mutex g_tune_mu;
static std::map<std::pair<int, int>, int> g_tune;
// 1: tune; 0: the size heuristics only; 2 / 3: the first / last applicable candidate; 4: the
// second of three (tests force each variant this way)
static int g_tune_mode = 1;

static int tune_mode() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    return g_tune_mode;
}

int tune_get(int kind, int size) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (g_tune_mode != 1) return -1;
    auto it = g_tune.find({kind, size});
    return it == g_tune.end() ? -1 : it->second;
}

bool tune_enabled() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    return g_tune_mode != 0;
}

void tune_put(int kind, int size, int choice) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.emplace(std::make_pair(kind, size), choice);
}

int tune_launch(qs_handle *h, int kind, int size, const int *cand, int ncand, int fallback,
                const std::function<int(int)> &launch) {
    const int mode = tune_mode();
    if (mode == 2 || mode == 3) return launch(cand[mode == 2 ? 0 : ncand - 1]);
    if (mode == 4) return launch(cand[ncand >= 3 ? 1 : 0]);
    if (ncand <= 1 || mode == 0) return launch(ncand == 1 ? cand[0] : fallback);
    const int known = tune_get(kind, size);
    if (known >= 0) return launch(known);
    cudaEvent_t e0, e1;
    QS_CUDA(h, cudaEventCreate(&e0));
    QS_CUDA(h, cudaEventCreate(&e1));
    // every candidate timed twice, in alternation, and judged by its faster run: other work
    // on the device (the serving loop's concurrent solves) slows single runs unevenly
    int best = cand[0];
    float best_ms = 0.0f;
    float cand_ms[8];
    for (int c = 0; c < ncand && c < 8; c++) cand_ms[c] = 0.0f;
    for (int rep = 0; rep < 2; rep++)
        for (int c = 0; c < ncand && c < 8; c++) {
            QS_CUDA(h, cudaEventRecord(e0, h->stream));
            int rc = launch(cand[c]);
            if (rc) {
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                return rc;
            }
            QS_CUDA(h, cudaEventRecord(e1, h->stream));
            QS_CUDA(h, cudaEventSynchronize(e1));
            float ms = 0.0f;
            QS_CUDA(h, cudaEventElapsedTime(&ms, e0, e1));
            if (rep == 0 || ms < cand_ms[c]) cand_ms[c] = ms;
        }
    for (int c = 0; c < ncand && c < 8; c++)
        if (c == 0 || cand_ms[c] < best_ms) {
            best_ms = cand_ms[c];
            best = cand[c];
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    tune_put(kind, size, best);  // the first record wins when threads tune a size at once
    // the step's output comes from the recorded choice, as on every later launch: results
    // do not depend on when, or by which thread, the size was tuned
    const int chosen = tune_get(kind, size);
    const int use = chosen >= 0 ? chosen : best;
    return use == cand[ncand - 1] ? 0 : launch(use);
}

}  // namespace qs

extern "C" {

int qs_autotune(int mode) {
    std::lock_guard<std::mutex> lk(qs::g_tune_mu);
    if (mode < 0) qs::g_tune.clear();
    else if (mode <= 4) qs::g_tune_mode = mode;
    else return -1;
    return 0;
}

int qs_tuned_choice(int kind, int size) { return qs::tune_get(kind, size); }

}  // extern "C"
