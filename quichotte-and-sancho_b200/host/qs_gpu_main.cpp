// qs_gpu_main.cpp -- the QUICHOTTE program on the B200 solver (drop-in for bin/quichotte.x).
// Usage: quichotte_b200 [case_dir]   (default: the current directory)
// Environment: QS_DEVICE (CUDA device ordinal, default 0).
#include <cstdio>
#include <cstdlib>

#include "qs_host.h"
#include "qsb200.h"

int main(int argc, char **argv) {
    qsh_solver_api api{};
    api.name = "b200";
    api.create = (int (*)(const qs_problem *, void **))qs_create;
    api.destroy = (void (*)(void *))qs_destroy;
    api.last_error = (const char *(*)(const void *))qs_last_error;
    api.solve_scf = (int (*)(void *, double, int, qs_scf_result *))qs_solve_scf;
    api.current = (int (*)(void *, double, double *, double *))qs_current;
    api.get_observables = (int (*)(void *, double *, double *, double *, double *))qs_get_observables;
    api.hermitian_eigenvalues = qs_hermitian_eigenvalues;
    api.dftb_lowdin = qs_dftb_lowdin;
    const char *dev = std::getenv("QS_DEVICE");
    return qsh_run(argc > 1 ? argv[1] : ".", &api, QS_PREC_FP64, dev ? std::atoi(dev) : 0, stdout);
}
