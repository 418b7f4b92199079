// sancho_gpu_main.cpp -- the SANCHO program on the B200 solver (drop-in for SANCHO's
// bin/sancho.x). Usage: sancho_b200 [case_dir] (default: the current directory).
// Environment: QS_DEVICE (CUDA device ordinal, default 0).
#include <cstdio>
#include <cstdlib>

#include "qsa_host.h"

int main(int argc, char **argv) {
    qsah_solver_api api{};
    api.name = "b200";
    api.create = (int (*)(const qsa_problem *, void **))qsa_create;
    api.destroy = (void (*)(void *))qsa_destroy;
    api.last_error = (const char *(*)(const void *))qsa_last_error;
    api.solve_scf = (int (*)(void *, double, int, qs_scf_result *))qsa_solve_scf;
    api.current = (int (*)(void *, double, double *))qsa_current;
    api.get_observables = (int (*)(void *, double *, double *))qsa_get_observables;
    const char *dev = std::getenv("QS_DEVICE");
    return qsah_run(argc > 1 ? argv[1] : ".", &api, dev ? std::atoi(dev) : 0, stdout);
}
