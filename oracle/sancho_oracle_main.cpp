// sancho_oracle_main.cpp -- TEST INFRASTRUCTURE: the SANCHO program run by the CPU oracle.
// Usage: sancho_oracle [case_dir]. Same input.dat, output files and exit codes as SANCHO's
// reference binary (SANCHO/src/sancho.f90), so a case of its regression suite runs unchanged.
#include <cstdio>

#include "../include/qsa_host.h"

struct qsao_state;
extern "C" {
int qsao_create(const qsa_problem *p, qsao_state **out);
void qsao_destroy(qsao_state *s);
const char *qsao_last_error(const qsao_state *s);
int qsao_solve_scf(qsao_state *s, double Volt, int fresh_start, qs_scf_result *res);
int qsao_current(qsao_state *s, double Volt, double *J);
int qsao_get_observables(qsao_state *s, double *G_less_t0, double *spectral);
}

int main(int argc, char **argv) {
    qsah_solver_api api{};
    api.name = "cpu-oracle";
    api.create = (int (*)(const qsa_problem *, void **))qsao_create;
    api.destroy = (void (*)(void *))qsao_destroy;
    api.last_error = (const char *(*)(const void *))qsao_last_error;
    api.solve_scf = (int (*)(void *, double, int, qs_scf_result *))qsao_solve_scf;
    api.current = (int (*)(void *, double, double *))qsao_current;
    api.get_observables = (int (*)(void *, double *, double *))qsao_get_observables;
    return qsah_run(argc > 1 ? argv[1] : ".", &api, 0, stdout);
}
