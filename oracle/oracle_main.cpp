// oracle_main.cpp -- TEST INFRASTRUCTURE: the QUICHOTTE program run by the CPU oracle.
// Usage: quichotte_oracle [case_dir]. Same input.dat, output files and exit codes as the
// reference binary (src/quichotte.f90), so a case directory of the reference's
// regression suite runs unchanged.
#include <cstdio>

#include "../include/qs_host.h"

struct qso_state;
extern "C" {
int qso_create(const qs_problem *p, qso_state **out);
void qso_destroy(qso_state *s);
const char *qso_last_error(const qso_state *s);
int qso_solve_scf(qso_state *s, double Volt, int fresh_start, qs_scf_result *res);
int qso_current(qso_state *s, double Volt, double *J_up, double *J_down);
int qso_get_observables(qso_state *s, double *G_less_obs, double *dosd, double *trU, double *trD);
}

int main(int argc, char **argv) {
    qsh_solver_api api{};
    api.name = "cpu-oracle";
    api.create = (int (*)(const qs_problem *, void **))qso_create;
    api.destroy = (void (*)(void *))qso_destroy;
    api.last_error = (const char *(*)(const void *))qso_last_error;
    api.solve_scf = (int (*)(void *, double, int, qs_scf_result *))qso_solve_scf;
    api.current = (int (*)(void *, double, double *, double *))qso_current;
    api.get_observables = (int (*)(void *, double *, double *, double *, double *))qso_get_observables;
    return qsh_run(argc > 1 ? argv[1] : ".", &api, QS_PREC_FP64, 0, stdout);
}
