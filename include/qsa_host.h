/*
 * qsa_host.h -- host layer of SANCHO on B200 (libqs_host.so): input.dat reader, the chain
 * models, the energy grid, the voltage sweep and the reference's output files. The solver
 * behind it is any library with the entry points of qsa200.h (the B200 solver, or the CPU
 * oracle that checks it).
 *
 * Restates SANCHO/src/sancho.f90 (program flow), SANCHO/src/input_output.f90:28-132
 * (read_input, check_input, setup_hubbard), SANCHO/src/hamiltonian.f90:35-137 (chain and
 * custom models) and the file output of SANCHO/src/observables.f90:54-82. Returns 0, or the
 * reference's exit codes: 1 for an input error, 3 when some voltage did not converge.
 */
#ifndef QSA_HOST_H
#define QSA_HOST_H

#include <stdio.h>

#include "qsa200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct qsah_model {
    int N_sites, order, n_omega, n_volt_steps, nhist, maxscf, continuation;
    double V, Vf, delv, T, mu, beta, delta, w_init, w_fin, dw, up, alpha_mix, tolf;
    double *H, *GammaL, *GammaR; /* N_sites x N_sites complex, column-major */
    double *U_site, *omega, *Ev;
    char model_name[32];
} qsah_model;

/* read_input + build_hamiltonian + leads + setup_hubbard + grid of the case in dir. */
int qsah_load(const char *dir, qsah_model **out, char *errbuf, int errlen, FILE *log);
void qsah_free(qsah_model *m);

typedef struct qsah_solver_api {
    const char *name;
    int (*create)(const qsa_problem *, void **);
    void (*destroy)(void *);
    const char *(*last_error)(const void *);
    int (*solve_scf)(void *, double, int, qs_scf_result *);
    int (*current)(void *, double, double *);
    int (*get_observables)(void *, double *, double *);
} qsah_solver_api;

/* The SANCHO program in dir with the given solver (device: CUDA device for the B200 one). */
int qsah_run(const char *dir, const qsah_solver_api *api, int device, FILE *log);

#ifdef __cplusplus
}
#endif
#endif
