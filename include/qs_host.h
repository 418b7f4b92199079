/*
 * qs_host.h -- C ABI of the QUICHOTTE host layer (input, model set-up, output files).
 *
 * This is the host side that sits above the NEGF solver (qsb200.h). It restates the
 * parts of the reference program that are not on the hot path but that every run needs:
 *
 *   qsh_load          read_input + build_hamiltonian + setup_leads + setup_hubbard +
 *                     the energy grid (src/input_output.f90:31-139,310-346,432-462,
 *                     src/hamiltonian.f90:44-63, src/quichotte.f90:224-253)
 *   qsh_write_*       the output files of src/quichotte.f90:268-306 and
 *                     src/observables.f90:41-158, in gfortran's list-directed layout
 *
 * All matrices are column-major (Fortran order). Complex numbers are two doubles
 * (re, im), i.e. C99 `double _Complex` / Fortran `complex(dp)` memory layout.
 * Indices in atom_first are 1-based, as in the reference.
 *
 * Error convention: functions return 0 on success. qsh_load returns 1 for an input
 * that the reference rejects with `stop 1`, with the message in errbuf.
 */
#ifndef QS_HOST_H
#define QS_HOST_H

#include <stdint.h>
#include <stdio.h>

#include "qsb200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct qsh_model {
    /* sizes (src/parameters.f90:17-24) */
    int N_sites, Norb, N_atoms, order, n_omega, n_volt_steps;
    /* voltage sweep, temperature, grid (src/parameters.f90:50-56) */
    double V, Vf, delv, T, mu, beta;
    double delta, w_init, w_fin, dw, up;
    double Ev_min, Ev_max;
    /* SCF settings (src/scf.f90:38-43) */
    double alpha_mix, tolf, tolf_order1;
    int nhist, maxscf, continuation, broyden_single_precision;
    int write_hamiltonian, per_atom;
    /* arrays owned by the model (freed by qsh_free) */
    double *H;       /* Norb*Norb complex, column-major                    */
    double *GammaL;  /* Norb*Norb complex                                  */
    double *GammaR;  /* Norb*Norb complex                                  */
    double *U_site;  /* Norb: U on the spin-up index of each site, 0 else  */
    double *omega;   /* n_omega: omega(i) = w_init + i*delta, i = 1..n     */
    double *Ev;      /* Norb eigenvalues of H, ascending                   */
    int *atom_norb;  /* N_atoms                                            */
    int *atom_first; /* N_atoms, 1-based first site of each atom           */
    char model_name[32];
    char input_file[32];
} qsh_model;

/* Read <dir>/input.dat (or inputSOC.dat) and build the model. Returns 0, or 1 with
 * the reference's error message in errbuf. Warnings go to `log` if non-NULL. */
int qsh_load(const char *dir, qsh_model **out, char *errbuf, int errlen, FILE *log);
/* qsh_load with the set-up linear algebra of `api` where it provides it, on CUDA device
 * `device` (api NULL: qsh_load). The solver API type is declared below. */
struct qsh_solver_api;
int qsh_load_with(const char *dir, const struct qsh_solver_api *api, int device, qsh_model **out, char *errbuf,
                  int errlen, FILE *log);
void qsh_free(qsh_model *m);

/* Synthetic helix model without an input file (the input.dat keys of a helix run). */
int qsh_helix(int N_ions, int N_turns, double hel_length, double hel_radius, double hand,
              double E_CC, double t_hop, double lamb, double U_int, double GammaL_up,
              double GammaL_down, double GammaR, double T, double mu, double dw, double up,
              double delta, int order, qsh_model **out);

/* gfortran list-directed formatting of one REAL(8) / INTEGER item (26 / 12 chars). */
int qsh_fmt_real(double x, char *buf);
int qsh_fmt_int(long v, char *buf);

/* Output files of the reference, appended to open streams. */
int qsh_write_iv(FILE *f, double V, double J_up, double J_down, int converged);
int qsh_write_spin_texture(FILE *f, const qsh_model *m, double V, const double *G_less_obs);
int qsh_write_atom_texture(FILE *f, const qsh_model *m, double V, const double *G_less_obs);
int qsh_write_spectral(FILE *f, const qsh_model *m, double V, const double *dosd);
int qsh_write_hamiltonian_matrix(const qsh_model *m, const char *path);
int qsh_write_hamiltonian_info(const qsh_model *m, const char *path);

/* One line of scf_V_<V>.dat: '(i6,2es16.6,i6)' (common/broyden_mixing.f90:94). */
int qsh_write_scf_line(FILE *f, int step, double fmax, double rms, int nh);
/* scf_V_<V>.dat file name for a voltage (src/scf.f90:98-99). */
int qsh_scf_log_name(double V, char *buf, int len);

/* The solver behind the program: the B200 library (qs_*) or any library with the same
 * entry points. qsh_run uses only these. */
typedef struct qsh_solver_api {
    const char *name;
    int (*create)(const qs_problem *p, void **h);
    void (*destroy)(void *h);
    const char *(*last_error)(const void *h);
    int (*solve_scf)(void *h, double Volt, int fresh_start, qs_scf_result *res);
    int (*current)(void *h, double Volt, double *J_up, double *J_down);
    int (*get_observables)(void *h, double *G_less_obs, double *dosd, double *trU, double *trD);
    /* optional: the set-up's dense linear algebra (qs_hermitian_eigenvalues, qs_dftb_lowdin
     * of qsb200.h); NULL uses the host's own (cyclic Jacobi and plain products) */
    int (*hermitian_eigenvalues)(int N, int batch, const double *A, double *E, int *info, int device);
    int (*dftb_lowdin)(int N, const double *S, const double *H0, const double *Lam, int soc_dual, double *H,
                       double *evmin, int device);
} qsh_solver_api;

/* The program QUICHOTTE (src/quichotte.f90:31-166) on <dir>: reads input.dat, runs
 * the voltage sweep through `api` and writes the reference's output files into <dir>.
 * Returns the reference's exit code: 0, 1 (bad input) or 3 (some voltage did not
 * converge); 2 for a solver failure the reference would stop on. precision and device
 * are passed to the solver (QS_PREC_FP64 for the reference's arithmetic). */
int qsh_run(const char *dir, const qsh_solver_api *api, int precision, int device, FILE *log);

#ifdef __cplusplus
}
#endif
#endif
