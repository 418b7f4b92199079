/*
 * qsa200.h -- C ABI of the B200 (sm_100a) solver for SANCHO (libqsb200.so): the spinless
 * chain to third order in U, with the second- and third-order self-energies as
 * particle-hole / particle-particle bubble sums over the energy grid.
 *
 * Each entry point names the reference routine it replaces (file:line, paths relative to
 * the reference project's SANCHO/ directory). Conventions as in qsb200.h: column-major
 * complex(dp) arrays as double pairs, packed SCF vectors in pack_gf's layout
 * (common/linear_algebra.f90:155-191) with nb = N_sites, status 0 / > 0 (a numerical stop
 * of the reference, e.g. a singular Dyson matrix) / < 0 (CUDA or admission failure).
 */
#ifndef QSA200_H
#define QSA200_H

#include <stdint.h>

#include "qsb200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The module globals of Parameters / Hamiltonian / GreenFunctions after set-up
 * (src/parameters.f90, src/sancho.f90:58-92). One orbital per site. */
typedef struct qsa_problem {
    int N_sites, order, n_omega;
    const double *H;      /* N_sites*N_sites complex, column-major              */
    const double *GammaL; /* N_sites*N_sites complex (site 1)                   */
    const double *GammaR; /* N_sites*N_sites complex (last site)                */
    const double *U_site; /* N_sites                                            */
    const double *omega;  /* n_omega energies                                   */
    double mu, beta, delta;
    double alpha_mix, tolf;
    int nhist, maxscf;
    int device;
} qsa_problem;

typedef struct qsa_handle qsa_handle;

/* Storage and sizes (src/sancho.f90:94-110): G_in, G_out on the whole grid, n_vec. */
int qsa_create(const qsa_problem *p, qsa_handle **h);
void qsa_destroy(qsa_handle *h);
const char *qsa_last_error(const qsa_handle *h);
int64_t qsa_vector_length(const qsa_handle *h);

/* solve_scf(Volt, fresh_start, converged) (src/scf.f90:53-95): the non-interacting start
 * or continuation, Broyden over the device residual (double-precision history, as the
 * reference calls broyden_solve), check_gf_sanity on G_out. res->converged, n_iter, fmax,
 * aborted, runaway, unphysical, i_worst, n_worst, w_worst, log, seconds as in qsb200.h. */
int qsa_solve_scf(qsa_handle *h, double Volt, int fresh_start, qs_scf_result *res);

/* Current(Volt) (src/observables.f90:18-52), from the last residual's input G_in. */
int qsa_current(qsa_handle *h, double Volt, double *J);

/* What write_populations and write_spectral print (src/observables.f90:54-82): G_less_t0
 * (N_sites complex) and the spectral function A_ii(w) = -2 Im G^r_ii(w) (N_sites x n_omega,
 * site fastest). Either pointer may be NULL. */
int qsa_get_observables(qsa_handle *h, double *G_less_t0, double *spectral);

/* noninteracting_gr_ga + noninteracting_gl_gg + pack_gf (src/green_functions.f90:55-96):
 * the fresh-start SCF vector. */
int qsa_initial_vector(qsa_handle *h, double Volt, double *x);

/* scf_residual + interacting_gf (src/scf.f90:102-195): F = pack(G_out[x]) - x, abort on a runaway. */
int qsa_residual(qsa_handle *h, double Volt, const double *x, double *F, int *abort_flag);

/* complete_input_gf + build_self_energies (src/green_functions.f90:164-173,
 * src/self_energies.f90:40-207) for the G_in of
 * x: Sigma2^r, Sigma2^< and (order 3) Sigma3^r, Sigma3^< as (N_sites, N_sites, n_omega)
 * complex arrays; any pointer may be NULL. */
int qsa_self_energies(qsa_handle *h, const double *x, double *Sig2R, double *Sig2L, double *Sig3R,
                      double *Sig3L);

/* Extension (no counterpart in SANCHO): per-family device time in ms and launch counts since
 * the last call, as qs_profile (enable 1/0 switches event timing on/off, -1 only reads).
 * Families: 0 Dyson (W build + inversion), 1 Keldysh (products + pack), 2 bubbles chi/phi,
 * 3 order-3 products D/E, 4 self-energy convolutions, 5 (unused), 6 Broyden, 7 reductions,
 * 8 other. Returns the number of families. */
int qsa_profile(qsa_handle *h, int enable, double *ms, int64_t *launches, int nfam);

#ifdef __cplusplus
}
#endif
#endif
