// qs_main.cpp -- the QUICHOTTE program flow (src/quichotte.f90:31-166) over a solver
// library: read input.dat, build the model, sweep the voltages, write the output files.
//
// The reference program does, per voltage V1 = V + k*delv (src/quichotte.f90:285-303):
//   solve_scf -> Current -> Volt_Current_<order>.dat -> spin_texture -> atom_texture
//   -> write_spectral, with continuation from the previous converged voltage.
// Exit codes follow src/quichotte.f90:188-189 and 321-325: 0 all converged, 1 bad input
// (or a singular Dyson matrix, common/linear_algebra.f90:73-76), 3 some voltage did not
// converge. A CUDA or memory failure of the solver returns 2.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "qs_host.h"

extern "C" int qsh_run(const char *dir, const qsh_solver_api *api, int precision, int device, FILE *log) {
    auto t0 = std::chrono::steady_clock::now();
    std::string d = dir ? dir : ".";
    auto P = [&](const char *f) { return d + "/" + f; };
    char err[4096] = {0};
    qsh_model *m = nullptr;
    if (qsh_load_with(d.c_str(), api, device, &m, err, sizeof err, log) != 0) {
        std::fprintf(stderr, "%s\n", err);
        return 1;
    }
    if (m->write_hamiltonian) qsh_write_hamiltonian_matrix(m, P("hamiltonian_matrix.dat").c_str());
    qsh_write_hamiltonian_info(m, P("info_Hamiltonian.dat").c_str());
    if (log)
        std::fprintf(log, " n_omega: %d  w_fin: %.10f  w_init: %.10f  solver: %s\n", m->n_omega, m->w_fin, m->w_init,
                     api->name);

    qs_problem p{};
    p.Norb = m->Norb;
    p.N_sites = m->N_sites;
    p.N_atoms = m->N_atoms;
    p.order = m->order;
    p.n_omega = m->n_omega;
    p.H = m->H;
    p.GammaL = m->GammaL;
    p.GammaR = m->GammaR;
    p.U_site = m->U_site;
    p.omega = m->omega;
    p.atom_norb = m->atom_norb;
    p.atom_first = m->atom_first;
    p.mu = m->mu;
    p.beta = m->beta;
    p.delta = m->delta;
    p.alpha_mix = m->alpha_mix;
    p.tolf = m->tolf;
    p.tolf_order1 = m->tolf_order1;
    p.nhist = m->nhist;
    p.maxscf = m->maxscf;
    p.single_history = m->broyden_single_precision;
    p.precision = precision;
    p.device = device;

    void *h = nullptr;
    int rc = api->create(&p, &h);
    if (rc != 0) {
        std::fprintf(stderr, "ERROR: solver set-up failed (%d): %s\n", rc, h ? api->last_error(h) : "");
        if (h) api->destroy(h);
        qsh_free(m);
        return 2;
    }

    char name[64];
    std::snprintf(name, sizeof name, "Volt_Current_%d.dat", m->order);
    FILE *u_iv = std::fopen(P(name).c_str(), "w");
    FILE *u_pop = std::fopen(P("populations.dat").c_str(), "w");
    FILE *u_spec = std::fopen(P("spectral_function.dat").c_str(), "w");
    FILE *u_popat = m->per_atom ? std::fopen(P("populations_atoms.dat").c_str(), "w") : nullptr;
    FILE *u_rt = std::fopen(P("runtime_datasheet.dat").c_str(), "w");
    if (u_rt) std::fprintf(u_rt, " >>>>>>>>>>>>>>>>>>>>>>>>>>>>Runtime Data Sheet>>>>>>>>>>>>>>>>>>>>>>>>>>>>\n QUICHOTTE on B200, solver: %s\n", api->name);

    std::vector<qs_scf_step> steps(std::max(m->maxscf, 1) + 1);
    std::vector<double> Gl((size_t)2 * m->Norb * m->Norb), dosd((size_t)m->Norb * m->n_omega);
    bool fresh = true;
    int n_unconv = 0, status = 0;
    for (int k = 0; k <= m->n_volt_steps; k++) {
        double V1 = m->V + k * m->delv;
        if (u_rt) std::fprintf(u_rt, " ........SCF Calculations at Voltage: %.17g ..........\n", V1);
        qs_scf_result res{};
        res.log = steps.data();
        res.log_cap = (int)steps.size();
        rc = api->solve_scf(h, V1, fresh ? 1 : 0, &res);
        if (rc != 0) {
            std::fprintf(stderr, "ERROR: %s\n", api->last_error(h));
            status = rc > 0 ? 1 : 2;
            break;
        }
        // scf_V_<V>.dat (src/scf.f90:97-99,128-129; common/broyden_mixing.f90:83,94)
        char fn[64];
        qsh_scf_log_name(V1, fn, sizeof fn);
        if (FILE *u = std::fopen(P(fn).c_str(), "w")) {
            std::fprintf(u, "#  step        max|F|          rms|F|   nhist\n");
            for (int i = 0; i < res.n_log; i++) qsh_write_scf_line(u, steps[i].step, steps[i].fmax, steps[i].rms, steps[i].nh);
            std::fclose(u);
        }
        if (log) {
            if (!res.converged && !res.unphysical)
                std::fprintf(log, " NOT CONVERGED after %5d steps, max|F| = %11.3E\n", res.n_iter, res.fmax);
            else if (!res.converged)
                std::fprintf(log, " CONVERGED TO AN UNPHYSICAL SOLUTION: state %4d n = %11.3E, spectral weight = %11.3E\n",
                             res.i_worst, res.n_worst, res.w_worst);
            else
                std::fprintf(log, " V = %9.4f ... CONVERGED in %5d steps ... (%.3f s)\n", V1, res.n_iter, res.seconds);
        }
        if (!res.converged) n_unconv++;
        fresh = (!m->continuation) || (!res.converged);

        double Ju = 0, Jd = 0;
        api->current(h, V1, &Ju, &Jd);
        qsh_write_iv(u_iv, V1, Ju, Jd, res.converged);
        api->get_observables(h, Gl.data(), dosd.data(), nullptr, nullptr);
        qsh_write_spin_texture(u_pop, m, V1, Gl.data());
        if (u_popat) qsh_write_atom_texture(u_popat, m, V1, Gl.data());
        qsh_write_spectral(u_spec, m, V1, dosd.data());
    }
    std::fclose(u_iv);
    std::fclose(u_pop);
    std::fclose(u_spec);
    if (u_popat) std::fclose(u_popat);
    double mins = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() / 60.0;
    if (u_rt) {
        std::fprintf(u_rt, " <<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<\n Total Runtime: %.8f mins\n", mins);
        std::fclose(u_rt);
    }
    api->destroy(h);
    qsh_free(m);
    if (status) return status;
    if (n_unconv > 0) {
        if (log) std::fprintf(log, " WARNING: %d voltage(s) did not converge (column 5 = 0 in Volt_Current)\n", n_unconv);
        return 3;
    }
    return 0;
}
