// sancho_host.cpp -- host layer of SANCHO on B200 (include/qsa_host.h): input.dat, the chain
// models, the energy grid, the voltage sweep and the output files, over any solver with the
// qsa200.h entry points. Paths are relative to the reference project's SANCHO/ directory.
//   src/input_output.f90:28-132   read_input (keys, aliases, defaults), check_input, setup_hubbard
//   src/hamiltonian.f90:35-137    build_hamiltonian: chain, custom (the chain written out)
//   src/sancho.f90:47-167         program flow: leads on the first and last site, grid from the
//                                 spectrum, the sweep with continuation, exit codes 0 / 1 / 3
//   src/observables.f90:54-82     populations.dat and spectral_function.dat records
#include "qsa_host.h"

#include <chrono>
#include <cstring>

#include "qs_host.h"
#include "host_common.hpp"

namespace {

struct SModel {
    int Nsites = 0, order = 0, n_omega = 0, n_volt_steps = 0, nhist = 8, maxscf = 200;
    bool continuation = true;
    double V = 0, Vf = 0, delv = 0, T = 0, mu = 0, beta = 0, delta = 0, dw = 0, up = 0, E_CC = 0, t_hop = 0, U_int = 0;
    double GammaL = 1.0, GammaR = 1.0, alpha_mix = 0.3, tolf = 1e-6, w_init = 0, w_fin = 0;
    std::string model = "chain", hubbard_file;
    std::vector<cplx> H;
    std::vector<double> U, omega, Ev;
};

// read_input + check_input (src/input_output.f90:28-104)
void read_input(const std::string &dir, SModel &m, FILE *log) {
    InputParser ip;
    ip.log = log;
    ip.load(dir, {"input.dat"});
    const double d1 = 1.0, d03 = 0.3, d1em6 = 1e-6;
    const int i8 = 8, i200 = 200;
    const bool bt = true, bf = false;
    ip.get("V", m.V);
    ip.get("Vf", m.Vf);
    ip.get("delv", m.delv);
    ip.get("T", m.T);
    ip.get("mu", m.mu);
    ip.get("hamiltonian", m.model, "chain");
    ip.get("N_sites", m.Nsites, nullptr, "Nsites,Natoms");
    ip.get("E_CC", m.E_CC);
    ip.get("t_hop", m.t_hop);
    ip.get("U_int", m.U_int);
    ip.get("hubbard_file", m.hubbard_file, "");
    ip.get("order", m.order);
    ip.get("GammaL", m.GammaL, &d1);
    ip.get("GammaR", m.GammaR, &d1);
    ip.get("dw", m.dw);
    ip.get("up", m.up);
    ip.get("delta", m.delta);
    ip.get("alpha_mix", m.alpha_mix, &d03);
    ip.get("nhist", m.nhist, &i8);
    ip.get("maxscf", m.maxscf, &i200);
    ip.get("tolf", m.tolf, &d1em6);
    ip.get("continuation", m.continuation, &bt);
    bool restart_unused;
    std::string ver_unused;
    ip.get("restart", restart_unused, &bf);
    ip.get("ver", ver_unused, "");
    ip.finish();
    m.beta = 1.0 / (kB * m.T);
    m.n_volt_steps = (int)std::lround((m.Vf - m.V) / m.delv);
    std::string e;
    auto complain = [&](const char *msg) { e += std::string(" ERROR in input: ") + msg + "\n"; };
    if (m.Nsites < 1) complain("N_sites must be >= 1");
    if (m.order < 0 || m.order > 3) complain("order must be 0, 1, 2 or 3");
    if (m.delta <= 0.0) complain("delta (energy grid step) must be > 0");
    if (m.delv <= 0.0) complain("delv (voltage step) must be > 0");
    if (m.Vf < m.V) complain("Vf must be >= V");
    if (m.T <= 0.0) complain("T must be > 0");
    if (m.nhist < 0) complain("nhist must be >= 0");
    if (m.maxscf < 1) complain("maxscf must be >= 1");
    if (m.tolf <= 0.0) complain("tolf must be > 0");
    if (m.GammaL < 0.0 || m.GammaR < 0.0) complain("GammaL, GammaR must be >= 0");
    if (!e.empty()) throw InputError(e);
}

// build_hamiltonian (src/hamiltonian.f90:35-137): chain, or the custom template as shipped
// (the same chain, filled triangle by triangle)
void build_hamiltonian(SModel &m) {
    const int n = m.Nsites;
    m.H.assign((size_t)n * n, 0.0);
    auto h = [&](int i, int j) -> cplx & { return m.H[i + (size_t)j * n]; };
    if (m.model == "chain") {
        for (int i = 0; i < n; i++) {
            h(i, i) = m.E_CC;
            for (int j = 0; j < n; j++)
                if (i == j + 1 || j == i + 1) h(i, j) = m.t_hop;
        }
    } else if (m.model == "custom") {
        for (int i = 0; i < n; i++) h(i, i) = m.E_CC;
        for (int i = 0; i + 1 < n; i++) {
            h(i, i + 1) = m.t_hop;
            h(i + 1, i) = std::conj(h(i, i + 1));
        }
    } else {
        throw InputError(" ERROR: unknown hamiltonian = " + m.model + "\n        built in: chain, custom (see src/hamiltonian.f90)");
    }
}

// setup_hubbard (src/input_output.f90:106-132)
void setup_hubbard(const std::string &dir, SModel &m) {
    m.U.assign(m.Nsites, m.U_int);
    if (m.hubbard_file.empty()) return;
    std::ifstream f(dir + "/" + trim(m.hubbard_file));
    if (!f.good()) throw InputError(" ERROR: cannot open hubbard_file " + trim(m.hubbard_file));
    std::string line;
    for (int i = 0; i < m.Nsites; i++) {
        double v;
        if (!std::getline(f, line) || !read_real(line, v))
            throw InputError(" ERROR: " + trim(m.hubbard_file) + " needs one U per site (" + std::to_string(m.Nsites) +
                             " lines)");
        m.U[i] = v;
    }
}

// the whole set-up of src/sancho.f90:58-92: input, H, leads, U, grid
void load_model(const std::string &dir, SModel &m, FILE *log) {
    read_input(dir, m, log);
    build_hamiltonian(m);
    setup_hubbard(dir, m);
    std::vector<cplx> Z;
    jacobi_herm(m.Nsites, m.H, m.Ev, Z);
    m.w_init = m.Ev.front() - m.dw;
    m.w_fin = m.Ev.back() + m.up;
    m.n_omega = (int)((m.w_fin - m.w_init) / m.delta);
    if (m.n_omega < 1) throw InputError(" ERROR: the energy grid is empty (check dw, up, delta)");
    m.omega.resize(m.n_omega);
    for (int i = 1; i <= m.n_omega; i++) m.omega[i - 1] = m.w_init + i * m.delta;
}

template <class T> T *copy_out(const std::vector<T> &v) {
    T *p = (T *)std::malloc(sizeof(T) * std::max<size_t>(v.size(), 1));
    if (!v.empty()) std::memcpy(p, v.data(), sizeof(T) * v.size());
    return p;
}

}  // namespace

extern "C" {

int qsah_load(const char *dir, qsah_model **out, char *errbuf, int errlen, FILE *log) {
    *out = nullptr;
    SModel m;
    try {
        load_model(dir ? dir : ".", m, log);
    } catch (const InputError &e) {
        if (errbuf && errlen > 0) std::snprintf(errbuf, errlen, "%s", e.what());
        return 1;
    }
    auto *q = (qsah_model *)std::calloc(1, sizeof(qsah_model));
    q->N_sites = m.Nsites;
    q->order = m.order;
    q->n_omega = m.n_omega;
    q->n_volt_steps = m.n_volt_steps;
    q->nhist = m.nhist;
    q->maxscf = m.maxscf;
    q->continuation = m.continuation;
    q->V = m.V;
    q->Vf = m.Vf;
    q->delv = m.delv;
    q->T = m.T;
    q->mu = m.mu;
    q->beta = m.beta;
    q->delta = m.delta;
    q->w_init = m.w_init;
    q->w_fin = m.w_fin;
    q->dw = m.dw;
    q->up = m.up;
    q->alpha_mix = m.alpha_mix;
    q->tolf = m.tolf;
    const size_t nn = (size_t)m.Nsites * m.Nsites;
    std::vector<cplx> GL(nn, 0.0), GR(nn, 0.0);
    GL[0] = m.GammaL;                                                    // site 1
    GR[(m.Nsites - 1) + (size_t)(m.Nsites - 1) * m.Nsites] = m.GammaR;  // the last site
    q->H = (double *)copy_out(m.H);
    q->GammaL = (double *)copy_out(GL);
    q->GammaR = (double *)copy_out(GR);
    q->U_site = copy_out(m.U);
    q->omega = copy_out(m.omega);
    q->Ev = copy_out(m.Ev);
    std::snprintf(q->model_name, sizeof q->model_name, "%s", m.model.c_str());
    *out = q;
    return 0;
}

void qsah_free(qsah_model *m) {
    if (!m) return;
    for (void *p : {(void *)m->H, (void *)m->GammaL, (void *)m->GammaR, (void *)m->U_site, (void *)m->omega,
                    (void *)m->Ev})
        std::free(p);
    std::free(m);
}

int qsah_run(const char *dir, const qsah_solver_api *api, int device, FILE *log) {
    auto t0 = std::chrono::steady_clock::now();
    std::string d = dir ? dir : ".";
    auto P = [&](const char *f) { return d + "/" + f; };
    char err[4096] = {0};
    qsah_model *m = nullptr;
    if (qsah_load(d.c_str(), &m, err, sizeof err, log) != 0) {
        std::fprintf(stderr, "%s\n", err);
        return 1;
    }
    const int n = m->N_sites;
    // info_Hamiltonian.dat: H and its eigenvalues (write_hamiltonian_info, src/input_output.f90:151-183)
    if (FILE *u = std::fopen(P("info_Hamiltonian.dat").c_str(), "w")) {
        std::fprintf(u, "\n... Hamiltonian:\n");
        for (int i = 0; i < n; i++) {
            for (int j = 0; j < std::min(n, 10); j++)
                std::fprintf(u, " [%10.5f%10.5f] ", m->H[2 * (i + (size_t)j * n)], m->H[2 * (i + (size_t)j * n) + 1]);
            std::fprintf(u, "\n");
        }
        std::fprintf(u, "\n... Eigenvalues:\n");
        char b[64], c[64];
        for (int i = 0; i < n; i++) {
            qsh_fmt_int(i + 1, b);
            qsh_fmt_real(m->Ev[i], c);
            std::fprintf(u, "%s .%s\n", b, c);
        }
        std::fclose(u);
    }
    if (log) std::fprintf(log, " n_omega: %d  w_fin: %.10f  w_init: %.10f  solver: %s\n", m->n_omega, m->w_fin,
                          m->w_init, api->name);
    qsa_problem p{};
    p.N_sites = n;
    p.order = m->order;
    p.n_omega = m->n_omega;
    p.H = m->H;
    p.GammaL = m->GammaL;
    p.GammaR = m->GammaR;
    p.U_site = m->U_site;
    p.omega = m->omega;
    p.mu = m->mu;
    p.beta = m->beta;
    p.delta = m->delta;
    p.alpha_mix = m->alpha_mix;
    p.tolf = m->tolf;
    p.nhist = m->nhist;
    p.maxscf = m->maxscf;
    p.device = device;
    void *h = nullptr;
    int rc = api->create(&p, &h);
    if (rc != 0) {
        std::fprintf(stderr, "ERROR: solver set-up failed (%d): %s\n", rc, h ? api->last_error(h) : "");
        if (h) api->destroy(h);
        qsah_free(m);
        return 2;
    }
    char name[64];
    std::snprintf(name, sizeof name, "Volt_Current_%d.dat", m->order);
    FILE *u_iv = std::fopen(P(name).c_str(), "w");
    FILE *u_pop = std::fopen(P("populations.dat").c_str(), "w");
    FILE *u_spec = std::fopen(P("spectral_function.dat").c_str(), "w");
    FILE *u_rt = std::fopen(P("runtime_datasheet.dat").c_str(), "w");
    if (u_rt) std::fprintf(u_rt, " >>>>>>>>>>>>>>>>>>>>>>>>>>>>Runtime Data Sheet>>>>>>>>>>>>>>>>>>>>>>>>>>>>\n SANCHO on B200, solver: %s\n", api->name);
    std::vector<qs_scf_step> steps(std::max(m->maxscf, 1) + 1);
    std::vector<double> glt((size_t)2 * n), spec((size_t)n * m->n_omega);
    bool fresh = true;
    int n_unconv = 0, status = 0;
    char b[64];
    for (int k = 0; k <= m->n_volt_steps; k++) {
        const double V1 = m->V + k * m->delv;
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
                std::fprintf(log, " CONVERGED TO AN UNPHYSICAL SOLUTION: site %4d n = %11.3E, spectral weight = %11.3E\n",
                             res.i_worst, res.n_worst, res.w_worst);
            else
                std::fprintf(log, " V = %9.4f ... CONVERGED in %5d steps ... (%.3f s)\n", V1, res.n_iter, res.seconds);
        }
        if (!res.converged) n_unconv++;
        fresh = (!m->continuation) || (!res.converged);
        double J = 0;
        api->current(h, V1, &J);
        std::string s;
        // Volt_Current_<order>.dat: V, J, converged (src/sancho.f90:129)
        s += std::string(b, qsh_fmt_real(V1, b));
        s += std::string(b, qsh_fmt_real(J, b));
        s += std::string(b, qsh_fmt_int(res.converged ? 1 : 0, b));
        std::fprintf(u_iv, "%s\n", s.c_str());
        std::fflush(u_iv);
        api->get_observables(h, glt.data(), spec.data());
        // populations.dat: V, site, n per spin, n total (src/observables.f90:54-67)
        for (int i = 0; i < n; i++) {
            const double ni = glt[2 * i + 1];  // Re(-i hbar G^<_ii(t=0)) = Im G^<_ii(t=0)
            std::string r;
            r += std::string(b, qsh_fmt_real(V1, b));
            r += std::string(b, qsh_fmt_int(i + 1, b));
            r += std::string(b, qsh_fmt_real(ni, b));
            r += std::string(b, qsh_fmt_real(2.0 * ni, b));
            std::fprintf(u_pop, "%s\n", r.c_str());
        }
        std::fflush(u_pop);
        // spectral_function.dat (src/observables.f90:69-82)
        std::fprintf(u_spec, "# V = %10.5f   columns: V, omega, A_ii for i = 1..Nsites\n", V1);
        for (int iw = 0; iw < m->n_omega; iw++) {
            std::string r;
            r += std::string(b, qsh_fmt_real(V1, b));
            r += std::string(b, qsh_fmt_real(m->omega[iw], b));
            for (int i = 0; i < n; i++) r += std::string(b, qsh_fmt_real(spec[i + (size_t)iw * n], b));
            std::fprintf(u_spec, "%s\n", r.c_str());
        }
        std::fputs("\n\n", u_spec);
        std::fflush(u_spec);
    }
    std::fclose(u_iv);
    std::fclose(u_pop);
    std::fclose(u_spec);
    const double mins = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() / 60.0;
    if (u_rt) {
        std::fprintf(u_rt, " <<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<<\n Total Runtime: %.8f mins\n", mins);
        std::fclose(u_rt);
    }
    api->destroy(h);
    qsah_free(m);
    if (status) return status;
    if (n_unconv > 0) {
        if (log) std::fprintf(log, " WARNING: %d voltage(s) did not converge (column 3 = 0 in Volt_Current)\n", n_unconv);
        return 3;
    }
    return 0;
}

}  // extern "C"
