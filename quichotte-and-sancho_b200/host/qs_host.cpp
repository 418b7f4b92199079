// qs_host.cpp -- host layer of QUICHOTTE on B200: input.dat reader, model builders,
// energy grid and the reference's output files.
//
// Restates (the reference keeps these on the host as well; none is on the NEGF hot path):
//   common/input_parser.f90:49-249     key = value reader (aliases, duplicates, unknown keys)
//   src/input_output.f90:31-462        read_input, set_number_of_sites, setup_dftb_elements,
//                                      set_atom_map, setup_leads, check_input, setup_hubbard
//   src/hamiltonian.f90:44-755         helix, peptide, xyz, dftb, dftb_hs and custom models
//   src/quichotte.f90:241-253          energy grid from the spectrum of H
//   src/observables.f90:41-158         spin_texture, write_spectral, atom_texture (file output)
// The eigenproblems of the set-up (zheev for the grid, dsyev for the Loewdin S^-1/2 of
// dftb_hs) use a cyclic Jacobi method (jacobi_herm below): this code has no LAPACK.
#include "qs_host.h"

#include <algorithm>
#include <cctype>
#include <charconv>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "host_common.hpp"

namespace {

// ---------------------------------------------------------------------------------
// Model (module globals of Parameters / Hamiltonian / GreenFunctions / InputOutput)
// ---------------------------------------------------------------------------------
struct Model {
    std::string dir;
    FILE *log = nullptr;
    const qsh_solver_api *api = nullptr;  // its set-up linear algebra, where it has some
    int device = 0;
    // Parameters
    int N_sites = 0, Norb = 0, n_omega = 0, n_volt_steps = 0, N_ions = 0, N_turns = 0, order = 0;
    std::string hamiltonian_model = "helix", xyz_file = "molecule.xyz",
                ham_file = "hamiltonian_blocks_fortran.txt", overlap_file = "oversqr.dat";
    bool write_hamiltonian = false;
    std::string soc_form = "dual";
    std::vector<std::string> atom_elem, elem_name;
    std::vector<int> elem_lmax;
    std::vector<double> elem_xi;
    int N_atoms = 0;
    std::vector<int> atom_norb, atom_first, orb_atom;
    double V = 0, Vf = 0, delv = 0, T = 0, mu = 0, beta = 0;
    double delta = 0, w_init = 0, w_fin = 0, dw = 0, up = 0;
    double E_CC = 0, t_hop = 0, lamb = 0, U_int = 0, hel_radius = 0, hel_length = 0, hand = 1;
    double pep_twist = 100, pep_rise = 1.5, hop_decay = 1, dipole_ramp = 0;
    int hop_range = 1;
    std::string soc_model = "radial";
    double GammaL_up = 0, GammaL_down = 0, GammaR_both = 0;
    // SCF settings
    double alpha_mix = 0.5, tolf = 1e-6, tolf_order1 = 1e-8;
    int nhist = 16, maxscf = 300;
    bool continuation = true, broyden_single_precision = true;
    // InputOutput
    std::string hubbard_file, lead_left_atoms, lead_right_atoms, max_l_string, soc_xi_string;
    // arrays
    std::vector<cplx> H, GammaL, GammaR;
    std::vector<double> U_site, omega, Ev;

    cplx &h(int i, int j) { return H[(i - 1) + (size_t)(j - 1) * Norb]; }  // 1-based
    std::string path(const std::string &f) const {
        if (!f.empty() && f[0] == '/') return f;
        return dir + "/" + f;
    }
    [[noreturn]] void fail(const std::string &m) { throw InputError(m); }
    void say(const char *fmt, ...) {
        if (!log) return;
        va_list ap;
        va_start(ap, fmt);
        std::vfprintf(log, fmt, ap);
        va_end(ap);
    }

    // ----- src/input_output.f90:31-139 read_input
    void read_input() {
        InputParser ip;
        ip.log = log;
        ip.load(dir, {"input.dat", "inputSOC.dat"});
        input_file = ip.file_name;
        const double d0 = 0.0, d1 = 1.0;
        ip.get("V", V);
        ip.get("Vf", Vf);
        ip.get("delv", delv);
        ip.get("T", T);
        ip.get("mu", mu);
        ip.get("hamiltonian", hamiltonian_model, "helix");
        ip.get("xyz_file", xyz_file, "molecule.xyz");
        if (hamiltonian_model == "dftb_hs") {
            ip.get("ham_file", ham_file, "hamsqr1.dat");
            ip.get("overlap_file", overlap_file, "oversqr.dat");
            ip.get("max_angular_momentum", max_l_string);
        } else {
            ip.get("ham_file", ham_file, "hamiltonian_blocks_fortran.txt");
            ip.get("overlap_file", overlap_file, "oversqr.dat");
            ip.get("max_angular_momentum", max_l_string, "");
        }
        ip.get("soc_xi", soc_xi_string, "");
        ip.get("soc_form", soc_form, "dual");
        const bool bf = false, bt = true;
        ip.get("write_hamiltonian", write_hamiltonian, &bf);
        const int i0 = 0, i1 = 1, i16 = 16, i300 = 300;
        ip.get("N_sites", N_sites, &i0);
        if (hamiltonian_model == "helix") {
            ip.get("N_ions", N_ions);
            ip.get("N_turns", N_turns);
            ip.get("hel_length", hel_length);
            ip.get("hel_radius", hel_radius);
            ip.get("hand", hand);
        } else {
            ip.get("N_ions", N_ions, &i0);
            ip.get("N_turns", N_turns, &i0);
            ip.get("hel_length", hel_length, &d0);
            ip.get("hel_radius", hel_radius, &d0);
            ip.get("hand", hand, &d1);
        }
        const double d100 = 100.0, d15 = 1.5;
        ip.get("pep_twist", pep_twist, &d100);
        ip.get("pep_rise", pep_rise, &d15);
        ip.get("hop_range", hop_range, &i1);
        ip.get("hop_decay", hop_decay, &d1);
        ip.get("soc_model", soc_model, "radial");
        ip.get("dipole_ramp", dipole_ramp, &d0);
        if (hamiltonian_model == "dftb" || hamiltonian_model == "dftb_hs") {
            ip.get("E_CC", E_CC, &d0);
            ip.get("t_hop", t_hop, &d0);
        } else {
            ip.get("E_CC", E_CC);
            ip.get("t_hop", t_hop);
        }
        if (hamiltonian_model == "helix" || hamiltonian_model == "xyz" || hamiltonian_model == "peptide")
            ip.get("lamb", lamb);
        else
            ip.get("lamb", lamb, &d0);
        ip.get("U_int", U_int, nullptr, "Hubbard");
        ip.get("hubbard_file", hubbard_file, "");
        ip.get("order", order);
        ip.get("GammaL_up", GammaL_up);
        ip.get("GammaL_down", GammaL_down);
        ip.get("GammaR", GammaR_both, nullptr, "GammaR_both");
        ip.get("lead_left_atoms", lead_left_atoms, "");
        ip.get("lead_right_atoms", lead_right_atoms, "");
        ip.get("dw", dw);
        ip.get("up", up);
        ip.get("delta", delta);
        const double d05 = 0.5, d1m6 = 1e-6, d1m8 = 1e-8;
        ip.get("alpha_mix", alpha_mix, &d05, "pulay");
        ip.get("nhist", nhist, &i16);
        ip.get("maxscf", maxscf, &i300);
        ip.get("tolf", tolf, &d1m6);
        ip.get("tolf_order1", tolf_order1, &d1m8);
        ip.get("broyden_single_precision", broyden_single_precision, &bt);
        ip.get("continuation", continuation, &bt);
        bool restart_unused = false;
        ip.get("restart", restart_unused, &bf);
        ip.finish();

        set_number_of_sites();
        beta = 1.0 / (kB * T);
        Norb = 2 * N_sites;
        set_atom_map();
        n_volt_steps = (int)std::lround((Vf - V) / delv);  // Fortran nint
        check_input();
    }
    std::string input_file;

    // ----- src/input_output.f90:141-182
    void set_number_of_sites() {
        int n_model = 0;
        if (hamiltonian_model == "helix") {
            n_model = N_ions * N_turns;
        } else if (hamiltonian_model == "xyz") {
            n_model = xyz_site_count(xyz_file);
        } else if (hamiltonian_model == "dftb") {
            std::vector<int> norb;
            int n_at = 0;
            dftb_blocks_scan(ham_file, n_at, norb);
            n_model = 0;
            for (int v : norb) n_model += v;
            N_atoms = n_at;
            atom_norb = norb;
        } else if (hamiltonian_model == "dftb_hs") {
            setup_dftb_elements();
            n_model = 0;
            for (int v : atom_norb) n_model += v;
        } else {
            if (N_sites < 1)
                fail(" ERROR: hamiltonian = " + hamiltonian_model +
                     " needs the key N_sites\n       (built-in models: helix, xyz, custom)");
            return;
        }
        if (N_sites > 0 && N_sites != n_model)
            fail(" ERROR: N_sites = " + std::to_string(N_sites) + " but the " + hamiltonian_model +
                 " model has " + std::to_string(n_model));
        N_sites = n_model;
    }

    static std::string element_case(const std::string &e0) {
        std::string e = trim(e0);
        e = e.substr(0, std::min<size_t>(2, e.size()));
        if (e.size() >= 1 && e[0] >= 'a' && e[0] <= 'z') e[0] = (char)(e[0] - 32);
        if (e.size() >= 2 && e[1] >= 'A' && e[1] <= 'Z') e[1] = (char)(e[1] + 32);
        return e;
    }

    void split_pairs(const std::string &str, const std::string &key, std::vector<std::string> &names,
                     std::vector<std::string> &vals) {
        std::string s = str;
        for (char &c : s)
            if (c == ',') c = ' ';
        std::stringstream ss(s);
        std::string tok;
        std::vector<std::string> toks;
        while (ss >> tok)
            if (toks.size() < 100) toks.push_back(tok);
        if (toks.empty()) fail(" ERROR: " + key + " is empty");
        names.clear();
        vals.clear();
        for (auto &t : toks) {
            size_t c = t.find(':');
            if (c == std::string::npos || c < 1)
                fail(" ERROR: " + key + ": entries must look like Element:value, got \"" + t + "\"");
            names.push_back(t.substr(0, std::min<size_t>(c, 8)));
            vals.push_back(t.substr(c + 1));
        }
    }

    // ----- src/input_output.f90:184-237
    void setup_dftb_elements() {
        read_xyz_elements(xyz_file, N_atoms, atom_elem);
        for (auto &e : atom_elem) e = element_case(e);
        std::vector<std::string> names, vals;
        split_pairs(max_l_string, "max_angular_momentum", names, vals);
        elem_name.clear();
        elem_lmax.clear();
        elem_xi.assign(names.size(), 0.0);
        for (size_t e = 0; e < names.size(); e++) {
            elem_name.push_back(element_case(names[e]));
            std::string v = trim(vals[e]);
            if (v == "s" || v == "S") elem_lmax.push_back(0);
            else if (v == "p" || v == "P") elem_lmax.push_back(1);
            else
                fail(" ERROR: max_angular_momentum: only s and p shells are supported, not \"" + v + "\" for " +
                     names[e]);
        }
        if (!trim(soc_xi_string).empty()) {
            split_pairs(soc_xi_string, "soc_xi", names, vals);
            for (size_t k = 0; k < names.size(); k++) {
                auto it = std::find(elem_name.begin(), elem_name.end(), element_case(names[k]));
                double xv;
                bool ok = read_real(vals[k], xv);
                if (it == elem_name.end() || !ok)
                    fail(" ERROR: soc_xi: bad entry " + names[k] + ":" + vals[k] +
                         " (element must also appear in max_angular_momentum)");
                elem_xi[it - elem_name.begin()] = xv;
            }
        }
        atom_norb.assign(N_atoms, 0);
        for (int a = 0; a < N_atoms; a++) {
            auto it = std::find(elem_name.begin(), elem_name.end(), atom_elem[a]);
            if (it == elem_name.end())
                fail(" ERROR: element " + atom_elem[a] + " of " + xyz_file + " is missing from max_angular_momentum");
            atom_norb[a] = (elem_lmax[it - elem_name.begin()] == 1) ? 4 : 1;
        }
    }

    // ----- src/input_output.f90:292-308
    void set_atom_map() {
        if (atom_norb.empty()) {
            N_atoms = N_sites;
            atom_norb.assign(N_atoms, 1);
        }
        atom_first.assign(N_atoms, 0);
        orb_atom.assign(N_sites, 0);
        int i = 0;
        for (int a = 0; a < N_atoms; a++) {
            atom_first[a] = i + 1;
            for (int k = 0; k < atom_norb[a] && i + k < N_sites; k++) orb_atom[i + k] = a + 1;
            i += atom_norb[a];
        }
    }

    // ----- src/input_output.f90:348-394
    std::vector<int> parse_atom_list(const std::string &str, int default_atom, const std::string &key) {
        std::string s = str;
        for (char &c : s)
            if (c == ',') c = ' ';
        std::stringstream ss(s);
        std::string tok;
        std::vector<int> list;
        while (ss >> tok) {
            size_t k = tok.find(':');
            double a = 0, b = 0;
            bool ok;
            if (k != std::string::npos) {
                ok = read_real(tok.substr(0, k), a) && read_real(tok.substr(k + 1), b);
            } else {
                ok = read_real(tok, a);
                b = a;
            }
            bool integral = ok && a == std::floor(a) && b == std::floor(b);
            if (!integral || a < 1 || b > N_atoms || b < a)
                fail(" ERROR: " + key + ": bad atom or range \"" + tok + "\" (atoms are 1.." +
                     std::to_string(N_atoms) + ")");
            for (int q = (int)a; q <= (int)b; q++)
                if (list.size() < 10000) list.push_back(q);
        }
        if (list.empty()) list.push_back(default_atom);
        return list;
    }

    // ----- src/input_output.f90:310-346
    void setup_leads() {
        auto left = parse_atom_list(lead_left_atoms, 1, "lead_left_atoms");
        auto right = parse_atom_list(lead_right_atoms, N_atoms, "lead_right_atoms");
        for (int a : left)
            if (std::find(right.begin(), right.end(), a) != right.end())
                fail(" ERROR: atom " + std::to_string(a) + " is in both lead_left_atoms and lead_right_atoms");
        GammaL.assign((size_t)Norb * Norb, 0.0);
        GammaR.assign((size_t)Norb * Norb, 0.0);
        auto g = [&](std::vector<cplx> &G, int i, int j) -> cplx & { return G[(i - 1) + (size_t)(j - 1) * Norb]; };
        for (int a : left)
            for (int i = atom_first[a - 1]; i <= atom_first[a - 1] + atom_norb[a - 1] - 1; i++) {
                g(GammaL, 2 * i - 1, 2 * i - 1) = GammaL_up;
                g(GammaL, 2 * i, 2 * i) = GammaL_down;
            }
        for (int a : right)
            for (int i = atom_first[a - 1]; i <= atom_first[a - 1] + atom_norb[a - 1] - 1; i++) {
                g(GammaR, 2 * i - 1, 2 * i - 1) = GammaR_both;
                g(GammaR, 2 * i, 2 * i) = GammaR_both;
            }
    }

    // ----- src/input_output.f90:396-430
    void check_input() {
        std::string m;
        auto complain = [&](const std::string &msg) { m += " ERROR in input: " + msg + "\n"; };
        if (hamiltonian_model == "helix" && (N_ions < 2 || N_turns < 1)) complain("need N_ions >= 2 and N_turns >= 1");
        if (N_sites < 1) complain("need at least one site");
        if (hamiltonian_model == "peptide") {
            if (N_sites < 2) complain("peptide: need N_sites >= 2");
            if (hel_radius <= 0.0) complain("peptide: hel_radius must be > 0 (alpha-helix: 2.5)");
            if (std::fabs(std::fabs(hand) - 1.0) > 1e-12) complain("peptide: hand must be +1 or -1");
            if (hop_range < 1) complain("peptide: hop_range must be >= 1");
            if (hop_decay <= 0.0) complain("peptide: hop_decay must be > 0");
            if (soc_model != "radial" && soc_model != "torsion") complain("peptide: soc_model must be radial or torsion");
        }
        if (order < 0 || order > 2) complain("order must be 0, 1 or 2");
        if (delta <= 0.0) complain("delta (energy grid step) must be > 0");
        if (delv <= 0.0) complain("delv (voltage step) must be > 0");
        if (Vf < V) complain("Vf must be >= V");
        if (T <= 0.0) complain("T must be > 0");
        if (nhist < 0) complain("nhist must be >= 0");
        if (maxscf < 1) complain("maxscf must be >= 1");
        if (tolf <= 0.0) complain("tolf must be > 0");
        if (tolf_order1 <= 0.0) complain("tolf_order1 must be > 0");
        if (!m.empty()) fail(m);
    }

    // ----- src/input_output.f90:432-462
    void setup_hubbard() {
        U_site.assign(Norb, 0.0);
        if (trim(hubbard_file).empty()) {
            for (int i = 0; i < Norb; i += 2) U_site[i] = U_int;
            return;
        }
        std::ifstream f(path(trim(hubbard_file)));
        if (!f.good()) fail(" ERROR: cannot open hubbard_file " + trim(hubbard_file));
        std::string line;
        for (int i = 0; i < Norb; i += 2) {
            bool got = false;
            while (std::getline(f, line)) {  // one list-directed read: the first item found
                if (first_item(line).empty()) continue;
                got = read_real(line, U_site[i]);
                break;
            }
            if (!got)
                fail(" ERROR: " + trim(hubbard_file) + " needs one U per site/orbital (" + std::to_string(Norb / 2) +
                     " lines)");
        }
        say(" Site-dependent U read from %s\n", trim(hubbard_file).c_str());
    }

    // ----- src/hamiltonian.f90 readers
    int xyz_site_count(const std::string &fname) {
        std::ifstream f(path(trim(fname)));
        if (!f.good()) fail(" ERROR: cannot open xyz_file " + trim(fname));
        std::string line;
        double n = 0;
        bool ok = false;
        while (std::getline(f, line))
            if (!first_item(line).empty()) { ok = read_real(line, n); break; }
        if (!ok || n < 1 || n != std::floor(n)) fail(" ERROR: first line of " + trim(fname) + " must be the number of atoms");
        return (int)n;
    }

    void read_xyz_elements(const std::string &fname, int &n_at, std::vector<std::string> &elem) {
        std::ifstream f(path(trim(fname)));
        if (!f.good()) fail(" ERROR: cannot open xyz_file " + trim(fname));
        std::string line;
        double n = 0;
        if (!std::getline(f, line) || !read_real(line, n) || n < 1)
            fail(" ERROR: first line of " + trim(fname) + " must be the number of atoms");
        n_at = (int)n;
        std::getline(f, line);  // comment
        elem.clear();
        for (int a = 0; a < n_at; a++) {
            std::string tok;
            while (std::getline(f, line)) {
                tok = first_item(line);
                if (!tok.empty()) break;
            }
            if (tok.empty()) fail(" ERROR: " + trim(fname) + " has fewer than " + std::to_string(n_at) + " atom lines");
            elem.push_back(tok.substr(0, 2));
        }
    }

    static bool parse_block_header(const std::string &line, int &ai, int &aj, int &di, int &dj) {
        ai = aj = di = dj = 0;
        size_t k1 = line.find("Atom_I:"), k2 = line.find("Atom_J:"), k3 = line.find("Dim:");
        if (k1 == std::string::npos || k2 == std::string::npos || k3 == std::string::npos) return false;
        double v;
        if (!read_real(line.substr(k1 + 7), v)) return false;
        ai = (int)v;
        if (!read_real(line.substr(k2 + 7), v)) return false;
        aj = (int)v;
        size_t kx = line.find('x', k3);
        if (kx == std::string::npos) return false;
        if (!read_real(line.substr(k3 + 4, kx - (k3 + 4)), v)) return false;
        di = (int)v;
        if (!read_real(line.substr(kx + 1), v)) return false;
        dj = (int)v;
        return ai >= 1 && aj >= 1 && di >= 1 && dj >= 1;
    }

    void dftb_blocks_scan(const std::string &fname, int &n_at, std::vector<int> &norb) {
        n_at = 0;
        for (int pass = 1; pass <= 2; pass++) {
            std::ifstream f(path(trim(fname)));
            if (!f.good()) fail(" ERROR: cannot open ham_file " + trim(fname));
            if (pass == 2) norb.assign(n_at, 0);
            std::string line;
            while (std::getline(f, line)) {
                if (trim(line).rfind("BLOCK", 0) != 0) continue;
                int ai, aj, di, dj;
                if (!parse_block_header(line, ai, aj, di, dj))
                    fail(" ERROR: cannot read block header in " + trim(fname) + ": " + trim(line));
                if (di % 2 || dj % 2)
                    fail(" ERROR: block dimensions must be even (orbitals x 2 spins): " + trim(line));
                if (pass == 1) {
                    n_at = std::max({n_at, ai, aj});
                } else {
                    auto set = [&](int a, int n) {
                        if (norb[a - 1] != 0 && norb[a - 1] != n)
                            fail(" ERROR: atom " + std::to_string(a) + " has inconsistent block dimensions in " + trim(fname));
                        norb[a - 1] = n;
                    };
                    set(ai, di / 2);
                    set(aj, dj / 2);
                }
            }
        }
        bool bad = n_at < 1;
        for (int v : norb) bad = bad || v == 0;
        if (bad) fail(" ERROR: " + trim(fname) + " has no BLOCK for some atom (every atom needs its on-site block)");
    }

    // ----- src/hamiltonian.f90:44-63 dispatcher
    void build_hamiltonian() {
        H.assign((size_t)Norb * Norb, 0.0);
        if (hamiltonian_model == "helix") build_helix();
        else if (hamiltonian_model == "peptide") build_peptide();
        else if (hamiltonian_model == "xyz") build_from_xyz(trim(xyz_file));
        else if (hamiltonian_model == "dftb") build_from_dftb(trim(ham_file));
        else if (hamiltonian_model == "dftb_hs") build_from_dftb_hs();
        else if (hamiltonian_model == "custom") build_custom();
        else
            fail(" ERROR: unknown hamiltonian = " + hamiltonian_model +
                 "\n        built in: helix, peptide, xyz, dftb, dftb_hs, custom (see src/hamiltonian.f90)");
    }

    void helix_coordinate(double r[3], int i) const {
        r[0] = hel_radius * std::cos(hand * (i - 1) * 2 * PI / N_ions);
        r[1] = hel_radius * std::sin(hand * (i - 1) * 2 * PI / N_ions);
        r[2] = hel_length * (i - 1) / (N_turns * (N_ions - 1));
    }
    static void cross(const double a[3], const double b[3], double c[3]) {
        c[0] = a[1] * b[2] - a[2] * b[1];
        c[1] = a[2] * b[0] - a[0] * b[2];
        c[2] = a[0] * b[1] - b[0] * a[1];
    }
    static double norm3(const double r[3]) { return std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]); }

    // src/hamiltonian.f90:99-115
    void soc_matrix_elements(const double r[3], const double r1[3], const double r2[3], int ii, int jj) {
        double d1[3], d2[3], v[3], t1[3], t2[3];
        for (int k = 0; k < 3; k++) { t1[k] = r[k] - r1[k]; t2[k] = r[k] - r2[k]; }
        double n1 = norm3(t1), n2 = norm3(t2);
        for (int k = 0; k < 3; k++) { d1[k] = t1[k] / n1; d2[k] = t2[k] / n2; }
        cross(d1, d2, v);
        h(ii - 1, jj - 1) = IM * lamb * v[2];
        h(ii - 1, jj) = IM * lamb * (v[0] - IM * v[1]);
        h(ii, jj - 1) = IM * lamb * (v[0] + IM * v[1]);
        h(ii, jj) = IM * lamb * (-v[2]);
    }
    void make_hermitian() {
        for (int i = 1; i <= Norb; i++)
            for (int j = i; j <= Norb; j++) h(j, i) = std::conj(h(i, j));
    }

    // src/hamiltonian.f90:129-163
    void build_helix() {
        int Nat = Norb / 2;
        for (int i = 1; i <= Nat; i++) {
            int ii = 2 * i;
            h(ii - 1, ii - 1) = E_CC;
            h(ii, ii) = E_CC;
            if (i <= Nat - 1) {
                int jj = 2 * (i + 1);
                h(ii - 1, jj - 1) = t_hop;
                h(ii, jj) = t_hop;
            }
            if (i <= Nat - 2) {
                int jj = 2 * (i + 2);
                double r[3], r1[3], r2[3];
                helix_coordinate(r, i);
                helix_coordinate(r1, i + 1);
                helix_coordinate(r2, i + 2);
                soc_matrix_elements(r, r1, r2, ii, jj);
            }
        }
        make_hermitian();
    }

    // src/hamiltonian.f90:195-273
    void build_peptide() {
        int Nat = Norb / 2;
        int jmax = std::min(hop_range, Nat - 1);
        double dphi = hand * pep_twist * PI / 180.0;
        std::vector<double> rs(3 * (size_t)Nat), phi(Nat);
        for (int i = 1; i <= Nat; i++) {
            phi[i - 1] = i * dphi;
            rs[3 * (i - 1) + 0] = hel_radius * std::cos(phi[i - 1]);
            rs[3 * (i - 1) + 1] = hel_radius * std::sin(phi[i - 1]);
            rs[3 * (i - 1) + 2] = (i - 1) * pep_rise;
        }
        double d12[3] = {rs[3] - rs[0], rs[4] - rs[1], rs[5] - rs[2]};
        double l1 = norm3(d12);
        for (int i = 1; i <= Nat; i++) {
            int ii = 2 * i;
            h(ii - 1, ii - 1) = E_CC + dipole_ramp * ((double)(i - 1) / (double)(Nat - 1) - 0.5);
            h(ii, ii) = h(ii - 1, ii - 1);
        }
        if (soc_model == "torsion")
            for (int i = 1; i <= Nat - 2; i++)
                soc_matrix_elements(&rs[3 * (i - 1)], &rs[3 * i], &rs[3 * (i + 1)], 2 * i, 2 * (i + 2));
        for (int j = 1; j <= jmax; j++)
            for (int i = 1; i <= Nat - j; i++) {
                int m = i + j, ii = 2 * i, jj = 2 * m;
                double d[3], dhat[3], rhat[3], nu[3];
                for (int k = 0; k < 3; k++) d[k] = rs[3 * (m - 1) + k] - rs[3 * (i - 1) + k];
                double l = norm3(d);
                for (int k = 0; k < 3; k++) dhat[k] = d[k] / l;
                double fac = std::exp(-(l - l1) / hop_decay);
                h(ii - 1, jj - 1) += t_hop * fac;
                h(ii, jj) += t_hop * fac;
                if (soc_model == "radial") {
                    double phibar = 0.5 * (phi[i - 1] + phi[m - 1]);
                    rhat[0] = std::cos(phibar);
                    rhat[1] = std::sin(phibar);
                    rhat[2] = 0.0;
                    cross(rhat, dhat, nu);
                    double lj = 2.0 * lamb * fac * std::cos(0.5 * (phi[m - 1] - phi[i - 1]));
                    h(ii - 1, jj - 1) += IM * lj * nu[2];
                    h(ii - 1, jj) += IM * lj * (nu[0] - IM * nu[1]);
                    h(ii, jj - 1) += IM * lj * (nu[0] + IM * nu[1]);
                    h(ii, jj) -= IM * lj * nu[2];
                }
            }
        make_hermitian();
        FILE *u = std::fopen(path("peptide_geometry.xyz").c_str(), "w");
        if (u) {
            std::fprintf(u, "%d\nQUICHOTTE peptide sites [Angstrom]\n", Nat);
            for (int i = 0; i < Nat; i++)
                std::fprintf(u, "C %14.8f%14.8f%14.8f\n", rs[3 * i], rs[3 * i + 1], rs[3 * i + 2]);
            std::fclose(u);
        }
    }

    // src/hamiltonian.f90:275-326
    void build_from_xyz(const std::string &fname) {
        std::ifstream f(path(fname));
        if (!f.good()) fail(" ERROR: cannot open XYZ file: " + fname);
        std::string line;
        std::getline(f, line);
        double nd = 0;
        read_real(line, nd);
        int Nat = (int)nd;
        if (2 * Nat != Norb)
            fail(" ERROR: " + fname + " has " + std::to_string(Nat) + " atoms but the input gives " +
                 std::to_string(Norb / 2) + " sites");
        std::getline(f, line);
        std::vector<double> c(3 * (size_t)Nat);
        for (int i = 0; i < Nat; i++) {
            if (!std::getline(f, line)) fail(" ERROR: " + fname + ": too few atom lines");
            std::stringstream ss(line);
            std::string at, x, y, z;
            ss >> at >> x >> y >> z;
            read_real(x, c[3 * i]);
            read_real(y, c[3 * i + 1]);
            read_real(z, c[3 * i + 2]);
        }
        for (int i = 1; i <= Nat; i++) {
            int ii = 2 * i;
            h(ii - 1, ii - 1) = E_CC;
            h(ii, ii) = E_CC;
            if (i <= Nat - 1) {
                int jj = 2 * (i + 1);
                h(ii - 1, jj - 1) = t_hop;
                h(ii, jj) = t_hop;
            }
            if (i <= Nat - 2)
                soc_matrix_elements(&c[3 * (i - 1)], &c[3 * i], &c[3 * (i + 1)], ii, 2 * (i + 2));
        }
        make_hermitian();
    }

    // src/hamiltonian.f90:407-475
    void build_from_dftb(const std::string &fname) {
        std::vector<bool> onsite(N_atoms, false);
        std::ifstream f(path(fname));
        if (!f.good()) fail(" ERROR: cannot open ham_file " + fname);
        std::string line;
        int nblk = 0;
        while (std::getline(f, line)) {
            if (trim(line).rfind("BLOCK", 0) != 0) continue;
            int ai, aj, di, dj;
            bool ok = parse_block_header(line, ai, aj, di, dj);
            if (!ok || ai > N_atoms || aj > N_atoms || di != 2 * atom_norb[ai - 1] || dj != 2 * atom_norb[aj - 1])
                fail(" ERROR: bad block header in " + fname + ": " + trim(line));
            int r0 = 2 * (atom_first[ai - 1] - 1), c0 = 2 * (atom_first[aj - 1] - 1);
            for (int r = 1; r <= di; r++)
                for (int c = 1; c <= dj; c++) {
                    std::string l2;
                    double re = 0, im = 0;
                    bool got = false;
                    while (std::getline(f, l2)) {
                        std::stringstream ss(l2);
                        std::string a, b;
                        if (!(ss >> a)) continue;
                        ss >> b;
                        got = read_real(a, re) && read_real(b, im);
                        break;
                    }
                    if (!got) fail(" ERROR: block too short in " + fname + ": " + trim(line));
                    h(r0 + r, c0 + c) = cplx(re, im);
                }
            if (ai == aj) onsite[ai - 1] = true;
            nblk++;
        }
        for (bool b : onsite)
            if (!b) fail(" ERROR: " + fname + " is missing the on-site block of some atom");
        std::vector<cplx> Hh(H.size());
        for (int j = 1; j <= Norb; j++)
            for (int i = 1; i <= Norb; i++) Hh[(i - 1) + (size_t)(j - 1) * Norb] = 0.5 * (h(i, j) + std::conj(h(j, i)));
        H.swap(Hh);
        say(" DFTB Hamiltonian: %d blocks, %d atoms, %d orbitals\n", nblk, N_atoms, N_sites);
    }

    // DFTB+ square matrix file (src/hamiltonian.f90:559-604)
    void read_dftb_square(const std::string &fname, int n, std::vector<double> &A) {
        std::ifstream f(path(trim(fname)));
        if (!f.good()) fail(" ERROR: cannot open " + trim(fname));
        std::string line;
        auto next_data = [&](std::string &l) {
            while (std::getline(f, l)) {
                std::string t = trim(l);
                if (!t.empty() && t[0] != '#') return;
            }
            fail(" ERROR: unexpected end of " + trim(fname));
        };
        next_data(line);
        {
            std::stringstream ss(line);
            std::string flag, a, b;
            ss >> flag >> a >> b;
            double nall = -1, nk = -1;
            if (!read_real(a, nall) || !read_real(b, nk) || (int)nall != n)
                fail(" ERROR: " + trim(fname) + " has " + a + " orbitals; the geometry and shells give " + std::to_string(n));
            if ((int)nk != 1) fail(" ERROR: " + trim(fname) + ": only one k-point (a molecule) is supported");
        }
        next_data(line);  // k-point index
        A.assign((size_t)n * n, 0.0);
        std::vector<double> vals;
        std::string tok;
        for (int i = 0; i < n; i++) {
            // one list-directed read of n values: as many records as needed
            vals.clear();
            while ((int)vals.size() < n) {
                if (!std::getline(f, line)) fail(" ERROR: " + trim(fname) + ": cannot read row " + std::to_string(i + 1));
                std::string t = trim(line);
                if (t.empty() || t[0] == '#') {
                    if (vals.empty()) continue;
                }
                std::stringstream ss(line);
                while ((int)vals.size() < n && ss >> tok) {
                    double v;
                    if (!read_real(tok, v)) fail(" ERROR: " + trim(fname) + ": cannot read row " + std::to_string(i + 1));
                    vals.push_back(v);
                }
            }
            for (int j = 0; j < n; j++) A[i + (size_t)j * n] = vals[j];
        }
    }

    // the dense part on the solver's device (qs_dftb_lowdin): S^-1/2, the SOC form, H
    // (src/hamiltonian.f90:625-689); Lam as below (src/hamiltonian.f90:645-668)
    void build_dftb_lowdin_device(int N, const std::vector<double> &Ss, const std::vector<double> &Hs) {
        std::vector<cplx> Lam = soc_matrix();
        std::vector<cplx> Hn((size_t)Norb * Norb);
        double evmin = 0.0;
        int rc = api->dftb_lowdin(N, Ss.data(), Hs.data(), (const double *)Lam.data(), soc_form == "dual" ? 1 : 0,
                                  (double *)Hn.data(), &evmin, device);
        if (rc == 1) fail(" ERROR: overlap matrix is not positive definite (min eigenvalue " + std::to_string(evmin) + ")");
        if (rc != 0) fail(" ERROR: device set-up failed (dftb_lowdin status " + std::to_string(rc) + ")");
        say(" DFTB H0/S: smallest overlap eigenvalue = %10.2E\n", evmin);
        if (soc_form != "dual" && soc_form != "onsite") fail(" ERROR: soc_form must be dual or onsite, not " + soc_form);
        H = Hn;
        say(" DFTB H0/S Hamiltonian: %d atoms, %d orbitals, SOC form %s\n", N_atoms, N, soc_form.c_str());
    }

    // (L.S) xi on the p shells in the AO basis, spin fastest (src/hamiltonian.f90:645-668)
    std::vector<cplx> soc_matrix() const {
        // (L_k)_ab = -i eps_kab ; Pauli matrices
        cplx Lk[3][3][3] = {};
        Lk[0][1][2] = -IM; Lk[0][2][1] = IM;
        Lk[1][2][0] = -IM; Lk[1][0][2] = IM;
        Lk[2][0][1] = -IM; Lk[2][1][0] = IM;
        cplx sig[2][2][3] = {};
        sig[0][1][0] = 1.0; sig[1][0][0] = 1.0;
        sig[0][1][1] = -IM; sig[1][0][1] = IM;
        sig[0][0][2] = 1.0; sig[1][1][2] = -1.0;
        const int pidx[3] = {1, 2, 0};  // p_y, p_z, p_x -> y, z, x (0-based)
        std::vector<cplx> Lam((size_t)Norb * Norb, 0.0);
        for (int a = 0; a < N_atoms; a++) {
            if (atom_norb[a] < 4) continue;
            auto it = std::find(elem_name.begin(), elem_name.end(), atom_elem[a]);
            double xi = elem_xi[it - elem_name.begin()];
            if (xi == 0.0) continue;
            int i0 = atom_first[a];
            for (int p = 1; p <= 3; p++)
                for (int q = 1; q <= 3; q++)
                    for (int s1 = 1; s1 <= 2; s1++)
                        for (int s2 = 1; s2 <= 2; s2++) {
                            int i = 2 * (i0 + p - 1) + s1, j = 2 * (i0 + q - 1) + s2;
                            for (int k = 0; k < 3; k++)
                                Lam[(i - 1) + (size_t)(j - 1) * Norb] +=
                                    xi * Lk[k][pidx[p - 1]][pidx[q - 1]] * sig[s1 - 1][s2 - 1][k] / 2.0;
                        }
        }
        return Lam;
    }

    // src/hamiltonian.f90:606-708
    void build_from_dftb_hs() {
        const double hartree = 27.211386245988;
        int N = N_sites;
        std::vector<double> S, H0;
        read_dftb_square(overlap_file, N, S);
        read_dftb_square(ham_file, N, H0);
        std::vector<double> Ss((size_t)N * N), Hs((size_t)N * N);
        for (int j = 0; j < N; j++)
            for (int i = 0; i < N; i++) {
                Ss[i + (size_t)j * N] = 0.5 * (S[i + (size_t)j * N] + S[j + (size_t)i * N]);
                Hs[i + (size_t)j * N] = 0.5 * (H0[i + (size_t)j * N] + H0[j + (size_t)i * N]) * hartree;
            }
        if (api && api->dftb_lowdin) {
            build_dftb_lowdin_device(N, Ss, Hs);
            return;
        }
        // S^-1/2 = U diag(1/sqrt(s)) U^T
        std::vector<cplx> Sc(Ss.begin(), Ss.end()), Z;
        std::vector<double> ev;
        jacobi_herm(N, Sc, ev, Z);
        double evmin = *std::min_element(ev.begin(), ev.end());
        if (evmin <= 1e-8) fail(" ERROR: overlap matrix is not positive definite (min eigenvalue " + std::to_string(evmin) + ")");
        std::vector<double> U((size_t)N * N), Smh((size_t)N * N, 0.0);
        for (int k = 0; k < N; k++)
            for (int i = 0; i < N; i++) U[i + (size_t)k * N] = Z[i + (size_t)k * N].real() / std::sqrt(std::sqrt(ev[k]));
        for (int j = 0; j < N; j++)
            for (int i = 0; i < N; i++) {
                double s = 0;
                for (int k = 0; k < N; k++) s += U[i + (size_t)k * N] * U[j + (size_t)k * N];
                Smh[i + (size_t)j * N] = s;
            }
        say(" DFTB H0/S: smallest overlap eigenvalue = %10.2E\n", evmin);
        std::vector<cplx> Lam = soc_matrix();
        std::vector<cplx> Sx2((size_t)Norb * Norb, 0.0), Sm2((size_t)Norb * Norb, 0.0), Hao((size_t)Norb * Norb, 0.0);
        for (int j = 1; j <= N; j++)
            for (int i = 1; i <= N; i++)
                for (int s1 = 1; s1 <= 2; s1++) {
                    size_t id = (2 * (i - 1) + s1 - 1) + (size_t)(2 * (j - 1) + s1 - 1) * Norb;
                    Sx2[id] = Ss[(i - 1) + (size_t)(j - 1) * N];
                    Sm2[id] = Smh[(i - 1) + (size_t)(j - 1) * N];
                    Hao[id] = Hs[(i - 1) + (size_t)(j - 1) * N];
                }
        auto matmul = [&](const std::vector<cplx> &A, const std::vector<cplx> &B) {
            std::vector<cplx> C((size_t)Norb * Norb, 0.0);
            for (int j = 0; j < Norb; j++)
                for (int k = 0; k < Norb; k++) {
                    cplx b = B[k + (size_t)j * Norb];
                    if (b == 0.0) continue;
                    for (int i = 0; i < Norb; i++) C[i + (size_t)j * Norb] += A[i + (size_t)k * Norb] * b;
                }
            return C;
        };
        if (soc_form == "dual") {
            auto A1 = matmul(Sx2, Lam), A2 = matmul(Lam, Sx2);
            for (size_t k = 0; k < Hao.size(); k++) Hao[k] += 0.5 * (A1[k] + A2[k]);
        } else if (soc_form == "onsite") {
            for (size_t k = 0; k < Hao.size(); k++) Hao[k] += Lam[k];
        } else {
            fail(" ERROR: soc_form must be dual or onsite, not " + soc_form);
        }
        auto T1 = matmul(Hao, Sm2);
        auto Hn = matmul(Sm2, T1);
        for (int j = 0; j < Norb; j++)
            for (int i = 0; i < Norb; i++)
                H[i + (size_t)j * Norb] = 0.5 * (Hn[i + (size_t)j * Norb] + std::conj(Hn[j + (size_t)i * Norb]));
        say(" DFTB H0/S Hamiltonian: %d atoms, %d orbitals, SOC form %s\n", N_atoms, N, soc_form.c_str());
    }

    // src/hamiltonian.f90:741-755
    void build_custom() {
        for (int i = 1; i <= N_sites; i++) {
            int ii = 2 * i;
            h(ii - 1, ii - 1) = E_CC;
            h(ii, ii) = E_CC;
            if (i < N_sites) {
                h(ii - 1, ii + 1) = t_hop;
                h(ii, ii + 2) = t_hop;
            }
        }
        make_hermitian();
    }

    // src/quichotte.f90:241-253 energy grid from the spectrum of H
    void energy_grid() {
        if (api && api->hermitian_eigenvalues) {
            Ev.assign(Norb, 0.0);
            int info = 0;
            int rc = api->hermitian_eigenvalues(Norb, 1, (const double *)H.data(), Ev.data(), &info, device);
            if (rc == 1) fail(" ERROR: ZHEEV eigenproblem failed, INFO = " + std::to_string(info));
            if (rc != 0) fail(" ERROR: device set-up failed (hermitian_eigenvalues status " + std::to_string(rc) + ")");
        } else {
            std::vector<cplx> Z;
            jacobi_herm(Norb, H, Ev, Z);
        }
        w_init = Ev.front() - dw;
        w_fin = Ev.back() + up;
        n_omega = (int)((w_fin - w_init) / delta);  // Fortran int(): truncation
        omega.resize(n_omega);
        for (int i = 1; i <= n_omega; i++) omega[i - 1] = w_init + i * delta;
    }
};

qsh_model *to_c(const Model &m) {
    auto *c = (qsh_model *)std::calloc(1, sizeof(qsh_model));
    c->N_sites = m.N_sites;
    c->Norb = m.Norb;
    c->N_atoms = m.N_atoms;
    c->order = m.order;
    c->n_omega = m.n_omega;
    c->n_volt_steps = m.n_volt_steps;
    c->V = m.V; c->Vf = m.Vf; c->delv = m.delv; c->T = m.T; c->mu = m.mu; c->beta = m.beta;
    c->delta = m.delta; c->w_init = m.w_init; c->w_fin = m.w_fin; c->dw = m.dw; c->up = m.up;
    c->Ev_min = m.Ev.empty() ? 0 : m.Ev.front();
    c->Ev_max = m.Ev.empty() ? 0 : m.Ev.back();
    c->alpha_mix = m.alpha_mix; c->tolf = m.tolf; c->tolf_order1 = m.tolf_order1;
    c->nhist = m.nhist; c->maxscf = m.maxscf; c->continuation = m.continuation;
    c->broyden_single_precision = m.broyden_single_precision;
    c->write_hamiltonian = m.write_hamiltonian;
    int mx = 0;
    for (int v : m.atom_norb) mx = std::max(mx, v);
    c->per_atom = mx > 1;
    size_t nn = (size_t)m.Norb * m.Norb;
    auto cp = [](const void *src, size_t bytes) { void *d = std::malloc(bytes ? bytes : 1); if (bytes) std::memcpy(d, src, bytes); return d; };
    c->H = (double *)cp(m.H.data(), nn * sizeof(cplx));
    c->GammaL = (double *)cp(m.GammaL.data(), nn * sizeof(cplx));
    c->GammaR = (double *)cp(m.GammaR.data(), nn * sizeof(cplx));
    c->U_site = (double *)cp(m.U_site.data(), m.U_site.size() * sizeof(double));
    c->omega = (double *)cp(m.omega.data(), m.omega.size() * sizeof(double));
    c->Ev = (double *)cp(m.Ev.data(), m.Ev.size() * sizeof(double));
    c->atom_norb = (int *)cp(m.atom_norb.data(), m.atom_norb.size() * sizeof(int));
    c->atom_first = (int *)cp(m.atom_first.data(), m.atom_first.size() * sizeof(int));
    std::snprintf(c->model_name, sizeof c->model_name, "%s", m.hamiltonian_model.c_str());
    std::snprintf(c->input_file, sizeof c->input_file, "%s", m.input_file.c_str());
    return c;
}

// gfortran list-directed REAL(8): one blank separator + a 25-wide field; G editing with
// 17 significant digits: F form for 0.1 <= |x| < 1e17 (and for 0), left in the field
// with 5 trailing blanks; otherwise E form d.dddE+ddd right-aligned. The digits come from
// std::to_chars with a precision, which rounds exactly as printf does, several times
// faster (a spectral file holds n_omega x Norb numbers per voltage).
static int pad_right_aligned(char *buf, const char *val, int n, int width, int trail) {
    int k = 0;
    buf[k++] = ' ';
    for (int i = n; i < width; i++) buf[k++] = ' ';
    std::memcpy(buf + k, val, n);
    k += n;
    for (int i = 0; i < trail; i++) buf[k++] = ' ';
    buf[k] = 0;
    return k;
}

int fmt_real(double x, char *buf) {
    if (std::isnan(x)) return std::sprintf(buf, "%26s", "NaN");
    if (std::isinf(x)) return std::sprintf(buf, "%26s", x > 0 ? "Infinity" : "-Infinity");
    char val[64];
    if (x == 0.0) {
        const char *z = std::signbit(x) ? "-0.0000000000000000" : "0.0000000000000000";
        return pad_right_aligned(buf, z, (int)std::strlen(z), 20, 5);
    }
    char mant[48];
    const auto r = std::to_chars(mant, mant + sizeof mant, x, std::chars_format::scientific, 16);
    const char *ep = static_cast<const char *>(std::memchr(mant, 'e', r.ptr - mant));
    int e = 0;
    std::from_chars(ep[1] == '+' ? ep + 2 : ep + 1, r.ptr, e);
    if (e >= -1 && e < 17) {
        const auto f = std::to_chars(val, val + sizeof val, x, std::chars_format::fixed, 16 - e);
        return pad_right_aligned(buf, val, (int)(f.ptr - val), 20, 5);
    }
    // E form with a 3-digit exponent
    int n = (int)(ep - mant);
    std::memcpy(val, mant, n);
    n += std::sprintf(val + n, "E%c%03d", e < 0 ? '-' : '+', std::abs(e));
    return pad_right_aligned(buf, val, n, 25, 0);
}

}  // namespace

// ===================================================================================
// C ABI
// ===================================================================================
extern "C" {

int qsh_load(const char *dir, qsh_model **out, char *errbuf, int errlen, FILE *log) {
    return qsh_load_with(dir, nullptr, 0, out, errbuf, errlen, log);
}

int qsh_load_with(const char *dir, const qsh_solver_api *api, int device, qsh_model **out, char *errbuf, int errlen,
                  FILE *log) {
    Model m;
    m.dir = dir ? dir : ".";
    m.log = log;
    m.api = api;
    m.device = device;
    try {
        m.read_input();
        m.build_hamiltonian();
        m.setup_leads();
        m.setup_hubbard();
        m.energy_grid();
    } catch (const InputError &e) {
        if (errbuf && errlen > 0) std::snprintf(errbuf, errlen, "%s", e.what());
        *out = nullptr;
        return 1;
    }
    *out = to_c(m);
    return 0;
}

int qsh_helix(int N_ions, int N_turns, double hel_length, double hel_radius, double hand, double E_CC,
              double t_hop, double lamb, double U_int, double GammaL_up, double GammaL_down, double GammaR,
              double T, double mu, double dw, double up, double delta, int order, qsh_model **out) {
    Model m;
    m.N_ions = N_ions;
    m.N_turns = N_turns;
    m.hel_length = hel_length;
    m.hel_radius = hel_radius;
    m.hand = hand;
    m.E_CC = E_CC;
    m.t_hop = t_hop;
    m.lamb = lamb;
    m.U_int = U_int;
    m.GammaL_up = GammaL_up;
    m.GammaL_down = GammaL_down;
    m.GammaR_both = GammaR;
    m.T = T;
    m.mu = mu;
    m.dw = dw;
    m.up = up;
    m.delta = delta;
    m.order = order;
    m.V = m.Vf = 0.0;
    m.delv = 1.0;
    m.N_sites = N_ions * N_turns;
    try {
        m.check_input();
        m.beta = 1.0 / (kB * T);
        m.Norb = 2 * m.N_sites;
        m.set_atom_map();
        m.build_hamiltonian();
        m.setup_leads();
        m.setup_hubbard();
        m.energy_grid();
    } catch (const InputError &) {
        *out = nullptr;
        return 1;
    }
    *out = to_c(m);
    return 0;
}

void qsh_free(qsh_model *m) {
    if (!m) return;
    std::free(m->H);
    std::free(m->GammaL);
    std::free(m->GammaR);
    std::free(m->U_site);
    std::free(m->omega);
    std::free(m->Ev);
    std::free(m->atom_norb);
    std::free(m->atom_first);
    std::free(m);
}

int qsh_fmt_real(double x, char *buf) { return fmt_real(x, buf); }
int qsh_fmt_int(long v, char *buf) { return std::sprintf(buf, " %11ld", v); }

int qsh_write_iv(FILE *f, double V, double J_up, double J_down, int converged) {
    char b[64];
    std::string s;
    for (double x : {V, J_up, J_down, J_up + J_down}) { fmt_real(x, b); s += b; }
    qsh_fmt_int(converged ? 1 : 0, b);
    s += b;
    std::fprintf(f, "%s\n", s.c_str());
    std::fflush(f);
    return 0;
}

// src/observables.f90:41-86
int qsh_write_spin_texture(FILE *f, const qsh_model *m, double V, const double *Gl) {
    const int No = m->Norb;
    auto G = [&](int i, int j) { size_t k = 2 * ((i - 1) + (size_t)(j - 1) * No); return cplx(Gl[k], Gl[k + 1]); };
    const cplx px[2][2] = {{0.0, 1.0}, {1.0, 0.0}};
    const cplx py[2][2] = {{0.0, cplx(0, -1)}, {cplx(0, 1), 0.0}};
    const cplx pz[2][2] = {{1.0, 0.0}, {0.0, -1.0}};
    const cplx pref = -IM * 0.5;
    char b[64];
    for (int i = 1; i <= No; i += 2) {
        cplx tr[3] = {0.0, 0.0, 0.0};
        for (int s1 = 0; s1 <= 1; s1++)
            for (int s2 = 0; s2 <= 1; s2++) {
                cplx g = G(i + s2, i + s1);
                tr[0] += px[s1][s2] * g;
                tr[1] += py[s1][s2] * g;
                tr[2] += pz[s1][s2] * g;
            }
        cplx pu = -IM * G(i, i), pd = -IM * G(i + 1, i + 1), pt = pu + pd;
        std::string s;
        fmt_real(V, b); s += b;
        qsh_fmt_int((i + 1) / 2, b); s += b;
        for (int k = 0; k < 3; k++) { fmt_real((tr[k] * pref).real(), b); s += b; }
        for (double x : {pd.real(), pu.real(), pt.real()}) { fmt_real(x, b); s += b; }
        std::fprintf(f, "%s\n", s.c_str());
    }
    std::fflush(f);
    return 0;
}

// src/observables.f90:104-158
int qsh_write_atom_texture(FILE *f, const qsh_model *m, double V, const double *Gl) {
    const int No = m->Norb;
    auto G = [&](int i, int j) { size_t k = 2 * ((i - 1) + (size_t)(j - 1) * No); return cplx(Gl[k], Gl[k + 1]); };
    const cplx px[2][2] = {{0.0, 1.0}, {1.0, 0.0}};
    const cplx py[2][2] = {{0.0, cplx(0, -1)}, {cplx(0, 1), 0.0}};
    const cplx pz[2][2] = {{1.0, 0.0}, {0.0, -1.0}};
    cplx Lk[3][3][3] = {};
    for (int k = 1; k <= 3; k++) {
        Lk[k - 1][(k % 3)][((k + 1) % 3)] = -IM;
        Lk[k - 1][((k + 1) % 3)][(k % 3)] = IM;
    }
    const int cart[3] = {1, 2, 0};
    char b[64];
    for (int at = 0; at < m->N_atoms; at++) {
        double Sv[3] = {0, 0, 0}, Lv[3] = {0, 0, 0}, nu = 0, nd = 0;
        int first = m->atom_first[at], norb = m->atom_norb[at];
        for (int i = first; i <= first + norb - 1; i++) {
            cplx rho[2][2];
            for (int s1 = 1; s1 <= 2; s1++)
                for (int s2 = 1; s2 <= 2; s2++) rho[s1 - 1][s2 - 1] = -IM * G(2 * i - 2 + s1, 2 * i - 2 + s2);
            nu += rho[0][0].real();
            nd += rho[1][1].real();
            cplx sx = 0, sy = 0, sz = 0;
            for (int a = 0; a < 2; a++)
                for (int c = 0; c < 2; c++) {  // sum(pauli * transpose(rho))
                    sx += px[a][c] * rho[c][a];
                    sy += py[a][c] * rho[c][a];
                    sz += pz[a][c] * rho[c][a];
                }
            Sv[0] += 0.5 * sx.real();
            Sv[1] += 0.5 * sy.real();
            Sv[2] += 0.5 * sz.real();
        }
        if (norb == 4)
            for (int p = 1; p <= 3; p++)
                for (int q = 1; q <= 3; q++) {
                    int ip = first + p, iq = first + q;
                    cplx rhop = -IM * (G(2 * iq - 1, 2 * ip - 1) + G(2 * iq, 2 * ip));
                    for (int k = 0; k < 3; k++) Lv[k] += (Lk[k][cart[p - 1]][cart[q - 1]] * rhop).real();
                }
        std::string s;
        fmt_real(V, b); s += b;
        qsh_fmt_int(at + 1, b); s += b;
        for (double x : {Sv[0], Sv[1], Sv[2], nd, nu, nd + nu, Lv[0], Lv[1], Lv[2]}) { fmt_real(x, b); s += b; }
        std::fprintf(f, "%s\n", s.c_str());
    }
    std::fflush(f);
    return 0;
}

// src/observables.f90:89-102 (dosd is Norb x n_omega, column-major)
int qsh_write_spectral(FILE *f, const qsh_model *m, double V, const double *dosd) {
    std::fprintf(f, "# V = %10.5f   columns: V, omega, A_ii for i = 1..Norb\n", V);
    // rows are formatted in parallel blocks (n_omega x Norb numbers), then written in order
    const int nw = m->n_omega;
    const int nthr = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), nw / 256));
    std::vector<std::string> part(nthr);
    auto work = [&](int t) {
        const int w0 = (int)((int64_t)nw * t / nthr), w1 = (int)((int64_t)nw * (t + 1) / nthr);
        std::string &s = part[t];
        s.reserve((size_t)(w1 - w0) * (26 * (m->Norb + 2) + 1));
        char b[64];
        for (int iw = w0; iw < w1; iw++) {
            s.append(b, fmt_real(V, b));
            s.append(b, fmt_real(m->omega[iw], b));
            for (int i = 0; i < m->Norb; i++) s.append(b, fmt_real(-2.0 * dosd[i + (size_t)iw * m->Norb], b));
            s += '\n';
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nthr; t++) th.emplace_back(work, t);
    work(0);
    for (auto &x : th) x.join();
    for (auto &p : part) std::fwrite(p.data(), 1, p.size(), f);
    std::fputs("\n\n", f);
    std::fflush(f);
    return 0;
}

// src/hamiltonian.f90:710-721
int qsh_write_hamiltonian_matrix(const qsh_model *m, const char *path) {
    FILE *u = std::fopen(path, "w");
    if (!u) return 1;
    std::fprintf(u, "# QUICHOTTE Hamiltonian [eV]; state index 2*site-1 = up, 2*site = down\n");
    std::fprintf(u, "# Norb = %d\n", m->Norb);
    std::fprintf(u, "#   i   j   Re H_ij   Im H_ij\n");
    for (int j = 0; j < m->Norb; j++)
        for (int i = 0; i < m->Norb; i++) {
            double re = m->H[2 * (i + (size_t)j * m->Norb)], im = m->H[2 * (i + (size_t)j * m->Norb) + 1];
            if (re != 0.0 || im != 0.0) std::fprintf(u, "%6d%6d%25.16E%25.16E\n", i + 1, j + 1, re, im);
        }
    std::fclose(u);
    return 0;
}

// src/input_output.f90:464-497 (informational; not compared by the reference's tests)
int qsh_write_hamiltonian_info(const qsh_model *m, const char *path) {
    FILE *u = std::fopen(path, "w");
    if (!u) return 1;
    int No = m->Norb;
    std::fprintf(u, "\n... Hamiltonian:\n");
    for (int i = 0; i < No; i++) {
        for (int j = 0; j < No; j++)
            std::fprintf(u, " [%10.5f%10.5f] ", m->H[2 * (i + (size_t)j * No)], m->H[2 * (i + (size_t)j * No) + 1]);
        std::fprintf(u, "\n");
    }
    std::fprintf(u, "\n... Eigenvalues:\n");
    char b[64];
    for (int i = 0; i < No; i++) {
        qsh_fmt_int(i + 1, b);
        std::fprintf(u, "%s .", b);
        fmt_real(m->Ev[i], b);
        std::fprintf(u, "%s\n", b);
    }
    std::fprintf(u, " Norb:%12d\n", No);
    std::fclose(u);
    return 0;
}

int qsh_write_scf_line(FILE *f, int step, double fmax, double rms, int nh) {
    std::fprintf(f, "%6d%16.6E%16.6E%6d\n", step, fmax, rms, nh);
    std::fflush(f);
    return 0;
}

int qsh_scf_log_name(double V, char *buf, int len) {
    char t[32];
    std::snprintf(t, sizeof t, "%8.3f", V);
    std::string s = trim(t);
    return std::snprintf(buf, len, "scf_V_%s.dat", s.c_str());
}

}  // extern "C"
