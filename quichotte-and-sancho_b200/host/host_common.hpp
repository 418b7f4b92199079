// host_common.hpp -- pieces shared by the host layers of QUICHOTTE and SANCHO (qs_host.cpp,
// sancho_host.cpp): the input.dat reader (common/input_parser.f90:49-249, identical in both
// codes), Fortran list-directed value reads, and a cyclic Jacobi Hermitian eigensolver for
// the set-up (the host layers have no LAPACK). Included inside an anonymous namespace.
#pragma once

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

using cplx = std::complex<double>;
constexpr double kB = 8.6173303e-5;  // eV/K, common/constants.f90:20
constexpr double PI = 3.14159265358979323846;
const cplx IM(0.0, 1.0);

struct InputError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

std::string trim(const std::string &s) {
    size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

// First list-directed item of a string: blanks skipped, ended by blank, comma or slash.
std::string first_item(const std::string &s) {
    size_t a = s.find_first_not_of(" \t\r\n,");
    if (a == std::string::npos) return "";
    size_t b = s.find_first_of(" \t\r\n,/", a);
    return s.substr(a, b == std::string::npos ? std::string::npos : b - a);
}

// Fortran list-directed REAL read of one item (accepts d/D exponents, '2', '.5').
bool read_real(const std::string &s, double &v) {
    std::string t = first_item(s);
    if (t.empty()) return false;
    for (char &c : t)
        if (c == 'd' || c == 'D' || c == 'q' || c == 'Q') c = 'e';
    char *end = nullptr;
    errno = 0;
    v = std::strtod(t.c_str(), &end);
    return end && *end == '\0' && end != t.c_str();
}

// Fortran list-directed LOGICAL: optional '.', then T/F, rest ignored.
bool read_logical(const std::string &s, bool &v) {
    std::string t = first_item(s);
    if (t.empty()) return false;
    size_t p = (t[0] == '.') ? 1 : 0;
    if (p >= t.size()) return false;
    char c = (char)std::toupper((unsigned char)t[p]);
    if (c == 'T') { v = true; return true; }
    if (c == 'F') { v = false; return true; }
    return false;
}

// ---------------------------------------------------------------------------------
// InputParser (common/input_parser.f90)
// ---------------------------------------------------------------------------------
struct InputParser {
    struct Entry { std::string key, val; int line; bool used; };
    std::vector<Entry> keys;
    int n_missing = 0;
    bool duplicate_found = false;
    std::string file_name;
    std::string errors;  // accumulated error text (reference: error_unit)
    FILE *log = nullptr;

    void load(const std::string &dir, const std::vector<std::string> &cands) {
        file_name.clear();
        for (auto &c : cands) {
            std::ifstream f(dir + "/" + c);
            if (f.good()) { file_name = c; break; }
        }
        if (file_name.empty()) {
            std::string m = " ERROR: no input file found; looked for:\n";
            for (auto &c : cands) m += "    " + c + "\n";
            throw InputError(m);
        }
        std::ifstream f(dir + "/" + file_name);
        std::string line;
        int nline = 0;
        while (std::getline(f, line)) {
            nline++;
            std::string l = trim(line);
            if (l.empty() || l[0] == '#') continue;
            size_t hash = l.find('#');
            if (hash != std::string::npos) l = l.substr(0, hash);
            size_t eq = l.find('=');
            if (eq == std::string::npos) {
                if (log) std::fprintf(log, " WARNING: line %d of %s has no \"=\" (ignored): %s\n", nline,
                                      file_name.c_str(), trim(l).c_str());
                continue;
            }
            std::string key = trim(l.substr(0, eq)).substr(0, 64);
            std::string val = trim(l.substr(eq + 1));
            for (auto &e : keys)
                if (e.key == key) {
                    errors += " ERROR: key \"" + key + "\" given twice, lines " + std::to_string(e.line) +
                              " and " + std::to_string(nline) + "\n";
                    duplicate_found = true;
                }
            if (keys.size() == 200) throw InputError(" ERROR: more than 200 keys in " + file_name);
            keys.push_back({key, val, nline, false});
        }
    }
    int find(const std::string &key, const char *alias) {
        int j = -1;
        for (size_t i = 0; i < keys.size(); i++)
            if (keys[i].key == key) { j = (int)i; break; }
        if (j < 0 && alias) {
            std::stringstream ss(alias);
            std::string a;
            while (j < 0 && std::getline(ss, a, ',')) {
                a = trim(a);
                for (size_t i = 0; i < keys.size(); i++)
                    if (keys[i].key == a) { j = (int)i; break; }
            }
        }
        if (j >= 0) keys[j].used = true;
        return j;
    }
    void missing(const std::string &key) {
        errors += " ERROR: required key \"" + key + "\" missing from " + file_name + "\n";
        n_missing++;
    }
    [[noreturn]] void bad_value(int j) {
        throw InputError(errors + " ERROR: cannot read the value of \"" + keys[j].key + "\" on line " +
                         std::to_string(keys[j].line) + " of " + file_name + "\n        value was: \"" +
                         keys[j].val + "\"");
    }
    void get(const std::string &key, double &v, const double *def = nullptr, const char *alias = nullptr) {
        int j = find(key, alias);
        if (j < 0) { if (def) v = *def; else missing(key); return; }
        if (!read_real(keys[j].val, v)) bad_value(j);
    }
    void get(const std::string &key, int &v, const int *def = nullptr, const char *alias = nullptr) {
        int j = find(key, alias);
        if (j < 0) { if (def) v = *def; else missing(key); return; }
        double r;
        if (!read_real(keys[j].val, r) || std::fabs(r - std::nearbyint(r)) > 1e-9) bad_value(j);
        v = (int)std::lround(r);
    }
    void get(const std::string &key, bool &v, const bool *def = nullptr, const char *alias = nullptr) {
        int j = find(key, alias);
        if (j < 0) { if (def) v = *def; else missing(key); return; }
        if (!read_logical(keys[j].val, v)) bad_value(j);
    }
    void get(const std::string &key, std::string &v, const char *def = nullptr, const char *alias = nullptr) {
        int j = find(key, alias);
        if (j < 0) { if (def) v = def; else missing(key); return; }
        v = keys[j].val;
    }
    void finish() {
        for (auto &e : keys)
            if (!e.used && log)
                std::fprintf(log, " WARNING: unknown input key \"%s\" on line %d (ignored -- typo?)\n",
                             e.key.c_str(), e.line);
        if (n_missing > 0 || duplicate_found)
            throw InputError(errors + " Stopping: fix the input file (see the examples/ folder).");
    }
};

// ---------------------------------------------------------------------------------
// Hermitian eigenproblem by cyclic Jacobi rotations (replaces LAPACK zheev/dsyev of the
// set-up). A (n x n, column-major, Hermitian) is destroyed; eigenvalues ascending in E,
// eigenvectors in the columns of Z.
// ---------------------------------------------------------------------------------
void jacobi_herm(int n, std::vector<cplx> A, std::vector<double> &E, std::vector<cplx> &Z) {
    auto a = [&](int i, int j) -> cplx & { return A[i + (size_t)j * n]; };
    Z.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) Z[i + (size_t)i * n] = 1.0;
    for (int i = 0; i < n; i++) a(i, i) = a(i, i).real();
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, tot = 0.0;
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                double v = std::norm(a(i, j));
                tot += v;
                if (i != j) off += v;
            }
        if (off <= 1e-30 * tot || off == 0.0) break;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                cplx apq = a(p, q);
                double mag = std::abs(apq);
                if (mag == 0.0) continue;
                double app = a(p, p).real(), aqq = a(q, q).real();
                // rotate in the (p,q) plane: phase removal then a real Givens rotation
                cplx ph = apq / mag;  // a_pq = mag * ph
                double theta = 0.5 * std::atan2(2.0 * mag, aqq - app);
                double c = std::cos(theta), s = std::sin(theta);
                // J = [[c, s*ph], [-s*conj(ph), c]] acting on columns p,q (A <- J^H A J)
                for (int k = 0; k < n; k++) {  // columns
                    cplx akp = a(k, p), akq = a(k, q);
                    a(k, p) = c * akp - s * std::conj(ph) * akq;
                    a(k, q) = s * ph * akp + c * akq;
                }
                for (int k = 0; k < n; k++) {  // rows
                    cplx apk = a(p, k), aqk = a(q, k);
                    a(p, k) = c * apk - s * ph * aqk;
                    a(q, k) = s * std::conj(ph) * apk + c * aqk;
                }
                a(p, q) = 0.0;
                a(q, p) = 0.0;
                a(p, p) = a(p, p).real();
                a(q, q) = a(q, q).real();
                for (int k = 0; k < n; k++) {
                    cplx zkp = Z[k + (size_t)p * n], zkq = Z[k + (size_t)q * n];
                    Z[k + (size_t)p * n] = c * zkp - s * std::conj(ph) * zkq;
                    Z[k + (size_t)q * n] = s * ph * zkp + c * zkq;
                }
            }
    }
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return a(x, x).real() < a(y, y).real(); });
    E.resize(n);
    std::vector<cplx> Zs((size_t)n * n);
    for (int k = 0; k < n; k++) {
        E[k] = a(idx[k], idx[k]).real();
        for (int i = 0; i < n; i++) Zs[i + (size_t)k * n] = Z[i + (size_t)idx[k] * n];
    }
    Z.swap(Zs);
}

}  // namespace
