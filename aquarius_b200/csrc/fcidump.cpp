// FCIDUMP reader and the closed-shell Fock build that goes with it.
//
// Role of the reference's "fcidump" task (src/operator/fcidump.cxx:35-516):
// * header: the lines up to one holding "/", "&END" or "$END" (case-insensitive), with
//   NORB and NELEC read from them; the first NELEC/2 orbitals are occupied (C1, closed
//   shell) (fcidump.cxx:50-67);
// * records "value p q r s" with 1-based orbital indices: p = 0 is the core energy,
//   q = 0 (orbital energies) is skipped, r = 0 is h_pq (mirrored to h_qp unless the
//   one-electron integrals are given in full), anything else is (pq|rs) in chemists'
//   notation, taken only from its canonical image (p >= q, r >= s, pq >= rs) and set on
//   all eight (fcidump.cxx:100-277);
// * Fock matrix f = h + sum_i [2 (pq|ii) - (pi|iq)] and E(SCF) = E_core + sum_i (h_ii + f_ii)
//   (the accumulations of fcidump.cxx:122-259);
// * optional semicanonical orbitals: the occupied and the virtual Fock blocks are
//   diagonalised and every integral rotated (fcidump.cxx:362-470).
// Integrals are held densely (n^4 doubles), which is what the device gather consumes.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

#include "engine.hpp"
#include "hbuild.hpp"

namespace ccsd {

namespace {

std::string upper(std::string s) {
    for (auto& c : s) c = (char)std::toupper((unsigned char)c);
    return s;
}

bool header_value(const std::string& header, const char* key, int& out) {
    const std::string H = upper(header);
    const std::string K = key;
    size_t pos = 0;
    while ((pos = H.find(K, pos)) != std::string::npos) {
        // whole word: not preceded by a letter
        if (pos > 0 && std::isalpha((unsigned char)H[pos - 1])) {
            pos += K.size();
            continue;
        }
        size_t q = pos + K.size();
        while (q < H.size() && std::isspace((unsigned char)H[q])) q++;
        if (q < H.size() && H[q] == '=') {
            q++;
            while (q < H.size() && std::isspace((unsigned char)H[q])) q++;
            if (q < H.size() && std::isdigit((unsigned char)H[q])) {
                out = std::atoi(H.c_str() + q);
                return true;
            }
        }
        pos += K.size();
    }
    return false;
}

// symmetric eigen-decomposition by cyclic Jacobi rotations: A (m x m, row-major) is
// destroyed, eigenvalues ascending in w, eigenvectors as the columns of V
void jacobi_eigen(int m, std::vector<double>& A, std::vector<double>& w, std::vector<double>& V) {
    V.assign((size_t)m * m, 0.0);
    for (int i = 0; i < m; i++) V[(size_t)i * m + i] = 1.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < m; i++)
            for (int j = 0; j < m; j++) (i == j ? diag : off) += A[(size_t)i * m + j] * A[(size_t)i * m + j];
        if (off <= 1e-30 * std::max(diag, 1e-300)) break;
        for (int p = 0; p < m; p++)
            for (int q = p + 1; q < m; q++) {
                const double apq = A[(size_t)p * m + q];
                if (apq == 0.0) continue;
                const double app = A[(size_t)p * m + p], aqq = A[(size_t)q * m + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < m; k++) {
                    const double akp = A[(size_t)k * m + p], akq = A[(size_t)k * m + q];
                    A[(size_t)k * m + p] = c * akp - s * akq;
                    A[(size_t)k * m + q] = s * akp + c * akq;
                }
                for (int k = 0; k < m; k++) {
                    const double apk = A[(size_t)p * m + k], aqk = A[(size_t)q * m + k];
                    A[(size_t)p * m + k] = c * apk - s * aqk;
                    A[(size_t)q * m + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < m; k++) {
                    const double vkp = V[(size_t)k * m + p], vkq = V[(size_t)k * m + q];
                    V[(size_t)k * m + p] = c * vkp - s * vkq;
                    V[(size_t)k * m + q] = s * vkp + c * vkq;
                }
            }
    }
    std::vector<int> order(m);
    for (int i = 0; i < m; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return A[(size_t)a * m + a] < A[(size_t)b * m + b]; });
    w.resize(m);
    std::vector<double> Vs((size_t)m * m);
    for (int j = 0; j < m; j++) {
        w[j] = A[(size_t)order[j] * m + order[j]];
        for (int k = 0; k < m; k++) Vs[(size_t)k * m + j] = V[(size_t)k * m + order[j]];
    }
    V.swap(Vs);
}

}  // namespace

Fcidump read_fcidump(const char* path, bool full_fock, bool header_only) {
    std::ifstream in(path);
    if (!in) throw Error(CCSD_ERR_ARG, std::string("cannot open FCIDUMP file ") + path);
    Fcidump d;
    std::string header, line;
    bool ended = false;
    while (std::getline(in, line)) {
        header += " " + line;
        const std::string U = upper(line);
        if (U.find('/') != std::string::npos || U.find("&END") != std::string::npos ||
            U.find("$END") != std::string::npos) {
            ended = true;
            break;
        }
    }
    if (!ended) throw Error(CCSD_ERR_ARG, "FCIDUMP header has no terminator (/, &END or $END)");
    if (!header_value(header, "NORB", d.norb) || d.norb <= 0) throw Error(CCSD_ERR_ARG, "FCIDUMP header lacks NORB");
    if (!header_value(header, "NELEC", d.nelec) || d.nelec < 0)
        throw Error(CCSD_ERR_ARG, "FCIDUMP header lacks NELEC");
    if (d.nelec > 2 * d.norb) throw Error(CCSD_ERR_ARG, "FCIDUMP NELEC exceeds 2*NORB");
    if (header_only) return d;
    const int64_t n = d.norb;
    if (n > 400) throw Error(CCSD_ERR_UNSUPPORTED, "FCIDUMP with more than 400 orbitals (dense n^4 storage)");
    d.h.assign(n * n, 0.0);
    d.eri.assign(n * n * n * n, 0.0);
    auto at = [n](int64_t p, int64_t q, int64_t r, int64_t s) { return ((p * n + q) * n + r) * n + s; };
    int64_t lineno = 0;
    while (std::getline(in, line)) {
        lineno++;
        for (auto& c : line)
            if (c == 'D' || c == 'd') c = 'E';   // Fortran exponents
        std::istringstream ls(line);
        double val;
        int64_t p, q, r, s;
        if (line.find_first_not_of(" \t\r") == std::string::npos) continue;   // blank line
        if (!(ls >> val >> p >> q >> r >> s)) throw Error(CCSD_ERR_ARG, "malformed FCIDUMP record at data line " + std::to_string(lineno));
        if (p < 0 || q < 0 || r < 0 || s < 0 || p > n || q > n || r > n || s > n)
            throw Error(CCSD_ERR_ARG, "FCIDUMP orbital index out of range at data line " + std::to_string(lineno));
        if (p == 0) {
            d.ecore += val;
        } else if (q == 0) {
            continue;
        } else if (r == 0) {
            p--;
            q--;
            d.h[p * n + q] += val;
            if (!full_fock && p != q) d.h[q * n + p] += val;
        } else {
            if (p < q) std::swap(p, q);
            if (r < s) std::swap(r, s);
            if (p < r || (p == r && q < s)) continue;   // non-canonical image: skipped
            p--;
            q--;
            r--;
            s--;
            for (int64_t k : {at(p, q, r, s), at(q, p, r, s), at(p, q, s, r), at(q, p, s, r), at(r, s, p, q),
                              at(s, r, p, q), at(r, s, q, p), at(s, r, q, p)})
                d.eri[k] = val;
        }
    }
    return d;
}

double closed_shell_fock(int n, int nocc, const double* h, const double* eri, double* fock) {
    const int64_t N = n;
    auto at = [N](int64_t p, int64_t q, int64_t r, int64_t s) { return ((p * N + q) * N + r) * N + s; };
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < N; p++)
        for (int64_t q = 0; q < N; q++) {
            double f = h[p * N + q];
            for (int64_t i = 0; i < nocc; i++) f += 2.0 * eri[at(p, q, i, i)] - eri[at(p, i, i, q)];
            fock[p * N + q] = f;
        }
    double e = 0.0;
    for (int64_t i = 0; i < nocc; i++) e += h[i * N + i] + fock[i * N + i];
    return e;
}

void semicanonicalize(int n, int nocc, double* fock, double* eri) {
    const int64_t N = n;
    // U = blockdiag(U_occ, U_vrt): eigenvectors of the two diagonal Fock blocks
    std::vector<double> U(N * N, 0.0);
    for (int blk = 0; blk < 2; blk++) {
        const int lo = blk == 0 ? 0 : nocc, m = blk == 0 ? nocc : n - nocc;
        if (m == 0) continue;
        std::vector<double> A((size_t)m * m), w, V;
        for (int i = 0; i < m; i++)
            for (int j = 0; j < m; j++) A[(size_t)i * m + j] = 0.5 * (fock[(lo + i) * N + lo + j] + fock[(lo + j) * N + lo + i]);
        jacobi_eigen(m, A, w, V);
        for (int i = 0; i < m; i++)
            for (int j = 0; j < m; j++) U[(lo + i) * N + lo + j] = V[(size_t)i * m + j];
    }
    // f' = U^T f U
    std::vector<double> t(N * N, 0.0), f2(N * N, 0.0);
    for (int64_t p = 0; p < N; p++)
        for (int64_t b = 0; b < N; b++) {
            double acc = 0.0;
            for (int64_t q = 0; q < N; q++) acc += fock[p * N + q] * U[q * N + b];
            t[p * N + b] = acc;
        }
    for (int64_t a = 0; a < N; a++)
        for (int64_t b = 0; b < N; b++) {
            double acc = 0.0;
            for (int64_t p = 0; p < N; p++) acc += U[p * N + a] * t[p * N + b];
            f2[a * N + b] = acc;
        }
    std::copy(f2.begin(), f2.end(), fock);
    // four passes of "transform the last index, rotate the index order (p,q,r,s) -> (s,p,q,r)"
    const int64_t n3 = N * N * N;
    std::vector<double> out(n3 * N);
    for (int pass = 0; pass < 4; pass++) {
#pragma omp parallel for schedule(static)
        for (int64_t pqr = 0; pqr < n3; pqr++) {
            const double* row = eri + pqr * N;
            for (int64_t s = 0; s < N; s++) {
                double acc = 0.0;
                for (int64_t x = 0; x < N; x++) acc += row[x] * U[x * N + s];
                out[s * n3 + pqr] = acc;
            }
        }
        std::copy(out.begin(), out.end(), eri);
    }
}

}  // namespace ccsd
