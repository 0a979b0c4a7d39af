// Seeded synthetic closed-shell integral producer.
//
// Plays the role of the reference's size-only H producer
// (src/operator/fakemoints.cxx:15-52) but with non-zero, reproducible values:
//
//   orbital energies  occ ~ U[-1.2,-0.4] Eh, vrt ~ U[0.3,4.0] Eh, sorted
//                      ascending within each irrep, Fock = diag(eps);
//   factor            B[P,p,q] = B[P,q,p] = N(0,1) * 0.25/sqrt(NP) * exp(-|p-q|/n),
//                      NP = 3 n, nonzero only when irrep(P) = irrep(p) ^ irrep(q);
//   integrals          (pq|rs) = sum_P B[P,p,q] B[P,r,s].
//
// Every draw comes from a counter-based generator (splitmix64 finaliser of a
// hashed (seed, stream, index) triple), so any subset of B can be produced
// independently and the host and every consumer see bit-identical values.
// Normal draws use the Box-Muller transform; irrep sizes (D2h) use a
// Dirichlet(1.5) split (Marsaglia-Tsang gamma sampler) rounded with largest
// remainders, every irrep getting at least one orbital.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <numeric>

#include "ccsd_b200.h"

namespace {

inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

inline uint64_t draw(uint64_t seed, uint64_t stream, uint64_t idx) {
    return mix64(mix64(seed * 0xD1B54A32D192ED03ull + stream) ^ (idx * 0x8CB92BA72F3D8DD7ull));
}

// uniform in [0,1)
inline double uni(uint64_t seed, uint64_t stream, uint64_t idx) {
    return (double)(draw(seed, stream, idx) >> 11) * 0x1.0p-53;
}

// standard normal, one Box-Muller draw per index
inline double gauss(uint64_t seed, uint64_t stream, uint64_t idx) {
    double u1 = 1.0 - uni(seed, stream, 2 * idx);      // (0,1]
    double u2 = uni(seed, stream, 2 * idx + 1);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

// Marsaglia-Tsang gamma(alpha >= 1) using a private counter
double gamma_draw(uint64_t seed, uint64_t stream, uint64_t& ctr, double alpha) {
    const double d = alpha - 1.0 / 3.0, c = 1.0 / std::sqrt(9.0 * d);
    for (int guard = 0; guard < 1000; guard++) {
        double x = gauss(seed, stream, ctr++);
        double v = 1.0 + c * x;
        if (v <= 0) continue;
        v = v * v * v;
        double u = uni(seed, stream + 1000, ctr++);
        if (std::log(u) < 0.5 * x * x + d - d * v + d * std::log(v)) return d * v;
    }
    return d;
}

// split `total` into nirrep parts, each >= 1, proportional to a Dirichlet draw
void dirichlet_split(uint64_t seed, uint64_t stream, int total, int nirrep, int* out) {
    if (nirrep == 1) { out[0] = total; return; }
    std::vector<double> g(nirrep);
    uint64_t ctr = 0;
    double s = 0;
    for (int h = 0; h < nirrep; h++) { g[h] = gamma_draw(seed, stream, ctr, 1.5); s += g[h]; }
    int rest = total - nirrep;              // one orbital per irrep up front
    std::vector<double> share(nirrep);
    std::vector<int> cnt(nirrep);
    int used = 0;
    for (int h = 0; h < nirrep; h++) {
        share[h] = rest * g[h] / s;
        cnt[h] = (int)std::floor(share[h]);
        used += cnt[h];
    }
    std::vector<int> order(nirrep);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (share[a] - cnt[a]) > (share[b] - cnt[b]);
    });
    for (int k = 0; used < rest; k++, used++) cnt[order[k % nirrep]]++;
    for (int h = 0; h < nirrep; h++) out[h] = cnt[h] + 1;
}

} // namespace

extern "C" {

int ccsd_synth_irreps(uint64_t seed, int nirrep, int o, int v,
                      int* occ_per_irrep, int* vrt_per_irrep, int* aux_per_irrep)
{
    if (nirrep != 1 && nirrep != 2 && nirrep != 4 && nirrep != 8) return CCSD_ERR_ARG;
    if (o < nirrep || v < nirrep) return CCSD_ERR_ARG;
    const int n = o + v, naux = 3 * n;
    dirichlet_split(seed, 4, o, nirrep, occ_per_irrep);
    dirichlet_split(seed, 5, v, nirrep, vrt_per_irrep);
    if (aux_per_irrep) dirichlet_split(seed, 6, naux, nirrep, aux_per_irrep);
    return CCSD_OK;
}

int ccsd_synth_problem(uint64_t seed, int nirrep,
                       const int* occ_per_irrep, const int* vrt_per_irrep, const int* aux_per_irrep,
                       double* eps, double* B)
{
    if (nirrep != 1 && nirrep != 2 && nirrep != 4 && nirrep != 8) return CCSD_ERR_ARG;
    int o = 0, v = 0, naux = 0;
    for (int h = 0; h < nirrep; h++) { o += occ_per_irrep[h]; v += vrt_per_irrep[h]; naux += aux_per_irrep[h]; }
    const int n = o + v;
    // irrep label of every spatial orbital: occupied first (irrep-major), then virtual
    std::vector<int> irr(n), auxirr(naux);
    {
        int p = 0;
        for (int h = 0; h < nirrep; h++) for (int i = 0; i < occ_per_irrep[h]; i++) irr[p++] = h;
        for (int h = 0; h < nirrep; h++) for (int a = 0; a < vrt_per_irrep[h]; a++) irr[p++] = h;
        int P = 0;
        for (int h = 0; h < nirrep; h++) for (int k = 0; k < aux_per_irrep[h]; k++) auxirr[P++] = h;
    }
    if (eps) {
        for (int p = 0; p < n; p++) {
            eps[p] = p < o ? -1.2 + 0.8 * uni(seed, 1, p) : 0.3 + 3.7 * uni(seed, 2, p);
        }
        int p = 0;
        for (int h = 0; h < nirrep; h++) { std::sort(eps + p, eps + p + occ_per_irrep[h]); p += occ_per_irrep[h]; }
        for (int h = 0; h < nirrep; h++) { std::sort(eps + p, eps + p + vrt_per_irrep[h]); p += vrt_per_irrep[h]; }
    }
    if (B) {
        const double scale = 0.25 / std::sqrt((double)naux);
        #pragma omp parallel for schedule(static)
        for (int P = 0; P < naux; P++) {
            double* BP = B + (size_t)P * n * n;
            for (int p = 0; p < n; p++) {
                for (int q = p; q < n; q++) {
                    double val = 0.0;
                    if ((irr[p] ^ irr[q]) == auxirr[P]) {
                        uint64_t idx = ((uint64_t)P * n + p) * n + q;
                        val = gauss(seed, 3, idx) * scale * std::exp(-(double)(q - p) / n);
                    }
                    BP[p * n + q] = val;
                    BP[q * n + p] = val;
                }
            }
        }
    }
    return CCSD_OK;
}

} // extern "C"
