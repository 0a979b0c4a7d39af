// AO -> MO integral transformation on the device for a closed-shell reference: the role of
// the reference's integral transformation (src/operator/aomoints.cxx:1017-1450, closed
// shell rhfaomoints.cxx:37-180) ahead of the CCSD iteration.  Four quarter
// transformations, each one gather-GEMM of the FP64 kernels over the contracted AO index:
//
//     X[a0][a1][a2][a3] (a3 fastest)  ->  Y[p][a0][a1][a2] = sum_a3 X[a0][a1][a2][a3] C[a3][p]
//
// so that the new index comes out slowest and four steps return (mu nu|la si) as (pq|rs) in
// the original order.  The MO Fock matrix of the occupied orbitals follows from the
// transformed integrals on the device: f = C^T h C + sum_i 2 (pq|ii) - (pi|iq).
#include <algorithm>
#include <cstring>

#include "engine.hpp"
#include "hbuild.hpp"

namespace ccsd {

namespace {

struct DeviceTables {
    Context& ctx;
    std::vector<std::pair<void*, size_t>> held;
    template <class T>
    T* up(const std::vector<T>& h) {
        const size_t b = std::max<size_t>(h.size(), 1) * sizeof(T);
        T* d = (T*)ctx.dmalloc(b);
        ctx.stage_h2d(d, h.data(), h.size() * sizeof(T));
        held.push_back({d, b});
        return d;
    }
    ~DeviceTables() {
        for (auto& p : held) ctx.dfree(p.first, p.second);   // stream-ordered
    }
};

// Y[p][m] = sum_k X[m * d3 + k] C[k * nmo + p],  m < M = d0 d1 d2, k < d3, p < nmo
void quarter(Context& ctx, const double* X, int64_t M, int d3, const double* dC, int nmo, double* Y) {
    if (M > INT32_MAX) throw Error(CCSD_ERR_UNSUPPORTED, "AO->MO transformation too large for one GEMM");
    DeviceTables tb{ctx, {}};
    std::vector<int64_t> am(M), cm(M), ak(d3), bk(d3), bn(nmo), cn(nmo);
    for (int64_t m = 0; m < M; m++) {
        am[m] = m * d3;
        cm[m] = m;
    }
    for (int k = 0; k < d3; k++) {
        ak[k] = k;
        bk[k] = (int64_t)k * nmo;
    }
    for (int p = 0; p < nmo; p++) {
        bn[p] = p;
        cn[p] = (int64_t)p * M;
    }
    kern::GemmArgs a;
    a.A = X;
    a.B = dC;
    a.C = Y;
    a.M = (int)M;
    a.N = nmo;
    a.K = d3;
    a.alpha = 1.0;
    a.Am = tb.up(am);
    a.Ak = tb.up(ak);
    a.Bk = tb.up(bk);
    a.Bn = tb.up(bn);
    a.Cm[0] = tb.up(cm);
    a.Cn[0] = tb.up(cn);
    a.a_kcontig = true;
    a.b_kcontig = false;
    a.ak_affine = true;
    a.ak0 = 0;
    a.ak_step = 1;
    a.bk_affine = true;
    a.bk0 = 0;
    a.bk_step = nmo;
    CCSD_CUDA(cudaMemsetAsync(Y, 0, (size_t)M * nmo * sizeof(double), ctx.stream));
    kern::gemm_fp64(a, ctx.stream);
}

}  // namespace

double ao_to_mo(Context& ctx, int nao, int nmo, int nocc, const double* hcore, const double* eri_ao,
                const double* C, double* d_mo, double* fock) {
    if (nao <= 0 || nmo <= 0 || nmo > nao || nocc < 0 || nocc > nmo)
        throw Error(CCSD_ERR_ARG, "AO->MO: need 0 < nmo <= nao and 0 <= nocc <= nmo");
    const int64_t n1 = nao, m1 = nmo;
    const int64_t big = n1 * n1 * n1 * n1, mid = m1 * n1 * n1 * n1;
    double* bufA = (double*)ctx.dmalloc(big * sizeof(double));   // AO integrals, then the half-transformed
    double* bufB = (double*)ctx.dmalloc(mid * sizeof(double));   // first and third quarters
    double* dC = (double*)ctx.dmalloc(n1 * m1 * sizeof(double));
    double* dF = (double*)ctx.dmalloc(m1 * m1 * sizeof(double));
    struct Free {
        Context& c;
        std::vector<std::pair<void*, size_t>> p;
        ~Free() {
            cudaStreamSynchronize(c.stream);
            for (auto& x : p) c.dfree(x.first, x.second);
        }
    } guard{ctx, {{bufA, big * sizeof(double)}, {bufB, mid * sizeof(double)}, {dC, n1 * m1 * sizeof(double)},
                  {dF, m1 * m1 * sizeof(double)}}};
    CCSD_CUDA(cudaMemcpyAsync(bufA, eri_ao, big * sizeof(double), cudaMemcpyHostToDevice, ctx.stream));
    CCSD_CUDA(cudaMemcpyAsync(dC, C, n1 * m1 * sizeof(double), cudaMemcpyHostToDevice, ctx.stream));
    // (mu nu|la si) -> [s][mu][nu][la] -> [r][s][mu][nu] -> [q][r][s][mu] -> [p][q][r][s]
    quarter(ctx, bufA, n1 * n1 * n1, nao, dC, nmo, bufB);
    quarter(ctx, bufB, m1 * n1 * n1, nao, dC, nmo, bufA);
    quarter(ctx, bufA, m1 * m1 * n1, nao, dC, nmo, bufB);
    quarter(ctx, bufB, m1 * m1 * m1, nao, dC, nmo, d_mo);
    // MO Fock matrix: the core part on the host (nao^2 nmo), the two-electron part on the device
    kern::closed_shell_jk(d_mo, nmo, nocc, dF, ctx.stream);
    std::vector<double> f2(m1 * m1), t(n1 * m1), h(m1 * m1);
    CCSD_CUDA(cudaMemcpyAsync(f2.data(), dF, m1 * m1 * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
    for (int mu = 0; mu < nao; mu++)
        for (int q = 0; q < nmo; q++) {
            double x = 0;
            for (int nu = 0; nu < nao; nu++) x += hcore[(int64_t)mu * nao + nu] * C[(int64_t)nu * nmo + q];
            t[(int64_t)mu * nmo + q] = x;
        }
    for (int p = 0; p < nmo; p++)
        for (int q = 0; q < nmo; q++) {
            double x = 0;
            for (int mu = 0; mu < nao; mu++) x += C[(int64_t)mu * nmo + p] * t[(int64_t)mu * nmo + q];
            h[(int64_t)p * nmo + q] = x;
        }
    CCSD_CUDA(cudaStreamSynchronize(ctx.stream));
    double e = 0;
    for (int p = 0; p < nmo; p++)
        for (int q = 0; q < nmo; q++) {
            // the core part is symmetrised (the AO matrix is symmetric up to rounding)
            const double hs = 0.5 * (h[(int64_t)p * nmo + q] + h[(int64_t)q * nmo + p]);
            fock[(int64_t)p * nmo + q] = hs + f2[(int64_t)p * nmo + q];
        }
    for (int i = 0; i < nocc; i++) e += h[(int64_t)i * nmo + i] + fock[(int64_t)i * nmo + i];
    return e;
}

}  // namespace ccsd
