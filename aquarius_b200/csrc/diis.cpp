// Standalone DIIS over caller tensors: the reference's DIIS<T>::extrapolate
// (src/convergence/diis.hpp:70-227) for a caller that keeps its own iteration, on the
// same device ring, error-matrix dots, bordered solve and linear combinations as the
// CCSD solver's.  A vector is the concatenation of the caller's pieces (e.g. T1 and T2);
// its inner product is the weighted sum of the pieces' full spin-orbital dots
// (ExcitationOperator::dot, src/operator/excitationoperator.hpp:77-87: weights 1 for
// T1 and 1/4 for T2 by default).
#include "diis.hpp"

#include <cmath>
#include <cstring>
#include <string>

#include "kernels.hpp"

namespace ccsd {

DiisRing::DiisRing(Context& c, int order_, int start_, double damping_)
    : ctx(c), order(order_), start(start_), damping(damping_) {
    if (order < 1 || order > 16) throw Error(CCSD_ERR_ARG, "DIIS order must be in 1..16");
    if (damping < 0.0 || !std::isfinite(damping)) throw Error(CCSD_ERR_ARG, "DIIS damping must be >= 0");
    CCSD_CUDA(cudaMallocHost(&h_state, 8 * sizeof(int)));
    CCSD_CUDA(cudaMallocHost(&h_c, 17 * sizeof(double)));
}

DiisRing::~DiisRing() {
    const size_t vb = (size_t)std::max<int64_t>(vec_len, 1) * sizeof(double);
    for (double* p : xs) ctx.dfree(p, vb);
    for (double* p : dxs) ctx.dfree(p, vb);
    ctx.dfree(d_xs, order * sizeof(double*));
    ctx.dfree(d_dxs, order * sizeof(double*));
    ctx.dfree(d_e, (order + 1) * (order + 1) * sizeof(double));
    ctx.dfree(d_c, (order + 1) * sizeof(double));
    ctx.dfree(d_dots, order * sizeof(double));
    ctx.dfree(d_state, 8 * sizeof(int));
    if (h_state) cudaFreeHost(h_state);
    if (h_c) cudaFreeHost(h_c);
}

void DiisRing::lay_out(const std::vector<int>& x, const std::vector<int>& dx, const double* weights) {
    int64_t off = 0;
    for (size_t k = 0; k < x.size(); k++) {
        Tensor& X = ctx.tensor(x[k]);
        piece_off.push_back(off);
        piece_len.push_back(X.total);
        // default weight 1 / (upper! lower!): ExcitationOperator::dot's 1 (T1) and 1/4 (T2);
        // plain (spatial) tensors take the plain dot
        double w = 1.0;
        if (weights) {
            w = weights[k];
        } else if (!X.plain()) {
            int nu = X.nout[0] + X.nout[1], nl = X.nin[0] + X.nin[1];
            for (int i = 2; i <= nu; i++) w /= i;
            for (int i = 2; i <= nl; i++) w /= i;
        }
        // times the number of spin-orbital arrangements each stored spin case stands for
        const int gs[4] = {X.nout[0], X.nout[1], X.nin[0], X.nin[1]};
        for (auto& sc : X.cases) {
            if (sc.blocks.empty()) continue;
            int64_t lo = sc.blocks.front().offset, hi = sc.blocks.back().offset + sc.blocks.back().size;
            double mult = 1;
            for (int g = 0; g < 4; g++) {
                double b = 1;
                for (int i = 0; i < sc.alpha[g]; i++) b = b * (gs[g] - i) / (i + 1);
                mult *= b;
            }
            segs.push_back({off + lo, hi - lo, w * mult});
        }
        off += X.total;
    }
    vec_len = off;
    if (order <= 1) {
        laid_out = true;
        return;
    }
    const size_t vb = (size_t)std::max<int64_t>(vec_len, 1) * sizeof(double);
    for (int i = 0; i < order; i++) {
        xs.push_back((double*)ctx.dmalloc(vb));
        dxs.push_back((double*)ctx.dmalloc(vb));
    }
    d_xs = (const double**)ctx.dmalloc(order * sizeof(double*));
    d_dxs = (const double**)ctx.dmalloc(order * sizeof(double*));
    d_e = (double*)ctx.dmalloc((order + 1) * (order + 1) * sizeof(double));
    d_c = (double*)ctx.dmalloc((order + 1) * sizeof(double));
    d_dots = (double*)ctx.dmalloc(order * sizeof(double));
    d_state = (int*)ctx.dmalloc(8 * sizeof(int));
    cudaStream_t s = ctx.stream;
    for (int i = 0; i < order; i++) {
        CCSD_CUDA(cudaMemsetAsync(xs[i], 0, vb, s));
        CCSD_CUDA(cudaMemsetAsync(dxs[i], 0, vb, s));
    }
    CCSD_CUDA(cudaMemcpyAsync(d_xs, xs.data(), order * sizeof(double*), cudaMemcpyHostToDevice, s));
    CCSD_CUDA(cudaMemcpyAsync(d_dxs, dxs.data(), order * sizeof(double*), cudaMemcpyHostToDevice, s));
    CCSD_CUDA(cudaMemsetAsync(d_e, 0, (order + 1) * (order + 1) * sizeof(double), s));
    CCSD_CUDA(cudaMemsetAsync(d_c, 0, (order + 1) * sizeof(double), s));
    int st[8] = {0, 0, start, 0, 0, 0, 0, 0};   // head, count, start counter, singular flag
    std::memcpy(h_state, st, sizeof(st));
    CCSD_CUDA(cudaMemcpyAsync(d_state, h_state, sizeof(st), cudaMemcpyHostToDevice, s));
    CCSD_CUDA(cudaStreamSynchronize(s));   // the pinned source is reused below
    laid_out = true;
}

void DiisRing::extrapolate(const std::vector<int>& x, const std::vector<int>& dx, const double* weights) {
    if (x.empty() || x.size() != dx.size()) throw Error(CCSD_ERR_ARG, "DIIS: x and dx need the same number of pieces");
    for (size_t k = 0; k < x.size(); k++) {
        Tensor& X = ctx.tensor(x[k]);
        Tensor& D = ctx.tensor(dx[k]);
        if (X.packed() || D.packed())
            throw Error(CCSD_ERR_UNSUPPORTED, "DIIS: packed tensors are not supported (pass unpacked amplitudes)");
        bool same = X.total == D.total && X.cases.size() == D.cases.size() && X.flags == D.flags;
        for (int g = 0; g < 2 && same; g++) same = X.nout[g] == D.nout[g] && X.nin[g] == D.nin[g];
        if (!same) throw Error(CCSD_ERR_ARG, "DIIS: x and dx piece " + std::to_string(k) + " differ in shape");
        if (laid_out && (k >= piece_len.size() || piece_len[k] != X.total))
            throw Error(CCSD_ERR_ARG, "DIIS: the pieces differ from the first call's");
    }
    if (!laid_out) lay_out(x, dx, weights);
    if (x.size() != piece_len.size()) throw Error(CCSD_ERR_ARG, "DIIS: the pieces differ from the first call's");
    if (order <= 1) return;   // diis.hpp:72: nothing to extrapolate with one vector
    cudaStream_t s = ctx.stream;
    CCSD_CUDA(cudaMemsetAsync(d_state + 3, 0, sizeof(int), s));
    kern::diis_advance(d_state, order, s);
    for (size_t k = 0; k < x.size(); k++)
        kern::diis_store_segment(d_state, d_xs, d_dxs, piece_off[k], ctx.tensor(x[k]).data, ctx.tensor(dx[k]).data,
                                 piece_len[k], s);
    CCSD_CUDA(cudaMemsetAsync(d_dots, 0, order * sizeof(double), s));
    for (auto& sg : segs) kern::diis_dots(d_state, d_dxs, order, sg.off, sg.len, sg.w, d_dots, s);
    kern::diis_solve(d_state, d_e, d_c, d_dots, order, s);
    // x = sum c_i x_i, dx = sum c_i dx_i (diis.hpp:205-226); with no extrapolation c is the
    // unit vector of the stored newest pair and x, dx keep their values
    for (size_t k = 0; k < x.size(); k++) {
        kern::lincomb_segment(ctx.tensor(x[k]).data, piece_len[k], d_xs, piece_off[k], d_c, order, s);
        kern::lincomb_segment(ctx.tensor(dx[k]).data, piece_len[k], d_dxs, piece_off[k], d_c, order, s);
    }
    kern::diis_damp(d_state, d_xs, order, vec_len, damping, s);
    CCSD_CUDA(cudaMemcpyAsync(h_state, d_state, 8 * sizeof(int), cudaMemcpyDeviceToHost, s));
    CCSD_CUDA(cudaMemcpyAsync(h_c, d_c, (order + 1) * sizeof(double), cudaMemcpyDeviceToHost, s));
    CCSD_CUDA(cudaStreamSynchronize(s));
    if (h_state[3]) throw Error(CCSD_ERR_SINGULAR, "DIIS: singular error matrix after the eps retry");
}

int DiisRing::coefficients(double* c_by_age) {
    if (order <= 1 || !laid_out) {
        if (c_by_age) c_by_age[0] = 1.0;
        return laid_out ? 1 : 0;
    }
    const int head = h_state[0], cnt = h_state[1];
    for (int i = 0; i < order; i++) {
        int slot = ((head - i) % order + order) % order;
        if (c_by_age) c_by_age[i] = i < cnt ? h_c[slot] : 0.0;
    }
    return cnt;
}

}  // namespace ccsd
