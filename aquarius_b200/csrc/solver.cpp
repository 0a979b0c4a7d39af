// CCSD solver: CCSD<U>::run / iterate (src/cc/ccsd.cxx:29-193), the iterative driver
// (src/util/iterative.hpp:126-188) and DIIS (src/convergence/diis.hpp:70-227), kept on
// the device so that one iteration is a fixed sequence of kernel launches (and can be
// captured as a CUDA graph).
#include <algorithm>
#include <map>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>

#include "expr.hpp"
#include "solver.hpp"

namespace ccsd {

namespace {

int mk(Context& c, const char* name, int o0, int o1, int i0, int i1, int flags = 0) {
    int nout[2] = {o0, o1}, nin[2] = {i0, i1};
    return c.create_tensor(name, nout, nin, flags);
}

}  // namespace

void options_default(ccsd_options* o) {
    o->conv_tol = 1e-9;
    o->max_iter = 50;
    o->diis_order = 5;
    o->diis_start = 1;
    o->diis_damping = 0.0;
    o->precision = CCSD_PREC_FP64;
    o->slices = 0;
    o->use_graph = 0;
    o->refine_tol = 0.0;
    o->autotune_de = 0.0;
}

// The slice autotuner's rule: smallest |dE| first while the running sum stays within the
// budget (a stable order keeps ties in statement order).
std::vector<int> slice_choice(const std::vector<double>& dE, double budget) {
    std::vector<int> order(dE.size()), drop(dE.size(), 0);
    for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
    // a change that is not finite never takes a slice away (sorted last)
    auto key = [&](int i) { return std::isfinite(dE[i]) ? std::fabs(dE[i]) : std::numeric_limits<double>::infinity(); };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key(a) < key(b); });
    double used = 0.0;
    for (int i : order) {
        const double d = std::fabs(dE[i]);
        if (!std::isfinite(d) || used + d > budget) break;
        used += d;
        drop[i] = 1;
    }
    return drop;
}

Solver::Solver(Context& c, const ccsd_hamiltonian& h, const ccsd_options& o) : ctx(c), H(h), opts(o) {
    // ccsd.cxx:37-48
    T1 = mk(ctx, "T(1)", 1, 0, 0, 1);
    T2 = mk(ctx, "T(2)", 2, 0, 0, 2);
    Z1 = mk(ctx, "Z(1)", 1, 0, 0, 1);
    Z2 = mk(ctx, "Z(2)", 2, 0, 0, 2);
    Tau = mk(ctx, "Tau", 2, 0, 0, 2);
    FME = mk(ctx, "F(me)", 0, 1, 1, 0);
    FMI = mk(ctx, "F(mi)", 0, 1, 0, 1);
    FAE = mk(ctx, "F(ae)", 1, 0, 1, 0);
    WMNIJ = mk(ctx, "W(mn,ij)", 0, 2, 0, 2);
    WMNEJ = mk(ctx, "W(mn,ej)", 0, 2, 1, 1);
    WAMIJ = mk(ctx, "W~(am,ij)", 1, 1, 0, 2);
    WAMEI = mk(ctx, "W~(am,ei)", 1, 1, 1, 1);
    setup_or_teardown();
}

// Closed-shell spin-adapted form (rhfccsd.cxx:44-110): plain spatial tensors, positions in
// [upper vrt, upper occ, lower vrt, lower occ] order (VAIJBSA and W(Am,Ie) therefore hold
// their [a, i, j, b] elements at [a, i, b, j]).
Solver::Solver(Context& c, const ccsd_rhf_hamiltonian& h, const ccsd_options& o)
    : ctx(c), HR(h), rhf(true), opts(o) {
    const int P = CCSD_TENSOR_PLAIN;
    T1 = mk(ctx, "T1", 1, 0, 0, 1, P);
    T2 = mk(ctx, "T2", 2, 0, 0, 2, P);
    Z1 = mk(ctx, "Z1", 1, 0, 0, 1, P);
    Z2 = mk(ctx, "Z2", 2, 0, 0, 2, P);
    Z2c = mk(ctx, "Z2 (copy)", 2, 0, 0, 2, P);
    Tau = mk(ctx, "Tau", 2, 0, 0, 2, P);
    T2SA = mk(ctx, "T2SA", 2, 0, 0, 2, P);
    TauSA = mk(ctx, "TauSA", 2, 0, 0, 2, P);
    VABIJSA = mk(ctx, "VABIJSA", 2, 0, 0, 2, P);
    VAIJBSA = mk(ctx, "VAIJBSA", 1, 1, 1, 1, P);
    FME = mk(ctx, "F(ME)", 0, 1, 1, 0, P);
    FMI = mk(ctx, "F(MI)", 0, 1, 0, 1, P);
    FAE = mk(ctx, "F(AE)", 1, 0, 1, 0, P);
    WMNIJ = mk(ctx, "W(Mn,Ij)", 0, 2, 0, 2, P);
    WMNIJc = mk(ctx, "W(Mn,Ij) (copy)", 0, 2, 0, 2, P);
    WMNEJ = mk(ctx, "W(Mn,Ej)", 0, 2, 1, 1, P);
    WAMIJ = mk(ctx, "W(Am,Ij)", 1, 1, 0, 2, P);
    WAMEI = mk(ctx, "W(Am,Ei)", 1, 1, 1, 1, P);
    WAMIE = mk(ctx, "W(Am,Ie)", 1, 1, 1, 1, P);
    setup_or_teardown();
}

// LambdaCCSD<U>::run (lambdaccsd.cxx:27-58): L(1), L(2) in the reference's layout (upper
// occupied, lower virtual), Z of the same shapes and the two G intermediates.  The Hbar
// blocks take the place of H, so the denominators come from the diagonals of its F(ae) and
// F(mi), as Denominator(Hbar) reads them (denominator.hpp:22-73).
Solver::Solver(Context& c, Solver& ccsd, const ccsd_hamiltonian& hbar, const ccsd_options& o)
    : ctx(c), H(hbar), opts(o), lambda(true), source(&ccsd) {
    if (ccsd.rhf || ccsd.lambda) throw Error(CCSD_ERR_ARG, "Lambda-CCSD needs a spin-orbital CCSD solver");
    if (&ccsd.ctx != &ctx) throw Error(CCSD_ERR_ARG, "the CCSD solver belongs to another context");
    struct Want {
        int h;
        int o0, o1, i0, i1;
        const char* name;
    };
    const Want want[] = {{H.fAI, 1, 0, 0, 1, "fAI"},     {H.fME, 0, 1, 1, 0, "fME"},     {H.fAE, 1, 0, 1, 0, "fAE"},
                         {H.fMI, 0, 1, 0, 1, "fMI"},     {H.VMNIJ, 0, 2, 0, 2, "VMNIJ"}, {H.VAMIJ, 1, 1, 0, 2, "VAMIJ"},
                         {H.VMNEJ, 0, 2, 1, 1, "VMNEJ"}, {H.VABIJ, 2, 0, 0, 2, "VABIJ"}, {H.VMNEF, 0, 2, 2, 0, "VMNEF"},
                         {H.VAMEI, 1, 1, 1, 1, "VAMEI"}, {H.VAMEF, 1, 1, 2, 0, "VAMEF"}, {H.VABEJ, 2, 0, 1, 1, "VABEJ"},
                         {H.VABEF, 2, 0, 2, 0, "VABEF"}};
    for (const Want& w : want) {
        if (!ctx.tensors.count(w.h)) throw Error(CCSD_ERR_ARG, std::string("Hbar block ") + w.name + " is not a tensor");
        const Tensor& t = ctx.tensor(w.h);
        if (t.plain() || t.nout[0] != w.o0 || t.nout[1] != w.o1 || t.nin[0] != w.i0 || t.nin[1] != w.i1)
            throw Error(CCSD_ERR_ARG, std::string("Hbar block ") + w.name + " has the wrong shape");
    }
    T1 = mk(ctx, "L(1)", 0, 1, 1, 0);
    T2 = mk(ctx, "L(2)", 0, 2, 2, 0);
    Z1 = mk(ctx, "Z(1)", 0, 1, 1, 0);
    Z2 = mk(ctx, "Z(2)", 0, 2, 2, 0);
    GIM = mk(ctx, "G(im)", 0, 1, 0, 1);
    GEA = mk(ctx, "G(ea)", 1, 0, 1, 0);
    source->lambda_users++;
    setup_or_teardown();
}

std::vector<int> Solver::constants() const {
    if (rhf)
        return {HR.fAI, HR.fAB, HR.fIJ, HR.VABCD, HR.VABCI, HR.VABIJ, HR.VAIBJ, HR.VAIJB, HR.VAIJK, HR.VIJKL,
                VABIJSA, VAIJBSA};
    return {H.fAI, H.fME, H.fAE, H.fMI, H.VMNIJ, H.VAMIJ, H.VMNEJ, H.VABIJ, H.VMNEF, H.VAMEI, H.VAMEF, H.VABEJ, H.VABEF};
}

std::vector<int> Solver::owned_tensors() const {
    std::vector<int> t = {T1, T2, Z1, Z2, Tau, FME, FMI, FAE, WMNIJ, WMNEJ, WAMIJ, WAMEI};
    if (rhf)
        for (int x : {T2SA, TauSA, VABIJSA, VAIJBSA, WAMIE, WMNIJc, Z2c}) t.push_back(x);
    if (WABEJ) t.push_back(WABEJ);
    for (int x : {GIM, GEA}) t.push_back(x);
    if (hbar_formed)
        for (int x : {HB.fAI, HB.fME, HB.fAE, HB.fMI, HB.VMNIJ, HB.VAMIJ, HB.VMNEJ, HB.VABIJ, HB.VMNEF, HB.VAMEI,
                      HB.VAMEF, HB.VABEJ, HB.VABEF})
            t.push_back(x);
    return t;
}

void Solver::setup() {
    if (opts.diis_damping != 0.0) throw Error(CCSD_ERR_UNSUPPORTED, "DIIS damping is not supported");
    if (opts.diis_order < 1 || opts.diis_order > 16) throw Error(CCSD_ERR_ARG, "diis_order must be in 1..16");
    if (opts.precision != CCSD_PREC_FP64 && opts.precision != CCSD_PREC_SPLIT && opts.precision != CCSD_PREC_SPLIT_I8)
        throw Error(CCSD_ERR_ARG, "bad precision");
    if (opts.slices != 0 &&
        !kern::slice_scheme_ok(opts.precision == CCSD_PREC_SPLIT_I8 ? kern::SLICE_INT8 : kern::SLICE_BF16, opts.slices))
        throw Error(CCSD_ERR_ARG, "slices must be 0 (default) or 3, 4 (BF16) / 3, 4, 5 (INT8)");
    mode_precision = opts.precision;
    mode_slices = opts.slices;
    use_mode();
    // constants: the H blocks never change, so their split slices can be cached
    for (int t : constants()) ctx.constant_tensors.push_back(t);
    constants_registered = true;

    if (ctx.host_only) {
        // planning query: account every allocation and plan one iteration, launch nothing
        ctx.plan_refine = (opts.precision == CCSD_PREC_SPLIT || opts.precision == CCSD_PREC_SPLIT_I8) &&
                          opts.refine_tol > 0;
        for (int sp = 0; sp < 2; sp++)
            for (int s = 0; s < 2; s++) den[sp][s] = (double*)alloc(std::max(ctx.spaces.total(sp, s), 1) * sizeof(double));
        build_diis();
        d_red = (double*)alloc(8 * sizeof(double));
        if (!lambda) record_tau(tau_plan);
        record_energy(energy_plan);
        if (rhf) record_iteration_rhf();
        else if (lambda) record_iteration_lambda();
        else record_iteration();
        ctx.upload(iter_plan);
        ctx.upload(tau_plan);
        ctx.upload(energy_plan);
        flops_per_iter = iter_plan.flops() + tau_plan.flops();
        if (std::getenv("CCSD_PLAN_DUMP")) {
            for (auto& g : iter_plan.gemms)
                std::fprintf(stderr, "%-48s M=%-8d N=%-8d K=%-8d %.3e flop a_k=%d a_m=%d b_k=%d b_n=%d var=%dx%d\n",
                             g.label.c_str(), g.M, g.N, g.K, g.flops(), g.a_kcontig, g.a_mcontig, g.b_kcontig,
                             g.b_ncontig, g.nvm, g.nvn);
        }
        return;
    }
    build_denominators();
    build_diis();
    d_red = (double*)ctx.dmalloc(8 * sizeof(double));
    CCSD_CUDA(cudaMemsetAsync(d_red, 0, 8 * sizeof(double), ctx.stream));
    h_red = nullptr;
    CCSD_CUDA(cudaMallocHost(&h_red, 8 * sizeof(double)));
    CCSD_CUDA(cudaMallocHost(&h_state, 8 * sizeof(int)));

    // ---- initial guess and MP2 (ccsd.cxx:50-62; rhfccsd.cxx:72-86) -------------
    {
        Plan init;
        Recorder r{&ctx, &init};
        TensorRef t1{&r, T1}, t2{&r, T2};
        if (lambda) {
            // L(0) = 1, L(1)[ia] = T(1)[ai], L(2)[ijab] = T(2)[abij]  (lambdaccsd.cxx:52-55)
            TensorRef s1{&r, source->T1}, s2{&r, source->T2};
            t1["ia"] = s1["ai"];
            t2["ijab"] = s2["abij"];
        } else if (rhf) {
            TensorRef fai{&r, HR.fAI}, vabij{&r, HR.VABIJ}, vaijb{&r, HR.VAIJB}, vaibj{&r, HR.VAIBJ};
            TensorRef sa{&r, VABIJSA}, sb{&r, VAIJBSA};
            t1["ai"] = fai["ai"];
            t2["abij"] = vabij["abij"];
            sa["abij"] = 2.0 * vabij["abij"];
            sa["abij"] -= vabij["abji"];
            sb["aibj"] = 2.0 * vaijb["aibj"];
            sb["aibj"] -= vaibj["aibj"];
        } else {
            TensorRef fai{&r, H.fAI}, vabij{&r, H.VABIJ};
            t1["ai"] = fai["ai"];
            t2["abij"] = vabij["abij"];
        }
        ctx.run(init);
        if (!lambda) {
            weight_tensor(T1);
            weight_tensor(T2);
        }
    }
    if (!lambda) record_tau(tau_plan);
    record_energy(energy_plan);
    if (!lambda) build_tau_blocks();
    build_update();
    launch_tau();
    CCSD_CUDA(cudaMemsetAsync(d_red, 0, sizeof(double), ctx.stream));
    ctx.run(energy_plan, nullptr, d_red + 0);
    CCSD_CUDA(cudaMemcpyAsync(h_red, d_red, sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
    CCSD_CUDA(cudaStreamSynchronize(ctx.stream));
    mp2 = h_red[0];
    energy = mp2;
    conv = std::numeric_limits<double>::max();

    if (rhf) record_iteration_rhf();
    else if (lambda) record_iteration_lambda();
    else record_iteration();
    ctx.upload(iter_plan);
    ctx.upload(tau_plan);
    ctx.upload(energy_plan);
    flops_per_iter = iter_plan.flops() + tau_plan.flops();
}

// A constructor that fails gives back what it took (tensors, device memory, plans) before
// the exception leaves it: the destructor does not run for a half-built object.
void Solver::setup_or_teardown() {
    try {
        setup();
    } catch (...) {
        teardown();
        throw;
    }
}

Solver::~Solver() { teardown(); }

void Solver::teardown() {
    if (source) source->lambda_users--;
    source = nullptr;
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    ctx.release(iter_plan);
    ctx.release(tau_plan);
    ctx.release(energy_plan);
    ctx.release(hbar_plan);
    const std::vector<int> cons = constants_registered ? constants() : std::vector<int>{};
    constants_registered = false;
    for (int t : owned_tensors())
        if (ctx.tensors.count(t)) ctx.destroy_tensor(t);
    for (auto p : owned) ctx.dfree(p.first, p.second);
    owned.clear();
    if (h_red) cudaFreeHost(h_red);
    if (h_state) cudaFreeHost(h_state);
    h_red = nullptr;
    h_state = nullptr;
    // one registration each: another solver on the same H keeps its own
    for (int t : cons) {
        auto it = std::find(ctx.constant_tensors.begin(), ctx.constant_tensors.end(), t);
        if (it != ctx.constant_tensors.end()) ctx.constant_tensors.erase(it);
    }
}

void* Solver::alloc(size_t bytes) {
    void* p = ctx.dmalloc(bytes);
    owned.push_back({p, bytes});
    return p;
}

// Denominator (denominator.hpp:50-73): d_a = -f_aa for virtuals, d_i = +f_ii for occupied,
// per spin, concatenated over irreps.  Read from the diagonal of the fAE / fMI blocks.
void Solver::build_denominators() {
    const Spaces& S = ctx.spaces;
    for (int sp = 0; sp < 2; sp++)
        for (int s = 0; s < 2; s++) {
            int n = S.total(sp, s);
            den[sp][s] = (double*)alloc(std::max(n, 1) * sizeof(double));
            std::vector<double> host(std::max(n, 1), 0.0);
            const int tf = rhf ? (sp == VRT ? HR.fAB : HR.fIJ) : (sp == VRT ? H.fAE : H.fMI);
            Tensor& F = ctx.tensor(tf);
            if (rhf && s == BETA) {   // spatial orbitals: one set of denominators
                CCSD_CUDA(cudaMemcpy(den[sp][s], host.data(), std::max(n, 1) * sizeof(double), cudaMemcpyHostToDevice));
                continue;
            }
            int alpha[4] = {0, 0, 0, 0};
            if (s == ALPHA) {
                if (sp == VRT) alpha[0] = alpha[2] = 1;
                else alpha[1] = alpha[3] = 1;
            }
            int cs = F.find_case(alpha);
            int off = 0;
            for (int h = 0; h < S.nirrep; h++) {
                int nh = S.n[sp][s][h];
                auto it = F.cases[cs].block_of.find(std::vector<int>{h, h});
                if (nh > 0 && it != F.cases[cs].block_of.end()) {
                    const Block& b = F.cases[cs].blocks[it->second];
                    std::vector<double> blk(b.size);
                    CCSD_CUDA(cudaMemcpy(blk.data(), F.data + b.offset, b.size * sizeof(double), cudaMemcpyDeviceToHost));
                    for (int x = 0; x < nh; x++) host[off + x] = (sp == VRT ? -1.0 : 1.0) * blk[x + (int64_t)x * nh];
                }
                off += nh;
            }
            CCSD_CUDA(cudaMemcpy(den[sp][s], host.data(), std::max(n, 1) * sizeof(double), cudaMemcpyHostToDevice));
        }
}

kern::WeightArgs Solver::weight_args(const Tensor& T, int cs, const Block& b) const {
    kern::WeightArgs w;
    w.ndim = T.ndim;
    w.total = b.size;
    for (int p = 0; p < T.ndim; p++) {
        int sp = group_space(T.group[p]);
        int s = T.cases[cs].spin[p];
        w.len[p] = b.len[p];
        w.d[p] = den[sp][s] + ctx.spaces.off[sp][s][b.irrep[p]];
    }
    return w;
}

void Solver::weight_tensor(int h) {
    Tensor& T = ctx.tensor(h);
    for (size_t c = 0; c < T.cases.size(); c++)
        for (auto& b : T.cases[c].blocks) {
            if (b.size == 0) continue;
            kern::weight_block(T.data + b.offset, weight_args(T, (int)c, b), 0.0, ctx.stream);
        }
}

// ---- recorded statements ---------------------------------------------------------

// Fused Tau (ccsd.cxx:123-124): tau_abij = t_abij + t_ai t_bj - t_aj t_bi, one pass per
// block of Tau with the T1 blocks each product term needs (spin and irrep of a match i, ...)
void Solver::build_tau_blocks() {
    Tensor& tau = ctx.tensor(Tau);
    Tensor& t2 = ctx.tensor(T2);
    Tensor& t1 = ctx.tensor(T1);
    auto t1_block = [&](int spin, int h) -> const Block* {
        int alpha[4] = {spin == ALPHA ? 1 : 0, 0, 0, spin == ALPHA ? 1 : 0};
        int cs = t1.find_case(alpha);
        if (cs < 0) return nullptr;
        auto it = t1.cases[cs].block_of.find(std::vector<int>{h, h});
        return it == t1.cases[cs].block_of.end() ? nullptr : &t1.cases[cs].blocks[it->second];
    };
    tau_blocks.clear();
    for (size_t c = 0; c < tau.cases.size(); c++) {
        const SpinCase& sc = tau.cases[c];
        for (size_t bi = 0; bi < sc.blocks.size(); bi++) {
            const Block& b = sc.blocks[bi];
            if (b.size == 0) continue;
            const Block& b2 = t2.cases[c].blocks[bi];
            kern::TauArgs a;
            a.tau = tau.data + b.offset;
            a.t2 = t2.data + b2.offset;
            for (int p = 0; p < 4; p++) a.len[p] = b.len[p];
            const int sa = sc.spin[0], sb = sc.spin[1], si = sc.spin[2], sj = sc.spin[3];
            const int ha = b.irrep[0], hb = b.irrep[1], hi = b.irrep[2], hj = b.irrep[3];
            if (sa == si && sb == sj && ha == hi && hb == hj) {
                const Block* x = t1_block(sa, ha);
                const Block* y = t1_block(sb, hb);
                if (x && y && x->size && y->size) {
                    a.t1ai = t1.data + x->offset;
                    a.t1bj = t1.data + y->offset;
                }
            }
            if (!rhf && sa == sj && sb == si && ha == hj && hb == hi) {
                const Block* x = t1_block(sa, ha);
                const Block* y = t1_block(sb, hb);
                if (x && y && x->size && y->size) {
                    a.t1aj = t1.data + x->offset;
                    a.t1bi = t1.data + y->offset;
                }
            }
            tau_blocks.push_back(a);
        }
    }
    // descriptors of the one-launch form
    std::vector<int64_t> cs;
    tau_chunks = 0;
    for (auto& a : tau_blocks) {
        cs.push_back(tau_chunks);
        tau_chunks += (a.len[0] * a.len[1] * a.len[2] * a.len[3] + kern::kBatchChunk - 1) / kern::kBatchChunk;
    }
    if (tau_blocks.size() > 1) {
        d_tau = (kern::TauArgs*)alloc(tau_blocks.size() * sizeof(kern::TauArgs));
        d_tau_cs = (int64_t*)alloc(cs.size() * sizeof(int64_t));
        ctx.stage_h2d(d_tau, tau_blocks.data(), tau_blocks.size() * sizeof(kern::TauArgs));
        ctx.stage_h2d(d_tau_cs, cs.data(), cs.size() * sizeof(int64_t));
    }
}

void Solver::launch_tau() {
    if (d_tau) kern::tau_batched(d_tau, d_tau_cs, (int)tau_blocks.size(), tau_chunks, ctx.stream);
    else
        for (auto& a : tau_blocks) kern::tau_block(a, ctx.stream);
}

// Z.weight(D); T += Z; conv = Z.norm(00) over every block of Z1 and Z2, one launch
void Solver::build_update() {
    std::vector<kern::UpdateDesc> descs;
    std::vector<int64_t> cs;
    upd_chunks = 0;
    for (int pair = 0; pair < 2; pair++) {
        Tensor& Z = ctx.tensor(pair == 0 ? Z1 : Z2);
        Tensor& T = ctx.tensor(pair == 0 ? T1 : T2);
        for (size_t c = 0; c < Z.cases.size(); c++)
            for (auto& b : Z.cases[c].blocks) {
                if (b.size == 0) continue;
                kern::UpdateDesc u;
                u.Z = Z.data + b.offset;
                u.T = T.data + b.offset;
                u.w = weight_args(Z, (int)c, b);
                descs.push_back(u);
                cs.push_back(upd_chunks);
                upd_chunks += (b.size + kern::kBatchChunk - 1) / kern::kBatchChunk;
            }
    }
    n_upd = (int)descs.size();
    d_upd = (kern::UpdateDesc*)alloc(std::max<size_t>(descs.size(), 1) * sizeof(kern::UpdateDesc));
    d_upd_cs = (int64_t*)alloc(std::max<size_t>(cs.size(), 1) * sizeof(int64_t));
    ctx.stage_h2d(d_upd, descs.data(), descs.size() * sizeof(kern::UpdateDesc));
    ctx.stage_h2d(d_upd_cs, cs.data(), cs.size() * sizeof(int64_t));
}

void Solver::record_tau(Plan& p) {
    Recorder r{&ctx, &p};
    TensorRef tau{&r, Tau}, t1{&r, T1}, t2{&r, T2};
    // ccsd.cxx:123-124; rhfccsd.cxx:237-238 (no antisymmetriser: plain tensors)
    tau["abij"] = t2["abij"];
    tau["abij"] += (rhf ? 1.0 : 0.5) * t1["ai"] * t1["bj"];
}

void Solver::record_energy(Plan& p) {
    if (rhf) {
        // energy = 2 <fAI|T1> + <VABIJSA|Tau>  (rhfccsd.cxx:320)
        Plan a = plan_dot(ctx, HR.fAI, "ai", T1, "ai");
        for (auto& d : a.dots) d.alpha *= 2.0;
        Plan b = plan_dot(ctx, VABIJSA, "abij", Tau, "abij");
        p.append(std::move(a));
        p.append(std::move(b));
        return;
    }
    if (lambda) {
        // energy = 1/4 <WMNEF|L(2)>  (lambdaccsd.cxx:129)
        Plan b = plan_dot(ctx, H.VMNEF, "ijab", T2, "ijab");
        for (auto& d : b.dots) d.alpha *= 0.25;
        p.append(std::move(b));
        return;
    }
    // energy = <fAI|T1> + 1/4 <VABIJ|Tau> over full spin-orbital ranges (ccsd.cxx:189)
    Plan a = plan_dot(ctx, H.fAI, "ai", T1, "ai");
    Plan b = plan_dot(ctx, H.VABIJ, "abij", Tau, "abij");
    for (auto& d : b.dots) d.alpha *= 0.25;
    p.append(std::move(a));
    p.append(std::move(b));
}

void Solver::record_iteration() {
    Plan& p = iter_plan;
    std::vector<std::function<Plan()>> jobs;
    Recorder r{&ctx, &p, &jobs};
    TensorRef fAI{&r, H.fAI}, fME{&r, H.fME}, fAE{&r, H.fAE}, fMI{&r, H.fMI};
    TensorRef VABIJ{&r, H.VABIJ}, VMNEF{&r, H.VMNEF}, VAMEF{&r, H.VAMEF}, VABEJ{&r, H.VABEJ}, VABEF{&r, H.VABEF};
    TensorRef VMNIJ{&r, H.VMNIJ}, VMNEJ{&r, H.VMNEJ}, VAMIJ{&r, H.VAMIJ}, VAMEI{&r, H.VAMEI};
    TensorRef T1r{&r, T1}, T2r{&r, T2}, Z1r{&r, Z1}, Z2r{&r, Z2}, Taur{&r, Tau};
    TensorRef FMEr{&r, FME}, FAEr{&r, FAE}, FMIr{&r, FMI};
    TensorRef WMNIJr{&r, WMNIJ}, WMNEJr{&r, WMNEJ}, WAMIJr{&r, WAMIJ}, WAMEIr{&r, WAMEI};

    // ccsd.cxx:123-124 (Tau = T2 + 1/2 P(ab)P(ij) t_ai t_bj) is formed by the fused Tau
    // kernel before this plan runs (launch_tau); tau_plan keeps the statement's flop count

    // intermediates, ccsd.cxx:130-157
    FMEr["me"] = fME["me"];
    FMEr["me"] += VMNEF["mnef"] * T1r["fn"];

    FMIr["mi"] = fMI["mi"];
    FMIr["mi"] += 0.5 * VMNEF["mnef"] * T2r["efin"];
    FMIr["mi"] += FMEr["me"] * T1r["ei"];
    FMIr["mi"] += VMNEJ["nmfi"] * T1r["fn"];

    FAEr["ae"] = fAE["ae"];
    FAEr["ae"] -= 0.5 * VMNEF["mnef"] * T2r["afmn"];
    FAEr["ae"] -= FMEr["me"] * T1r["am"];
    FAEr["ae"] += VAMEF["amef"] * T1r["fm"];

    WMNIJr["mnij"] = VMNIJ["mnij"];
    WMNIJr["mnij"] += 0.5 * VMNEF["mnef"] * Taur["efij"];
    WMNIJr["mnij"] += VMNEJ["mnej"] * T1r["ei"];

    WMNEJr["mnej"] = VMNEJ["mnej"];
    WMNEJr["mnej"] += VMNEF["mnef"] * T1r["fj"];

    WAMIJr["amij"] = VAMIJ["amij"];
    WAMIJr["amij"] += 0.5 * VAMEF["amef"] * Taur["efij"];
    WAMIJr["amij"] += VAMEI["amej"] * T1r["ei"];

    WAMEIr["amei"] = VAMEI["amei"];
    WAMEIr["amei"] += 0.5 * VMNEF["mnef"] * T2r["afni"];
    WAMEIr["amei"] += VAMEF["amef"] * T1r["fi"];
    WAMEIr["amei"] -= WMNEJr["nmei"] * T1r["an"];

    // residual, ccsd.cxx:165-180
    Z1r["ai"] = fAI["ai"];
    Z1r["ai"] += fAE["ae"] * T1r["ei"];
    Z1r["ai"] -= FMIr["mi"] * T1r["am"];
    Z1r["ai"] -= VAMEI["amei"] * T1r["em"];
    Z1r["ai"] += FMEr["me"] * T2r["aeim"];
    Z1r["ai"] += 0.5 * VAMEF["amef"] * Taur["efim"];
    Z1r["ai"] -= 0.5 * WMNEJr["mnei"] * T2r["eamn"];

    Z2r["abij"] = VABIJ["abij"];
    Z2r["abij"] += VABEJ["abej"] * T1r["ei"];
    Z2r["abij"] -= WAMIJr["amij"] * T1r["bm"];
    Z2r["abij"] += FAEr["ae"] * T2r["ebij"];
    Z2r["abij"] -= FMIr["mi"] * T2r["abmj"];
    Z2r["abij"] += 0.5 * VABEF["abef"] * Taur["efij"];
    Z2r["abij"] += 0.5 * WMNIJr["mnij"] * Taur["abmn"];
    Z2r["abij"] += WAMEIr["amei"] * T2r["ebjm"];
    run_deferred(r);
}

// RHFCCSD<U>::iterate (rhfccsd.cxx:237-306) over plain tensors.  Index strings follow
// each tensor's stored position order; for VAIJB, VAIJBSA and W(Am,Ie), whose elements
// [a, i, j, b] sit at positions [a, i, b, j], the reference's "amie" reads "amei".
// The two in-place symmetrisations (W(Mn,Ij) += W(Mn,Ij)[nmji], Z2 += Z2[baji]) are
// accumulated in a second tensor and folded once.
void Solver::record_iteration_rhf() {
    Plan& p = iter_plan;
    std::vector<std::function<Plan()>> jobs;
    Recorder r{&ctx, &p, &jobs};
    TensorRef fAI{&r, HR.fAI}, fAB{&r, HR.fAB}, fIJ{&r, HR.fIJ};
    TensorRef VABCD{&r, HR.VABCD}, VABCI{&r, HR.VABCI}, VABIJ{&r, HR.VABIJ}, VAIBJ{&r, HR.VAIBJ};
    TensorRef VAIJB{&r, HR.VAIJB}, VAIJK{&r, HR.VAIJK}, VIJKL{&r, HR.VIJKL};
    TensorRef VABIJSAr{&r, VABIJSA}, VAIJBSAr{&r, VAIJBSA};
    TensorRef T1r{&r, T1}, T2r{&r, T2}, Z1r{&r, Z1}, Z2r{&r, Z2}, Z2cr{&r, Z2c}, Taur{&r, Tau};
    TensorRef T2SAr{&r, T2SA}, TauSAr{&r, TauSA};
    TensorRef FMEr{&r, FME}, FAEr{&r, FAE}, FMIr{&r, FMI};
    TensorRef WMNIJr{&r, WMNIJ}, WMNIJcr{&r, WMNIJc}, WMNEJr{&r, WMNEJ}, WAMIJr{&r, WAMIJ};
    TensorRef WAMEIr{&r, WAMEI}, WAMIEr{&r, WAMIE};

    // Tau = T2 + t_ai t_bj comes from the fused Tau kernel before this plan runs
    TauSAr["abij"] = 2.0 * Taur["abij"];
    TauSAr["abij"] -= Taur["abji"];
    T2SAr["abij"] = 2.0 * T2r["abij"];
    T2SAr["abij"] -= T2r["abji"];

    // intermediates (rhfccsd.cxx:249-288)
    FMEr["me"] = fAI["em"];
    FMEr["me"] += VABIJSAr["efmn"] * T1r["fn"];

    FMIr["mi"] = fIJ["mi"];
    FMIr["mi"] += VABIJSAr["efmn"] * T2r["efin"];
    FMIr["mi"] += FMEr["me"] * T1r["ei"];
    FMIr["mi"] += 2.0 * VAIJK["finm"] * T1r["fn"];
    FMIr["mi"] -= VAIJK["fimn"] * T1r["fn"];

    FAEr["ae"] = fAB["ae"];
    FAEr["ae"] -= VABIJSAr["efmn"] * T2r["afmn"];
    FAEr["ae"] -= FMEr["me"] * T1r["am"];
    FAEr["ae"] += 2.0 * VABCI["efam"] * T1r["fm"];
    FAEr["ae"] -= VABCI["feam"] * T1r["fm"];

    WMNIJcr["mnij"] = 0.5 * VIJKL["mnij"];
    WMNIJcr["mnij"] += 0.5 * VABIJ["efmn"] * Taur["efij"];
    WMNIJcr["mnij"] += VAIJK["ejmn"] * T1r["ei"];
    WMNIJr["mnij"] = WMNIJcr["mnij"];
    WMNIJr["mnij"] += WMNIJcr["nmji"];

    WMNEJr["mnej"] = VAIJK["ejmn"];
    WMNEJr["mnej"] += VABIJ["efmn"] * T1r["fj"];

    WAMIJr["amij"] = VAIJK["amij"];
    WAMIJr["amij"] += VABCI["efam"] * Taur["efij"];
    WAMIJr["amij"] += VAIBJ["amej"] * T1r["ei"];
    WAMIJr["amij"] += VAIJB["amei"] * T1r["ej"];

    WAMIEr["amei"] = VAIJBSAr["amei"];
    WAMIEr["amei"] += 0.5 * VABIJSAr["efmn"] * T2SAr["afin"];
    WAMIEr["amei"] += 2.0 * VABCI["feam"] * T1r["fi"];
    WAMIEr["amei"] -= VABCI["efam"] * T1r["fi"];
    WAMIEr["amei"] -= 2.0 * WMNEJr["mnei"] * T1r["an"];
    WAMIEr["amei"] += WMNEJr["nmei"] * T1r["an"];

    WAMEIr["amei"] = VAIBJ["amei"];
    WAMEIr["amei"] -= 0.5 * VABIJ["efnm"] * T2r["afni"];
    WAMEIr["amei"] += VABCI["efam"] * T1r["fi"];
    WAMEIr["amei"] -= WMNEJr["nmei"] * T1r["an"];

    // residual (rhfccsd.cxx:295-316)
    Z1r["ai"] = fAI["ai"];
    Z1r["ai"] += fAB["ae"] * T1r["ei"];
    Z1r["ai"] -= FMIr["mi"] * T1r["am"];
    Z1r["ai"] += VAIJBSAr["amei"] * T1r["em"];
    Z1r["ai"] += FMEr["me"] * T2SAr["aeim"];
    Z1r["ai"] += VABCI["efam"] * TauSAr["efim"];
    Z1r["ai"] -= WMNEJr["mnei"] * T2SAr["eamn"];

    Z2cr["abij"] = 0.5 * VABIJ["abij"];
    Z2cr["abij"] += VABCI["abej"] * T1r["ei"];
    Z2cr["abij"] -= WAMIJr["amij"] * T1r["bm"];
    Z2cr["abij"] += FAEr["ae"] * T2r["ebij"];
    Z2cr["abij"] -= FMIr["mi"] * T2r["abmj"];
    Z2cr["abij"] += 0.5 * VABCD["abef"] * Taur["efij"];
    Z2cr["abij"] += 0.5 * WMNIJr["mnij"] * Taur["abmn"];
    Z2cr["abij"] += 0.5 * WAMIEr["amei"] * T2SAr["ebmj"];
    Z2cr["abij"] -= 0.5 * WAMEIr["amei"] * T2r["ebjm"];
    Z2cr["abij"] -= WAMEIr["amej"] * T2r["ebim"];
    Z2r["abij"] = Z2cr["abij"];
    Z2r["abij"] += Z2cr["baji"];
    run_deferred(r);
}

// "Form Hbar" of RHFCCSD<U>::run (rhfccsd.cxx:110-186): the intermediates again, with the
// terms the iteration leaves out, and W(Ab,Ej), from the converged amplitudes.  Index
// strings as in record_iteration_rhf (W(Am,Ie), VAIJB: "amie" reads "amei").
void Solver::hbar_rhf() {
    if (!rhf) throw Error(CCSD_ERR_UNSUPPORTED, "Hbar intermediates are formed for the closed-shell solver");
    if (!WABEJ) {
        WABEJ = mk(ctx, "W(Ab,Ej)", 2, 0, 1, 1, CCSD_TENSOR_PLAIN);
        Plan& p = hbar_plan;
        std::vector<std::function<Plan()>> jobs;
        Recorder r{&ctx, &p, &jobs};
        TensorRef fAI{&r, HR.fAI}, fAB{&r, HR.fAB}, fIJ{&r, HR.fIJ};
        TensorRef VABCD{&r, HR.VABCD}, VABCI{&r, HR.VABCI}, VABIJ{&r, HR.VABIJ}, VAIBJ{&r, HR.VAIBJ};
        TensorRef VAIJB{&r, HR.VAIJB}, VAIJK{&r, HR.VAIJK}, VIJKL{&r, HR.VIJKL};
        TensorRef VABIJSAr{&r, VABIJSA}, VAIJBSAr{&r, VAIJBSA};
        TensorRef T1r{&r, T1}, T2r{&r, T2}, Taur{&r, Tau}, T2SAr{&r, T2SA};
        TensorRef FMEr{&r, FME}, FAEr{&r, FAE}, FMIr{&r, FMI};
        TensorRef WMNIJr{&r, WMNIJ}, WMNIJcr{&r, WMNIJc}, WMNEJr{&r, WMNEJ}, WAMIJr{&r, WAMIJ};
        TensorRef WAMEIr{&r, WAMEI}, WAMIEr{&r, WAMIE}, WABEJr{&r, WABEJ};

        Taur["abij"] = T2r["abij"];
        Taur["abij"] += T1r["ai"] * T1r["bj"];
        T2SAr["abij"] = 2.0 * T2r["abij"];
        T2SAr["abij"] -= T2r["abji"];

        FMEr["me"] = fAI["em"];
        FMEr["me"] += VABIJSAr["efmn"] * T1r["fn"];

        FMIr["mi"] = fIJ["mi"];
        FMIr["mi"] += VABIJSAr["efmn"] * T2r["efin"];
        FMIr["mi"] += FMEr["me"] * T1r["ei"];
        FMIr["mi"] += 2.0 * VAIJK["finm"] * T1r["fn"];
        FMIr["mi"] -= VAIJK["fimn"] * T1r["fn"];

        FAEr["ae"] = fAB["ae"];
        FAEr["ae"] -= VABIJSAr["efmn"] * T2r["afmn"];
        FAEr["ae"] -= FMEr["me"] * T1r["am"];
        FAEr["ae"] += 2.0 * VABCI["efam"] * T1r["fm"];
        FAEr["ae"] -= VABCI["feam"] * T1r["fm"];

        WMNIJcr["mnij"] = 0.5 * VIJKL["mnij"];
        WMNIJcr["mnij"] += 0.5 * VABIJ["efmn"] * Taur["efij"];
        WMNIJcr["mnij"] += VAIJK["ejmn"] * T1r["ei"];
        WMNIJr["mnij"] = WMNIJcr["mnij"];
        WMNIJr["mnij"] += WMNIJcr["nmji"];

        WMNEJr["mnej"] = VAIJK["ejmn"];
        WMNEJr["mnej"] += VABIJ["efmn"] * T1r["fj"];

        WAMIJr["amij"] = VAIJK["amij"];
        WAMIJr["amij"] += VABCI["efam"] * Taur["efij"];
        WAMIJr["amij"] += VAIBJ["amej"] * T1r["ei"];
        WAMIJr["amij"] += VAIJB["amei"] * T1r["ej"];
        WAMIJr["amij"] -= WMNIJr["nmij"] * T1r["an"];
        WAMIJr["amij"] += WMNEJr["nmej"] * T2SAr["aein"];
        WAMIJr["amij"] -= WMNEJr["mnej"] * T2r["aein"];
        WAMIJr["amij"] -= WMNEJr["mnei"] * T2r["aenj"];
        WAMIJr["amij"] += FMEr["me"] * T2r["aeij"];

        WAMIEr["amei"] = VAIJBSAr["amei"];
        WAMIEr["amei"] += VABIJSAr["efmn"] * T2SAr["afin"];
        WAMIEr["amei"] += 2.0 * VABCI["feam"] * T1r["fi"];
        WAMIEr["amei"] -= VABCI["efam"] * T1r["fi"];

        WAMEIr["amei"] = VAIBJ["amei"];
        WAMEIr["amei"] -= VABIJ["efnm"] * T2r["afni"];
        WAMEIr["amei"] += VABCI["efam"] * T1r["fi"];

        WABEJr["abej"] = VABCI["abej"];
        WABEJr["abej"] += WMNEJr["mnej"] * Taur["abmn"];
        WABEJr["abej"] -= 0.5 * WAMIEr["bmej"] * T1r["am"];
        WABEJr["abej"] -= 0.5 * WAMEIr["bmej"] * T1r["am"];
        WABEJr["abej"] -= WAMEIr["amej"] * T1r["bm"];
        WABEJr["abej"] += VABCD["abef"] * T1r["fj"];
        WABEJr["abej"] += VABCI["efam"] * T2SAr["fbmj"];
        WABEJr["abej"] -= VABCI["feam"] * T2r["fbmj"];
        WABEJr["abej"] -= VABCI["febm"] * T2r["afmj"];
        WABEJr["abej"] -= FMEr["me"] * T2r["abmj"];

        WAMIEr["amei"] -= 2.0 * WMNEJr["mnei"] * T1r["an"];
        WAMIEr["amei"] += WMNEJr["nmei"] * T1r["an"];

        WAMEIr["amei"] -= WMNEJr["nmei"] * T1r["an"];
        run_deferred(r);
        ctx.upload(hbar_plan);
    }
    if (ctx.host_only) return;
    use_mode();
    ctx.run(hbar_plan);
    CCSD_CUDA(cudaStreamSynchronize(ctx.stream));
}

// LambdaCCSD<U>::iterate (lambdaccsd.cxx:60-133): the G intermediates and the residual,
// statement for statement; weight, update, energy, norm and DIIS are the shared driver's.
void Solver::record_iteration_lambda() {
    Plan& p = iter_plan;
    std::vector<std::function<Plan()>> jobs;
    Recorder r{&ctx, &p, &jobs};
    TensorRef FME{&r, H.fME}, FAE{&r, H.fAE}, FMI{&r, H.fMI}, WMNEF{&r, H.VMNEF}, WAMEF{&r, H.VAMEF};
    TensorRef WABEJ{&r, H.VABEJ}, WABEF{&r, H.VABEF}, WMNIJ{&r, H.VMNIJ}, WMNEJ{&r, H.VMNEJ};
    TensorRef WAMIJ{&r, H.VAMIJ}, WAMEI{&r, H.VAMEI};
    TensorRef T2r{&r, source->T2}, L1{&r, T1}, L2{&r, T2}, Z1r{&r, Z1}, Z2r{&r, Z2};
    TensorRef GIMr{&r, GIM}, GEAr{&r, GEA};

    GIMr["mn"] = 0.5 * T2r["efno"] * L2["moef"];
    GEAr["ef"] = -0.5 * T2r["egmn"] * L2["mnfg"];

    Z1r["ia"] = FME["ia"];
    Z1r["ia"] += FAE["ea"] * L1["ie"];
    Z1r["ia"] -= FMI["im"] * L1["ma"];
    Z1r["ia"] -= WAMEI["eiam"] * L1["me"];
    Z1r["ia"] += 0.5 * WABEJ["efam"] * L2["imef"];
    Z1r["ia"] -= 0.5 * WAMIJ["eimn"] * L2["mnea"];
    Z1r["ia"] -= WMNEJ["inam"] * GIMr["mn"];
    Z1r["ia"] -= WAMEF["fiea"] * GEAr["ef"];

    Z2r["ijab"] = WMNEF["ijab"];
    Z2r["ijab"] += FME["ia"] * L1["jb"];
    Z2r["ijab"] += WAMEF["ejab"] * L1["ie"];
    Z2r["ijab"] -= WMNEJ["ijam"] * L1["mb"];
    Z2r["ijab"] += FAE["ea"] * L2["ijeb"];
    Z2r["ijab"] -= FMI["im"] * L2["mjab"];
    Z2r["ijab"] += 0.5 * WABEF["efab"] * L2["ijef"];
    Z2r["ijab"] += 0.5 * WMNIJ["ijmn"] * L2["mnab"];
    Z2r["ijab"] += WAMEI["eiam"] * L2["mjbe"];
    Z2r["ijab"] -= WMNEF["mjab"] * GIMr["im"];
    Z2r["ijab"] += WMNEF["ijeb"] * GEAr["ea"];
    run_deferred(r);
}

// The "Hbar" product of CCSD::run (ccsd.cxx:83-86): STTwoElectronOperator(H, T, isHbar =
// true) for T truncated at doubles (st2eoperator.hpp:59-130), statement for statement and
// in the reference's order (later statements read blocks that earlier ones updated).  The
// blocks start as copies of H; the occupied-virtual Fock block is assigned by the first
// statement (the bare f_me does not survive) and f(ai), <ab||ij> stay zero.
void Solver::record_hbar_so() {
    Plan& p = hbar_plan;
    std::vector<std::function<Plan()>> jobs;
    Recorder r{&ctx, &p, &jobs};
    TensorRef fME{&r, H.fME}, fAE{&r, H.fAE}, fMI{&r, H.fMI};
    TensorRef VMNIJ{&r, H.VMNIJ}, VAMIJ{&r, H.VAMIJ}, VMNEJ{&r, H.VMNEJ}, VMNEF{&r, H.VMNEF};
    TensorRef VAMEI{&r, H.VAMEI}, VAMEF{&r, H.VAMEF}, VABEJ{&r, H.VABEJ}, VABEF{&r, H.VABEF};
    TensorRef T1r{&r, T1}, T2r{&r, T2}, Taur{&r, Tau};
    TensorRef ia{&r, HB.fME}, ij{&r, HB.fMI}, ab{&r, HB.fAE}, ijkl{&r, HB.VMNIJ}, aijk{&r, HB.VAMIJ};
    TensorRef ijak{&r, HB.VMNEJ}, ijab{&r, HB.VMNEF}, aibj{&r, HB.VAMEI}, aibc{&r, HB.VAMEF};
    TensorRef abci{&r, HB.VABEJ}, abcd{&r, HB.VABEF};

    // TwoElectronOperator(name, X): the blocks of H
    ij["mi"] = fMI["mi"];
    ab["ae"] = fAE["ae"];
    ijkl["mnij"] = VMNIJ["mnij"];
    aijk["amij"] = VAMIJ["amij"];
    ijak["mnej"] = VMNEJ["mnej"];
    ijab["mnef"] = VMNEF["mnef"];
    aibj["amei"] = VAMEI["amei"];
    aibc["amef"] = VAMEF["amef"];
    abci["abej"] = VABEJ["abej"];
    abcd["abef"] = VABEF["abef"];

    // Tau = T2 + 1/2 P(ab)P(ij) t_ai t_bj from the current amplitudes
    Taur["abij"] = T2r["abij"];
    Taur["abij"] += 0.5 * T1r["ai"] * T1r["bj"];

    ia["me"] = ijab["mnef"] * T1r["fn"];

    ij["mi"] += 0.5 * ijab["nmef"] * T2r["efni"];
    ij["mi"] += ia["me"] * T1r["ei"];
    ij["mi"] += ijak["nmfi"] * T1r["fn"];

    ijkl["mnij"] += 0.5 * ijab["mnef"] * Taur["efij"];
    ijkl["mnij"] += ijak["nmei"] * T1r["ej"];

    ijak["mnej"] += ijab["mnef"] * T1r["fj"];

    ab["ae"] -= 0.5 * ijab["mnfe"] * T2r["famn"];
    ab["ae"] -= ia["me"] * T1r["am"];
    ab["ae"] += aibc["anef"] * T1r["fn"];

    aijk["amij"] += 0.5 * aibc["amef"] * Taur["efij"];
    aijk["amij"] += aibj["amej"] * T1r["ei"];

    aibj["amei"] -= 0.5 * ijab["mnef"] * T2r["afin"];
    aibj["amei"] -= aibc["amfe"] * T1r["fi"];
    aibj["amei"] -= ijak["nmei"] * T1r["an"];

    aijk["amij"] += ijak["nmej"] * T2r["aein"];
    aijk["amij"] -= ijkl["nmij"] * T1r["an"];
    aijk["amij"] += ia["me"] * T2r["aeij"];

    aibj["amei"] -= 0.5 * ijab["mnef"] * T2r["afin"];
    aibj["amei"] += 0.5 * ijak["nmei"] * T1r["an"];

    abci["abej"] += 0.5 * ijak["mnej"] * T2r["abmn"];
    abci["abej"] -= aibj["amej"] * T1r["bm"];
    abci["abej"] += aibc["amef"] * T2r["fbmj"];
    abci["abej"] += abcd["abef"] * T1r["fj"];
    abci["abej"] -= ia["me"] * T2r["abmj"];

    aibj["amei"] -= 0.5 * ijak["nmei"] * T1r["an"];

    abcd["abef"] += 0.5 * ijab["mnef"] * Taur["abmn"];
    abcd["abef"] -= aibc["amef"] * T1r["bm"];

    aibc["amef"] -= ijab["nmef"] * T1r["an"];
    run_deferred(r);
}

void Solver::hbar_so() {
    if (rhf || lambda) throw Error(CCSD_ERR_UNSUPPORTED, "the spin-orbital Hbar is formed by a spin-orbital CCSD solver");
    if (lambda_users > 0)
        throw Error(CCSD_ERR_ARG, "a Lambda solver reads this Hbar: destroy it before forming Hbar again");
    if (ctx.tensor(H.VABEF).packed())
        throw Error(CCSD_ERR_UNSUPPORTED, "the spin-orbital Hbar needs <ab||ef> stored unpacked (pack_vvvv = 0)");
    if (!hbar_formed) {
        HB.fAI = mk(ctx, "Hbar f(ai)", 1, 0, 0, 1);
        HB.fME = mk(ctx, "Hbar F(me)", 0, 1, 1, 0);
        HB.fAE = mk(ctx, "Hbar F(ae)", 1, 0, 1, 0);
        HB.fMI = mk(ctx, "Hbar F(mi)", 0, 1, 0, 1);
        HB.VMNIJ = mk(ctx, "Hbar W(mn,ij)", 0, 2, 0, 2);
        HB.VAMIJ = mk(ctx, "Hbar W(am,ij)", 1, 1, 0, 2);
        HB.VMNEJ = mk(ctx, "Hbar W(mn,ej)", 0, 2, 1, 1);
        HB.VABIJ = mk(ctx, "Hbar W(ab,ij)", 2, 0, 0, 2);
        HB.VMNEF = mk(ctx, "Hbar W(mn,ef)", 0, 2, 2, 0);
        HB.VAMEI = mk(ctx, "Hbar W(am,ei)", 1, 1, 1, 1);
        HB.VAMEF = mk(ctx, "Hbar W(am,ef)", 1, 1, 2, 0);
        HB.VABEJ = mk(ctx, "Hbar W(ab,ej)", 2, 0, 1, 1);
        HB.VABEF = mk(ctx, "Hbar W(ab,ef)", 2, 0, 2, 0);
        try {
            record_hbar_so();
            ctx.upload(hbar_plan);
        } catch (...) {
            // leave no half-recorded plan and no blocks behind: a later call starts afresh
            ctx.release(hbar_plan);
            hbar_plan = Plan();
            for (int t : {HB.fAI, HB.fME, HB.fAE, HB.fMI, HB.VMNIJ, HB.VAMIJ, HB.VMNEJ, HB.VABIJ, HB.VMNEF, HB.VAMEI,
                          HB.VAMEF, HB.VABEJ, HB.VABEF})
                if (ctx.tensors.count(t)) ctx.destroy_tensor(t);
            HB = ccsd_hamiltonian{};
            throw;
        }
        hbar_formed = true;
    }
    if (ctx.host_only) return;
    use_mode();
    ctx.run(hbar_plan);
    CCSD_CUDA(cudaStreamSynchronize(ctx.stream));
}

// ---- DIIS state ----------------------------------------------------------------------

void Solver::build_diis() {
    const int n = opts.diis_order;
    Tensor& t1 = ctx.tensor(T1);
    Tensor& t2 = ctx.tensor(T2);
    vec_len = t1.total + t2.total;
    // segments with the ExcitationOperator::dot weights (1 for T1, 1/4 for T2) times the
    // number of spin-orbital arrangements a stored spin case stands for
    // (binomial factors, spinorbital_tensor.cxx:1084-1088)
    auto add_segments = [&](Tensor& T, int64_t base, double w) {
        for (auto& sc : T.cases) {
            if (sc.blocks.empty()) continue;
            int64_t lo = sc.blocks.front().offset, hi = sc.blocks.back().offset + sc.blocks.back().size;
            double mult = 1;
            const int gs[4] = {T.nout[0], T.nout[1], T.nin[0], T.nin[1]};
            for (int g = 0; g < 4; g++) {
                double b = 1;
                for (int k = 0; k < sc.alpha[g]; k++) b = b * (gs[g] - k) / (k + 1);
                mult *= b;
            }
            segs.push_back({base + lo, hi - lo, w * mult});
        }
    };
    add_segments(t1, 0, 1.0);
    // (the RHF DIIS takes the plain dot of the spatial amplitudes, rhfccsd.cxx:102)
    add_segments(t2, t1.total, rhf ? 1.0 : 0.25);
    if (n <= 1) return;
    xs.resize(n);
    dxs.resize(n);
    for (int i = 0; i < n; i++) {
        xs[i] = (double*)alloc(vec_len * sizeof(double));
        dxs[i] = (double*)alloc(vec_len * sizeof(double));
    }
    d_xs = (const double**)alloc(n * sizeof(double*));
    d_dxs = (const double**)alloc(n * sizeof(double*));
    d_e = (double*)alloc((n + 1) * (n + 1) * sizeof(double));
    d_c = (double*)alloc((n + 1) * sizeof(double));
    d_dots = (double*)alloc(n * sizeof(double));
    d_state = (int*)alloc(8 * sizeof(int));
    if (ctx.host_only) return;
    for (int i = 0; i < n; i++) {
        CCSD_CUDA(cudaMemsetAsync(xs[i], 0, vec_len * sizeof(double), ctx.stream));
        CCSD_CUDA(cudaMemsetAsync(dxs[i], 0, vec_len * sizeof(double), ctx.stream));
    }
    CCSD_CUDA(cudaMemcpy(d_xs, xs.data(), n * sizeof(double*), cudaMemcpyHostToDevice));
    CCSD_CUDA(cudaMemcpy(d_dxs, dxs.data(), n * sizeof(double*), cudaMemcpyHostToDevice));
    CCSD_CUDA(cudaMemsetAsync(d_e, 0, (n + 1) * (n + 1) * sizeof(double), ctx.stream));
    CCSD_CUDA(cudaMemsetAsync(d_c, 0, (n + 1) * sizeof(double), ctx.stream));
    int st[8] = {0, 0, opts.diis_start, 0, 0, 0, 0, 0};   // head, count, start, status
    CCSD_CUDA(cudaMemcpy(d_state, st, sizeof(st), cudaMemcpyHostToDevice));
}

// ---- one iteration ---------------------------------------------------------------------

void Solver::launch_iteration() {
    cudaStream_t s = ctx.stream;
    // contractions (ccsd.cxx:123-180)
    launch_tau();
    ctx.run(iter_plan);
    // Z.weight(D); T += Z; conv = Z.norm(00)  (ccsd.cxx:184-185,190), fused, one launch
    CCSD_CUDA(cudaMemsetAsync(d_red, 0, 2 * sizeof(double), s));
    kern::update_batched(d_upd, d_upd_cs, n_upd, upd_chunks, d_red + 1, s);
    // Tau from the updated T, energy (ccsd.cxx:187-189)
    launch_tau();
    ctx.run(energy_plan, nullptr, d_red + 0);
    // DIIS (diis.hpp:70-227)
    if (opts.diis_order > 1) diis_step();
}

void Solver::diis_step() {
    cudaStream_t s = ctx.stream;
    const int n = opts.diis_order;
    Tensor& t1 = ctx.tensor(T1);
    Tensor& t2 = ctx.tensor(T2);
    Tensor& z1 = ctx.tensor(Z1);
    Tensor& z2 = ctx.tensor(Z2);
    // advance the ring: slot of the newest vector
    kern::diis_advance(d_state, n, s);
    // copy x, dx into the head slot (device-side slot index)
    kern::diis_store(d_state, d_xs, d_dxs, t1.data, t1.total, t2.data, t2.total, z1.data, z2.data, s);
    // new error-matrix row: <dx_head, dx_j> for all slots (absent slots are zero vectors)
    CCSD_CUDA(cudaMemsetAsync(d_dots, 0, n * sizeof(double), s));
    for (auto& sg : segs) kern::diis_dots(d_state, d_dxs, n, sg.off, sg.len, sg.w, d_dots, s);
    // bordered system, solve, coefficients by slot
    kern::diis_solve(d_state, d_e, d_c, d_dots, n, s);
    // x = sum c_j x_j (diis.hpp:205-226).  The reference also extrapolates dx into Z; every
    // iteration assigns Z afresh before reading it and the energy and residual are taken
    // before DIIS, so that second combination (nine full-vector passes) is not formed
    kern::lincomb(t1.data, t1.total, t2.data, t2.total, d_xs, d_c, n, s);
}

// Slice count per contraction (the autotuner).  From the current amplitudes, one trial
// evaluates the iteration's contractions, the Jacobi update and the energy (DIIS left out)
// with every contraction at the solver's slice count; then one trial per statement with
// split contractions, that statement one slice fewer.  The difference of each trial's
// energy from the first is that statement's measured energy change; slice_choice picks
// the statements that keep one slice fewer.  The amplitudes are restored after every
// trial, so the solve continues from where it was.
void Solver::autotune_slices() {
    tuned = true;
    cudaStream_t s = ctx.stream;
    Tensor& t1 = ctx.tensor(T1);
    Tensor& t2 = ctx.tensor(T2);
    const int64_t n1 = t1.total, n2 = t2.total;
    double* save = (double*)ctx.dmalloc((n1 + n2) * sizeof(double));
    CCSD_CUDA(cudaMemcpyAsync(save, t1.data, n1 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CCSD_CUDA(cudaMemcpyAsync(save + n1, t2.data, n2 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    std::vector<std::string> labels;
    std::map<std::string, std::vector<GemmStep*>> steps;
    for (auto& g : iter_plan.gemms) {
        if (!ctx.routes_split(g)) continue;
        if (!steps.count(g.label)) labels.push_back(g.label);
        steps[g.label].push_back(&g);
    }
    auto trial = [&]() {
        CCSD_CUDA(cudaMemsetAsync(d_red, 0, 2 * sizeof(double), s));
        launch_tau();
        ctx.run(iter_plan);
        kern::update_batched(d_upd, d_upd_cs, n_upd, upd_chunks, d_red + 1, s);
        launch_tau();
        ctx.run(energy_plan, nullptr, d_red + 0);
        CCSD_CUDA(cudaMemcpyAsync(h_red, d_red, sizeof(double), cudaMemcpyDeviceToHost, s));
        CCSD_CUDA(cudaMemcpyAsync(t1.data, save, n1 * sizeof(double), cudaMemcpyDeviceToDevice, s));
        CCSD_CUDA(cudaMemcpyAsync(t2.data, save + n1, n2 * sizeof(double), cudaMemcpyDeviceToDevice, s));
        CCSD_CUDA(cudaStreamSynchronize(s));
        return h_red[0];
    };
    const double e0 = trial();
    std::vector<double> dE;
    for (auto& l : labels) {
        for (GemmStep* g : steps[l]) g->slice_delta = -1;
        const double e = trial();
        for (GemmStep* g : steps[l]) g->slice_delta = 0;
        dE.push_back(e - e0);
    }
    const std::vector<int> drop = slice_choice(dE, opts.autotune_de);
    tune_report.clear();
    for (size_t i = 0; i < labels.size(); i++) {
        if (drop[i])
            for (GemmStep* g : steps[labels[i]]) g->slice_delta = -1;
        tune_report.push_back({labels[i], dE[i], drop[i] ? -1 : 0});
    }
    ctx.dfree(save, (n1 + n2) * sizeof(double));
    if (kern::split_error(true)) throw Error(CCSD_ERR_TIMEOUT, "split GEMM wait expired while tuning");
}

void Solver::iterate_async() {
    // Refinement of the split precision.  Three slices leave a residual floor (near 1e-9
    // for BF16, ~8x higher for INT8); once conv < refine_tol the contractions move to four
    // slices, and on a stall above conv_tol to five (INT8) and then to native FP64.
    // Graphs are recaptured after a switch.
    use_mode();
    const bool split_opts = opts.precision == CCSD_PREC_SPLIT || opts.precision == CCSD_PREC_SPLIT_I8;
    if (split_opts && opts.refine_tol > 0 && conv < opts.refine_tol && ctx.precision != CCSD_PREC_FP64) {
        bool escalate = false;
        if (ctx.split_slices() == 3) {
            ctx.slices = 4;
            ctx.refresh_split(iter_plan);
            escalate = true;
        } else if (conv_hist.size() >= 5) {
            // stalled: none of the last three residuals improves on the best one before
            // them by 20% (DIIS makes single steps non-monotone; a slowly converging
            // system still gains a factor ~2 over three iterations)
            const size_t n = conv_hist.size();
            const double before = *std::min_element(conv_hist.begin(), conv_hist.end() - 3);
            const double recent = std::min({conv_hist[n - 3], conv_hist[n - 2], conv_hist[n - 1]});
            if (recent > 0.8 * before) {
                if (kern::slice_scheme_ok(ctx.slice_kind(), ctx.split_slices() + 1)) {
                    ctx.slices = ctx.split_slices() + 1;
                    ctx.refresh_split(iter_plan);
                } else {
                    ctx.precision = CCSD_PREC_FP64;
                }
                escalate = true;
            }
        }
        if (escalate) {
            mode_precision = ctx.precision;
            mode_slices = ctx.slices;
            refined = true;
            conv_hist.clear();
            // the stored vectors carry the previous mode's contraction noise, which would
            // hold the extrapolated residual at that mode's floor until they age out of the
            // ring: restart the subspace from the current amplitudes
            if (opts.diis_order > 1) CCSD_CUDA(cudaMemsetAsync(d_state + 1, 0, sizeof(int), ctx.stream));
            if (graph_exec) cudaGraphExecDestroy(graph_exec);
            if (graph) cudaGraphDestroy(graph);
            graph_exec = nullptr;
            graph = nullptr;
            captured_once = false;
        }
    }
    // the autotuner runs once, on the first iteration at 4 or more slices after the first
    // (the amplitudes have left the MP2 guess), before any graph is captured
    if (opts.autotune_de > 0 && !tuned && iterations >= 1 && ctx.split_precision() && ctx.split_slices() >= 4 &&
        !ctx.host_only)
        autotune_slices();
    if (opts.use_graph) {
        if (!graph_exec) {
            // the first iteration runs eagerly (it also warms every kernel), the graph is
            // captured from the second one on
            if (captured_once) {
                CCSD_CUDA(cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeThreadLocal));
                try {
                    launch_iteration();
                } catch (...) {
                    cudaGraph_t g;
                    cudaStreamEndCapture(ctx.stream, &g);
                    if (g) cudaGraphDestroy(g);
                    throw;
                }
                CCSD_CUDA(cudaStreamEndCapture(ctx.stream, &graph));
                CCSD_CUDA(cudaGraphInstantiate(&graph_exec, graph, 0));
            } else {
                launch_iteration();
                captured_once = true;
                iterations++;
                return;
            }
        }
        CCSD_CUDA(cudaGraphLaunch(graph_exec, ctx.stream));
    } else {
        launch_iteration();
    }
    iterations++;
}

void Solver::read_status() {
    post_status();
    CCSD_CUDA(cudaStreamSynchronize(ctx.stream));
    check_status();
}

void Solver::post_status() {
    CCSD_CUDA(cudaMemcpyAsync(h_red, d_red, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
    if (opts.diis_order > 1) {
        CCSD_CUDA(cudaMemcpyAsync(h_state, d_state, 8 * sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    }
}

void Solver::check_status() {
    energy = h_red[0];
    conv = h_red[1];
    conv_hist.push_back(conv);
    if (opts.precision == CCSD_PREC_SPLIT || opts.precision == CCSD_PREC_SPLIT_I8) {
        int e = kern::split_error(true);
        if (e) throw Error(CCSD_ERR_TIMEOUT, "split GEMM wait " + std::to_string(e) + " expired");
    }
    if (opts.diis_order > 1 && h_state[3] != 0)
        throw Error(CCSD_ERR_SINGULAR, "DIIS: singular error matrix after the eps retry");
    if (!std::isfinite(energy) || !std::isfinite(conv)) throw Error(CCSD_DIVERGED, "NaN/Inf in energy or residual");
}

void Solver::iterate(double* e, double* c) {
    iterate_async();
    read_status();
    if (e) *e = energy;
    if (c) *c = conv;
}

int Solver::run(double* e, double* c, int* it) {
    // Iterative::run: for (iter = 1; iter <= maxiter && !converged; iter++)
    int status = CCSD_OK;
    while (iterations < opts.max_iter && !(conv < opts.conv_tol)) {
        iterate(nullptr, nullptr);
    }
    if (!(conv < opts.conv_tol)) status = CCSD_NOT_CONVERGED;
    if (e) *e = energy;
    if (c) *c = conv;
    if (it) *it = iterations;
    return status;
}

}  // namespace ccsd
