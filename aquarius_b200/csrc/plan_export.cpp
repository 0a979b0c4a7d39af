// Diagnostic export of one planned statement: the block contractions, permuted sums, block
// scalings and dots that ccsd_contract / ccsd_sum expanded it to (spin cases, irrep blocks,
// pair restrictions and antisymmetriser images already applied), with the block layout of
// every tensor the steps touch.  Plain text, one record per line:
//
//   scratch <elements>
//   tensor <handle> <ndim> <total> <view_of> <ncases> <name>
//   group <group per position>
//   case <alpha count per group x4> <spin per position>
//   block <irrep per position> <len per position> <stride per position> <offset> <size> <npairs>
//         then per packed pair <p> <q> <kind> <stride>: kind 1 stores x<y of equal irreps at
//         stride * (y(y-1)/2 + x), kind 2 (irrep p < irrep q) at stride * (x + len_p * y)
//   gemm <tA> <tB> <tC> <M> <N> <K> <alpha> <nvm> <nvn> <vsign x4>
//   Am|Ak|Bk|Bn|Cm0|Cm1|Cn0|Cn1 <offsets>
//   sum <tA> <tC> <ndim> <alpha> <offA> <offC> / len / sA / sC lines
//   scale <tC> <off> <n> <beta>
//   dot <tA> <tB> <ndim> <alpha> <offA> <offB> / len / sA / sB lines
//
// Offsets are element offsets into the storage of the tensor (a view's into its base's);
// handle -1 is the plan's scratch buffer.  Steps are listed in execution order.
#include <cstdio>
#include <set>

#include "engine.hpp"

namespace ccsd {

namespace {

void ints(FILE* f, const char* tag, const std::vector<int64_t>& v) {
    std::fprintf(f, "%s", tag);
    for (int64_t x : v) std::fprintf(f, " %lld", (long long)x);
    std::fprintf(f, "\n");
}

void ints(FILE* f, const char* tag, const int64_t* v, int n) {
    ints(f, tag, std::vector<int64_t>(v, v + n));
}

}  // namespace

void export_plan(const Context& ctx, const Plan& p, const char* path) {
    std::set<int> handles;
    for (auto& g : p.gemms) handles.insert({g.tA, g.tB, g.tC});
    for (auto& s : p.sums) handles.insert({s.tA, s.tC});
    for (auto& s : p.scales) handles.insert(s.tC);
    for (auto& d : p.dots) handles.insert({d.tA, d.tB});
    handles.erase(kScratch);
    std::set<int> all = handles;
    for (int h : handles) {
        auto it = ctx.tensors.find(h);
        if (it == ctx.tensors.end()) throw Error(CCSD_ERR_ARG, "plan refers to a destroyed tensor");
        if (it->second->view_of) all.insert(it->second->view_of);
    }
    FILE* f = std::fopen(path, "w");
    if (!f) throw Error(CCSD_ERR_ARG, std::string("cannot write ") + path);
    std::fprintf(f, "scratch %lld\n", (long long)p.scratch_elems);
    for (int h : all) {
        const Tensor& T = *ctx.tensors.at(h);
        std::fprintf(f, "tensor %d %d %lld %d %zu %s\n", h, T.ndim, (long long)T.total, T.view_of, T.cases.size(),
                     T.name.c_str());
        std::fprintf(f, "group");
        for (int g : T.group) std::fprintf(f, " %d", g);
        std::fprintf(f, "\n");
        for (auto& sc : T.cases) {
            std::fprintf(f, "case %d %d %d %d", sc.alpha[0], sc.alpha[1], sc.alpha[2], sc.alpha[3]);
            for (int s : sc.spin) std::fprintf(f, " %d", s);
            std::fprintf(f, "\n");
            for (auto& b : sc.blocks) {
                std::fprintf(f, "block");
                for (int x : b.irrep) std::fprintf(f, " %d", x);
                for (int x : b.len) std::fprintf(f, " %d", x);
                for (int64_t x : b.stride) std::fprintf(f, " %lld", (long long)x);
                std::fprintf(f, " %lld %lld %zu", (long long)b.offset, (long long)b.size, b.pairs.size());
                for (auto& pr : b.pairs)
                    std::fprintf(f, " %d %d %d %lld", pr.p, pr.q, pr.kind, (long long)pr.stride);
                std::fprintf(f, "\n");
            }
        }
    }
    for (auto& st : p.steps) {
        switch (st.kind) {
            case Step::GEMM: {
                const GemmStep& g = p.gemms[st.idx];
                std::fprintf(f, "gemm %d %d %d %d %d %d %.17g %d %d %.17g %.17g %.17g %.17g\n", g.tA, g.tB, g.tC, g.M,
                             g.N, g.K, g.alpha, g.nvm, g.nvn, g.vsign[0], g.vsign[1], g.vsign[2], g.vsign[3]);
                ints(f, "Am", g.hAm);
                ints(f, "Ak", g.hAk);
                ints(f, "Bk", g.hBk);
                ints(f, "Bn", g.hBn);
                ints(f, "Cm0", g.hCm[0]);
                ints(f, "Cm1", g.hCm[1]);
                ints(f, "Cn0", g.hCn[0]);
                ints(f, "Cn1", g.hCn[1]);
                break;
            }
            case Step::SUM: {
                const SumStep& s = p.sums[st.idx];
                std::fprintf(f, "sum %d %d %d %.17g %lld %lld\n", s.tA, s.tC, s.ndim, s.alpha, (long long)s.offA,
                             (long long)s.offC);
                ints(f, "len", s.len, s.ndim);
                ints(f, "sA", s.sA, s.ndim);
                ints(f, "sC", s.sC, s.ndim);
                break;
            }
            case Step::SCALE: {
                const ScaleStep& s = p.scales[st.idx];
                std::fprintf(f, "scale %d %lld %lld %.17g\n", s.tC, (long long)s.off, (long long)s.n, s.beta);
                break;
            }
            case Step::DOT: {
                const DotStep& d = p.dots[st.idx];
                std::fprintf(f, "dot %d %d %d %.17g %lld %lld\n", d.tA, d.tB, d.ndim, d.alpha, (long long)d.offA,
                             (long long)d.offB);
                ints(f, "len", d.len, d.ndim);
                ints(f, "sA", d.sA, d.ndim);
                ints(f, "sB", d.sB, d.ndim);
                break;
            }
        }
    }
    const bool ok = std::fclose(f) == 0;
    if (!ok) throw Error(CCSD_ERR_ARG, std::string("cannot write ") + path);
}

}  // namespace ccsd
