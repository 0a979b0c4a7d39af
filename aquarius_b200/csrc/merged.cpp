// Merged products of symmetry-blocked statements on the split path.
//
// A statement over irrep blocks lowers to one block product per irrep tuple: for a D2h
// ring term at o=48 v=336 that is 84k products of a few hundred rows, columns and k each,
// far too small for a 128-wide tensor-core tile.  The block products that share their
// rows (the irreps and spins of the row indices), their columns and their k range form a
// grid: within one class of the pair irrep, every row block meets every column block over
// every k block (the role of the block-triple walk of SymmetryBlockedTensor::mult,
// src/tensor/symblocked_tensor.cxx:1031-1088).  Such a class runs as ONE split GEMM: each
// block product contributes a rectangle of the merged A (its rows x its k), of the merged
// B and of the dense result; the rectangles of A and B are sliced straight from the
// tensors through the products' own offset tables, the GEMM writes a dense product, and a
// scatter adds each result rectangle into its C block (with the antisymmetriser variants
// of the product), in levels so that no two rectangles of a launch write one block.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <numeric>
#include <set>
#include <tuple>

#include "engine.hpp"

namespace ccsd {

void Context::build_merged(Plan& p, GemmRun& run, int first, int end, std::vector<char>& merged,
                           const std::function<std::pair<int, int64_t>(int, int64_t)>& block_of) {
    struct Cand {
        int i, r, c, k;
    };
    std::map<std::string, int> rid, cid, kid;
    auto id = [](std::map<std::string, int>& m, const std::string& key) {
        auto it = m.find(key);
        if (it != m.end()) return it->second;
        const int v = (int)m.size();
        m.emplace(key, v);
        return v;
    };
    // GEMM-shaped block products (those large enough for the split kernel alone too: a hole
    // they left would break the grid of their class)
    std::vector<Cand> cands;
    for (int i = first; i < end; i++) {
        const GemmStep& g = p.gemms[p.steps[i].idx];
        if (g.mkey.empty() || std::min(g.M, g.N) <= 8 || g.K <= 0) continue;
        cands.push_back({i, id(rid, g.mkey), id(cid, g.nkey), id(kid, g.kkey)});
    }
    if (std::getenv("CCSD_MERGE_REPORT")) {
        double all = 0, in = 0;
        for (int i = first; i < end; i++) all += p.gemms[p.steps[i].idx].flops();
        for (auto& c : cands) in += p.gemms[p.steps[c.i].idx].flops();
        std::fprintf(stderr, "[merge-run] %-48s %5d products %.3e flop, candidates %zu with %.3e flop\n",
                     p.gemms[p.steps[first].idx].label.c_str(), end - first, all, cands.size(), in);
    }
    if (cands.size() < 2) return;
    const int NR = (int)rid.size(), NK = (int)kid.size(), NC = (int)cid.size();
    std::vector<int> par(NR + NK + NC);
    std::iota(par.begin(), par.end(), 0);
    auto find = [&](int x) {
        while (par[x] != x) x = par[x] = par[par[x]];
        return x;
    };
    auto unite = [&](int a, int b) {
        a = find(a);
        b = find(b);
        if (a != b) par[a] = b;
    };
    for (auto& c : cands) {
        unite(c.r, NR + c.k);
        unite(NR + c.k, NR + NK + c.c);
    }
    std::map<int, std::vector<int>> comp;
    for (size_t j = 0; j < cands.size(); j++) comp[find(cands[j].r)].push_back((int)j);
    auto G = [&](int j) -> const GemmStep& { return p.gemms[p.steps[cands[j].i].idx]; };

    const bool report = std::getenv("CCSD_MERGE_REPORT") != nullptr;
    auto reject = [&](const std::vector<int>& js, const char* why, size_t nr, size_t nc, size_t nk) {
        if (!report) return;
        double fl = 0;
        for (int j : js) fl += G(j).flops();
        std::fprintf(stderr, "[merge-skip] %-48s %5zu products %.3e flop  R=%zu C=%zu K=%zu  %s\n",
                     G(js[0]).label.c_str(), js.size(), fl, nr, nc, nk, why);
    };
    // The grids to merge.  The rows of a component that meet the same k blocks form a class;
    // the rows and columns of a class that are linked through present (row, column) pairs
    // form a grid whose columns are every column block its rows meet.  Each present pair
    // must run over all of the grid's k blocks; the merged GEMM computes every pair and
    // scatters the present ones, which is worth it while they hold at least half of the
    // product, and otherwise the rows that meet the same columns form exact grids.  A
    // ring statement's component joins rows of several spin sectors and antisymmetriser
    // terms, each linked to its own columns, and the planner's canonical images leave
    // same-spin sectors triangular.
    struct Grid {
        std::vector<int> js, R, C, Kb;
    };
    std::vector<Grid> grids;
    auto add_grid = [&](const std::vector<int>& rows, const std::map<int, std::vector<int>>& of_row,
                        const std::vector<int>& kb) {
        Grid gr;
        std::set<int> cs;
        for (int r : rows) {
            gr.js.insert(gr.js.end(), of_row.at(r).begin(), of_row.at(r).end());
            for (int j : of_row.at(r)) cs.insert(cands[j].c);
        }
        if (gr.js.size() < 2) return;
        std::sort(gr.js.begin(), gr.js.end());   // plan order
        gr.R = rows;
        gr.C.assign(cs.begin(), cs.end());
        gr.Kb = kb;
        grids.push_back(std::move(gr));
    };
    for (auto& kv : comp) {
        const std::vector<int>& js = kv.second;
        if (js.size() < 2) continue;
        std::map<int, std::set<int>> kset, cset;
        std::map<int, std::vector<int>> of_row;
        std::map<int, int64_t> rlen, clen;
        for (int j : js) {
            kset[cands[j].r].insert(cands[j].k);
            cset[cands[j].r].insert(cands[j].c);
            of_row[cands[j].r].push_back(j);
            rlen[cands[j].r] = G(j).M;
            clen[cands[j].c] = G(j).N;
        }
        std::map<std::set<int>, std::vector<int>> cls;   // k blocks -> rows
        for (auto& rk : kset) cls[rk.second].push_back(rk.first);
        for (auto& cl : cls) {
            const std::vector<int> kb(cl.first.begin(), cl.first.end());
            // rows linked through shared columns
            std::map<int, int> up;   // union-find over rows (r) and columns (-1 - c)
            std::function<int(int)> root = [&](int x) {
                auto it = up.find(x);
                if (it == up.end() || it->second == x) return x;
                return it->second = root(it->second);
            };
            for (int r : cl.second) {
                up.emplace(r, r);
                for (int c : cset[r]) {
                    up.emplace(-1 - c, -1 - c);
                    const int a = root(r), b = root(-1 - c);
                    if (a != b) up[a] = b;
                }
            }
            std::map<int, std::vector<int>> linked;
            for (int r : cl.second) linked[root(r)].push_back(r);
            for (auto& lk : linked) {
                const std::vector<int>& rows = lk.second;
                std::set<int> cs;
                double present = 0, mr = 0, nc = 0;
                for (int r : rows) {
                    mr += rlen[r];
                    for (int c : cset[r]) present += (double)rlen[r] * clen[c], cs.insert(c);
                }
                for (int c : cs) nc += clen[c];
                if (present >= 0.5 * mr * nc) {
                    add_grid(rows, of_row, kb);
                    continue;
                }
                std::map<std::set<int>, std::vector<int>> exact;   // columns -> rows
                for (int r : rows) exact[cset[r]].push_back(r);
                for (auto& ex : exact) add_grid(ex.second, of_row, kb);
            }
        }
    }
    for (const Grid& gr : grids) {
        const std::vector<int>& js = gr.js;
        const std::vector<int>& R = gr.R;
        const std::vector<int>& C = gr.C;
        const std::vector<int>& Kb = gr.Kb;
        std::map<std::tuple<int, int, int>, int> at;
        std::map<int, int> Mr, Nc, Kl;
        std::set<std::pair<int, int>> present;
        bool ok = true;
        for (int j : js) {
            const Cand& c = cands[j];
            const GemmStep& g = G(j);
            auto t = std::make_tuple(c.r, c.c, c.k);
            if (at.count(t)) {
                ok = false;
                break;
            }
            at[t] = j;
            present.insert({c.r, c.c});
            if (!Mr.count(c.r)) Mr[c.r] = g.M;
            if (!Nc.count(c.c)) Nc[c.c] = g.N;
            if (!Kl.count(c.k)) Kl[c.k] = g.K;
            ok &= Mr[c.r] == g.M && Nc[c.c] == g.N && Kl[c.k] == g.K;
        }
        // every present pair over every k block
        if (!ok || at.size() != present.size() * Kb.size()) {
            reject(js, !ok ? "repeated or mismatched extents" : "a pair misses k blocks", R.size(), C.size(), Kb.size());
            continue;
        }
        auto J = [&](int r, int c, int k) { return at.at(std::make_tuple(r, c, k)); };
        std::map<int, std::vector<int>> cols_of, rows_of;   // present pairs by row / by column
        for (auto& rc : present) {
            cols_of[rc.first].push_back(rc.second);
            rows_of[rc.second].push_back(rc.first);
        }
        // the rectangles of A depend on (rows, k) only, of B on (k, columns), of C on (rows,
        // columns): the products that share them must agree on their tables
        for (int r : R)
            for (int k : Kb) {
                const GemmStep& a = G(J(r, cols_of[r][0], k));
                for (int c : cols_of[r]) {
                    const GemmStep& b = G(J(r, c, k));
                    ok &= b.tA == a.tA && b.hAm == a.hAm && b.hAk == a.hAk && b.a_kcontig == a.a_kcontig;
                }
            }
        if (!ok) {
            reject(js, "A tables differ", R.size(), C.size(), Kb.size());
            continue;
        }
        for (int k : Kb)
            for (int c : C) {
                const GemmStep& a = G(J(rows_of[c][0], c, k));
                for (int r : rows_of[c]) {
                    const GemmStep& b = G(J(r, c, k));
                    ok &= b.tB == a.tB && b.hBk == a.hBk && b.hBn == a.hBn && b.b_kcontig == a.b_kcontig;
                }
            }
        if (!ok) {
            reject(js, "B tables differ", R.size(), C.size(), Kb.size());
            continue;
        }
        // coefficients: alpha(r, c, k) = alpha(r, c, k0) * ratio(k), the ratio (spin weights and
        // reordering signs of the k block) folded into the k block's rectangles of B
        std::map<int, double> ratio;
        const int r0 = present.begin()->first, c0 = present.begin()->second;
        for (int k : Kb) ratio[k] = G(J(r0, c0, k)).alpha / G(J(r0, c0, Kb[0])).alpha;
        for (auto& rc : present) {
            const int r = rc.first, c = rc.second;
            const GemmStep& a = G(J(r, c, Kb[0]));
            for (int k : Kb) {
                const GemmStep& b = G(J(r, c, k));
                ok &= b.alpha == a.alpha * ratio[k];
                ok &= b.tC == a.tC && b.nvm == a.nvm && b.nvn == a.nvn;
                for (int v = 0; v < 2 && ok; v++) ok &= b.hCm[v] == a.hCm[v] && b.hCn[v] == a.hCn[v];
                for (int v = 0; v < 4 && ok; v++) ok &= b.vsign[v] == a.vsign[v];
            }
        }
        if (!ok) {
            reject(js, "coefficients or C tables differ", R.size(), C.size(), Kb.size());
            continue;
        }
        int64_t M = 0, N = 0, K = 0;
        std::map<int, int> roff, coff, koff;
        for (int r : R) roff[r] = (int)M, M += Mr[r];
        for (int c : C) coff[c] = (int)N, N += Nc[c];
        for (int k : Kb) koff[k] = (int)K, K += Kl[k];
        double used = 0;
        for (auto& rc : present) used += (double)Mr[rc.first] * Nc[rc.second];
        if (used < 0.5 * (double)M * N) {
            reject(js, "present pairs under half of the product", R.size(), C.size(), Kb.size());
            continue;
        }
        // a class worth one tensor-core GEMM and its four or more launches (slicing reads each
        // operand twice, the scatter the product once); below this the grouped FP64 launches
        // are cheaper
        if (M < 32 || N < 32 || K < 32 || 2.0 * M * N * K < 1e8 || M > (1 << 28) || N > (1 << 28) || K > (1 << 28)) {
            reject(js, "below the size bar", R.size(), C.size(), Kb.size());
            continue;
        }
        if (report)
            std::fprintf(stderr, "[merged] %-48s %5zu products  M=%-6lld N=%-6lld K=%-6lld ks=%d present %.2f\n",
                         G(js[0]).label.c_str(), js.size(), (long long)M, (long long)N, (long long)K,
                         kern::split_ksplit((int)M, (int)N, (int)K, 4, kern::SLICE_INT8), used / ((double)M * N));

        auto mp = std::make_shared<MergedProduct>();
        mp->M = (int)M;
        mp->N = (int)N;
        mp->K = (int)K;
        mp->first_gemm = p.steps[cands[js[0]].i].idx;
        mp->members = (int)js.size();
        std::vector<kern::RectDesc> A, B;
        std::vector<int64_t> tsA, tsB;
        for (int r : R)
            for (int k : Kb) {
                const GemmStep& g = G(J(r, cols_of[r][0], k));
                const kern::GemmArgs a = gemm_args(p, g);
                kern::RectDesc d;
                d.X = a.A;
                d.R = a.Am;
                d.Kt = a.Ak;
                d.nrows = g.M;
                d.nk = g.K;
                d.row0 = roff[r];
                d.k0 = koff[k];
                d.kc = g.a_kcontig ? 1 : 0;
                d.tiles_r = (g.M + 31) / 32;
                tsA.push_back(mp->tilesA);
                mp->tilesA += (int64_t)d.tiles_r * ((g.K + 63) / 64);
                A.push_back(d);
            }
        for (int c : C)
            for (int k : Kb) {
                const GemmStep& g = G(J(rows_of[c][0], c, k));
                const kern::GemmArgs a = gemm_args(p, g);
                kern::RectDesc d;
                d.X = a.B;
                d.R = a.Bn;
                d.Kt = a.Bk;
                d.nrows = g.N;
                d.nk = g.K;
                d.row0 = coff[c];
                d.k0 = koff[k];
                d.kc = g.b_kcontig ? 1 : 0;
                d.tiles_r = (g.N + 31) / 32;
                d.mul = ratio[k];
                tsB.push_back(mp->tilesB);
                mp->tilesB += (int64_t)d.tiles_r * ((g.K + 63) / 64);
                B.push_back(d);
            }
        // result rectangles, a level above the last one writing any of the same C blocks
        std::map<std::pair<int, int64_t>, int> last;
        std::vector<std::vector<kern::ScatterDesc>> lv;
        double flops = 0;
        for (int j : js) flops += G(j).flops();
        for (auto& rc : present) {
            const int r = rc.first, c = rc.second;
            const GemmStep& g = G(J(r, c, Kb[0]));
            const kern::GemmArgs a = gemm_args(p, g);
            kern::ScatterDesc s;
            s.C = a.C;
            for (int v = 0; v < 2; v++) {
                s.Cm[v] = a.Cm[v];
                s.Cn[v] = a.Cn[v];
            }
            s.nvm = g.nvm;
            s.nvn = g.nvn;
            for (int v = 0; v < 4; v++) s.vsign[v] = a.vsign[v];
            s.alpha = a.alpha;
            s.nrows = g.M;
            s.ncols = g.N;
            s.row0 = roff[r];
            s.col0 = coff[c];
            std::vector<std::pair<int, int64_t>> keys;
            for (int v = 0; v < g.nvm; v++)
                for (int w = 0; w < g.nvn; w++) {
                    if (g.hCm[v].empty() || g.hCn[w].empty()) continue;
                    keys.push_back(block_of(g.tC, *std::min_element(g.hCm[v].begin(), g.hCm[v].end()) +
                                                      *std::min_element(g.hCn[w].begin(), g.hCn[w].end())));
                }
            int L = 0;
            for (auto& key : keys) {
                auto f = last.find(key);
                if (f != last.end()) L = std::max(L, f->second + 1);
            }
            for (auto& key : keys) last[key] = L;
            if ((int)lv.size() <= L) lv.resize(L + 1);
            lv[L].push_back(s);
        }
        // cached slices of constant operands, within the split cache budget
        {
            bool constA = true, constB = true;
            for (int r : R)
                for (int k : Kb) {
                    const int h = G(J(r, cols_of[r][0], k)).tA;
                    constA &= h != kScratch && is_constant(h);
                }
            for (int c : C)
                for (int k : Kb) {
                    const int h = G(J(rows_of[c][0], c, k)).tB;
                    constB &= h != kScratch && is_constant(h);
                }
            int64_t used = merged_cache_bytes;
            for (auto& kv : split_cache) used += kv.second.bytes;
            const int deepest = 5;   // any slice count a refinement reaches
            const int64_t ba = kern::split_slice_bytes((int)M, (int)K, deepest, kern::SLICE_INT8) +
                               3 * (int64_t)kern::split_rows_pad((int)M) * 8;
            const int64_t bb = kern::split_slice_bytes((int)N, (int)K, deepest, kern::SLICE_INT8) +
                               3 * (int64_t)kern::split_rows_pad((int)N) * 8;
            if (constA && used + ba <= split_cache_budget()) {
                mp->cache_a = true;
                used += ba;
                mp->cache_bytes += ba;
            }
            if (constB && used + bb <= split_cache_budget()) {
                mp->cache_b = true;
                mp->cache_bytes += bb;
            }
            merged_cache_bytes += mp->cache_bytes;
        }
        mp->nA = (int)A.size();
        mp->nB = (int)B.size();
        mp->dA = (kern::RectDesc*)dmalloc(A.size() * sizeof(kern::RectDesc));
        mp->dB = (kern::RectDesc*)dmalloc(B.size() * sizeof(kern::RectDesc));
        mp->dA_ts = (int64_t*)dmalloc(tsA.size() * sizeof(int64_t));
        mp->dB_ts = (int64_t*)dmalloc(tsB.size() * sizeof(int64_t));
        stage_h2d(mp->dA, A.data(), A.size() * sizeof(kern::RectDesc));
        stage_h2d(mp->dB, B.data(), B.size() * sizeof(kern::RectDesc));
        stage_h2d(mp->dA_ts, tsA.data(), tsA.size() * sizeof(int64_t));
        stage_h2d(mp->dB_ts, tsB.data(), tsB.size() * sizeof(int64_t));
        for (auto& l : lv) {
            MergedProduct::Level L;
            std::vector<int64_t> cs;
            for (auto& s : l) {
                cs.push_back(L.chunks);
                L.chunks += ((int64_t)s.nrows * s.ncols + kern::kBatchChunk - 1) / kern::kBatchChunk;
            }
            L.n = (int)l.size();
            L.d = (kern::ScatterDesc*)dmalloc(l.size() * sizeof(kern::ScatterDesc));
            L.cs = (int64_t*)dmalloc(cs.size() * sizeof(int64_t));
            stage_h2d(L.d, l.data(), l.size() * sizeof(kern::ScatterDesc));
            stage_h2d(L.cs, cs.data(), cs.size() * sizeof(int64_t));
            mp->levels.push_back(L);
        }
        // the dense product (and its split-K partials) for any slice count a refinement reaches
        int64_t need = 0;
        for (int ns = 3; ns <= 5; ns++)
            need = std::max<int64_t>(need, (int64_t)kern::split_ksplit((int)M, (int)N, (int)K, ns, kern::SLICE_INT8) *
                                               M * N);
        if (need > merged_ws_elems) {
            // a smaller buffer stays allocated until the context goes: a captured graph of an
            // earlier plan may still name it
            if (merged_ws) merged_retired.push_back(merged_ws);
            merged_ws = (double*)dmalloc(need * sizeof(double));
            merged_ws_elems = need;
        }
        // the slice workspaces too are sized here, before any capture
        ensure_ws(split_ws.a, (int)M, (int)K);
        ensure_ws(split_ws.b, (int)N, (int)K);
        for (int j : js) merged[cands[j].i - first] = 1;
        GemmLaunch l;
        l.kind = GemmLaunch::MERGED_SPLIT;
        l.merged = mp;
        l.flops = flops;
        run.launches.push_back(l);
    }
}

void Context::run_merged(Plan& p, MergedProduct& m, const std::string& label) {
    const int ns = step_slices(p.gemms[m.first_gemm]), kind = slice_kind();
    split_launches++;
    // CCSD_PROFILE_KINDS=1: the phases of a merged product timed apart
    static const bool phases = std::getenv("CCSD_PROFILE_KINDS") != nullptr;
    const bool timed = profiling && phases;
    auto phase = [&](const char* name, const std::function<void()>& f) {
        if (!timed) return f();
        auto ev = prof_begin();
        f();
        prof_end(ev, label + " {merged:" + name + "}", 0.0);
    };
    auto operand = [&](bool is_a) {
        const int rows = is_a ? m.M : m.N;
        const kern::RectDesc* d = is_a ? m.dA : m.dB;
        const int64_t* ts = is_a ? m.dA_ts : m.dB_ts;
        const int n = is_a ? m.nA : m.nB;
        const int64_t tiles = is_a ? m.tilesA : m.tilesB;
        if (is_a ? m.cache_a : m.cache_b) {
            kern::SlicedOperand& c = is_a ? m.sA : m.sB;
            if (!c.data || c.kind != kind || c.nslices < ns) {
                if (c.data) free_sliced(c);
                c = alloc_sliced(rows, m.K, ns, kind);
                phase("slice-cached", [&] { kern::rect_slice(d, ts, n, tiles, ns, c, stream); });
            }
            // the first ns slices of a deeper slicing are the ns-slice slicing
            kern::SlicedOperand v = c;
            v.nslices = ns;
            return v;
        }
        kern::SlicedOperand& w = is_a ? split_ws.a : split_ws.b;
        ensure_ws(w, rows, m.K);
        kern::SlicedOperand v = w;
        v.rows = kern::split_rows_pad(rows);
        v.kpad = kern::split_k_pad(m.K, kind);
        v.nslices = ns;
        v.kind = kind;
        phase(is_a ? "slice-a" : "slice-b", [&] { kern::rect_slice(d, ts, n, tiles, ns, v, stream); });
        return v;
    };
    const kern::SlicedOperand va = operand(true);
    const kern::SlicedOperand vb = operand(false);
    kern::GemmArgs a;
    a.ws = merged_ws;
    a.ws_elems = merged_ws_elems;
    a.dense_out = true;
    a.alpha = 1.0;
    const int ks = kern::split_ksplit(m.M, m.N, m.K, ns, kind);
    phase("gemm", [&] { kern::gemm_split(va, vb, m.M, m.N, m.K, a, stream, ks); });
    phase("scatter", [&] {
        for (auto& L : m.levels)
            kern::rect_scatter(L.d, L.cs, L.n, L.chunks, merged_ws, m.N, (int64_t)m.M * m.N, ks, stream);
    });
}

void Context::free_merged(MergedProduct& m) {
    if (m.sA.data) free_sliced(m.sA);
    if (m.sB.data) free_sliced(m.sB);
    merged_cache_bytes -= m.cache_bytes;
    m.cache_bytes = 0;
    m.cache_a = m.cache_b = false;
    dfree(m.dA, m.nA * sizeof(kern::RectDesc));
    dfree(m.dB, m.nB * sizeof(kern::RectDesc));
    dfree(m.dA_ts, m.nA * sizeof(int64_t));
    dfree(m.dB_ts, m.nB * sizeof(int64_t));
    for (auto& L : m.levels) {
        dfree(L.d, L.n * sizeof(kern::ScatterDesc));
        dfree(L.cs, L.n * sizeof(int64_t));
    }
    m.levels.clear();
    m.dA = m.dB = nullptr;
    m.dA_ts = m.dB_ts = nullptr;
}

}  // namespace ccsd
