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
    const size_t launch0 = run.launches.size();
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
                mp->srcA.push_back({&g.hAm, &g.hAk});
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
                mp->srcB.push_back({&g.hBn, &g.hBk});
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
        for (int j : js) mp->self_read |= G(j).tA == G(j).tC || G(j).tB == G(j).tC;
        mp->hA = A;
        mp->hB = B;
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
    batch_merged_slicing(run, launch0);
    for (size_t li = launch0; li < run.launches.size(); li++)
        if (MergedProduct* m = run.launches[li].merged.get()) {   // build-time copies
            m->hA.clear();
            m->hB.clear();
            m->srcA.clear();
            m->srcB.clear();
        }
}

// The operands of a statement's merged products that are not cached (amplitudes and
// intermediates) are sliced by ONE rowmax and ONE slice launch for all of them, each into
// its own operand buffer, before the first merged GEMM: per product, slicing its two
// operands took four memsets and four launches around a GEMM of a fraction of a
// millisecond (the D2h ring statement has about 300 merged products).  The buffers keep
// five slice planes, zero outside the rectangles (zeroed once here: the rectangles cover
// every row and k below the product's extents, and only they are written).  Skipped when
// an operand is the statement's output or the buffers would take more than a quarter of
// the free device memory (CCSD_MERGED_BATCH=0: never).
void Context::batch_merged_slicing(GemmRun& run, size_t launch0) {
    const char* env = std::getenv("CCSD_MERGED_BATCH");
    if (env && env[0] == '0') return;
    struct Dest {
        MergedProduct* m;
        bool a;
        int rows_p, kpad;
        int64_t soff, roff;
    };
    std::vector<Dest> ds;
    int64_t slice_bytes = 0, aux_rows = 0;
    // merged operands with the same rectangles (same tensor, positions, tables and factors)
    // are sliced once and shared
    auto same = [](const MergedProduct& x, bool xa, const MergedProduct& y, bool ya) {
        const auto& rx = xa ? x.hA : x.hB;
        const auto& ry = ya ? y.hA : y.hB;
        const auto& sx = xa ? x.srcA : x.srcB;
        const auto& sy = ya ? y.srcA : y.srcB;
        if (rx.size() != ry.size() || (xa ? x.M : x.N) != (ya ? y.M : y.N) || x.K != y.K) return false;
        for (size_t i = 0; i < rx.size(); i++) {
            const kern::RectDesc &a = rx[i], &b = ry[i];
            if (a.X != b.X || a.nrows != b.nrows || a.nk != b.nk || a.row0 != b.row0 || a.k0 != b.k0 || a.kc != b.kc ||
                a.mul != b.mul)
                return false;
            if (*sx[i].first != *sy[i].first || *sx[i].second != *sy[i].second) return false;
        }
        return true;
    };
    auto digest = [](const MergedProduct& x, bool xa) {
        const auto& rx = xa ? x.hA : x.hB;
        const auto& sx = xa ? x.srcA : x.srcB;
        uint64_t h = 1469598103934665603ull;
        auto mix = [&](uint64_t v) { h = (h ^ v) * 1099511628211ull; };
        for (size_t i = 0; i < rx.size(); i++) {
            mix((uint64_t)(uintptr_t)rx[i].X);
            mix((uint64_t)rx[i].row0 << 32 | (uint32_t)rx[i].k0);
            mix((uint64_t)rx[i].nrows << 32 | (uint32_t)rx[i].nk);
            for (int64_t v : *sx[i].first) mix((uint64_t)v);
            for (int64_t v : *sx[i].second) mix((uint64_t)v);
        }
        return h;
    };
    std::map<uint64_t, std::vector<std::pair<MergedProduct*, bool>>> seen;
    std::vector<std::pair<std::pair<MergedProduct*, bool>, std::pair<MergedProduct*, bool>>> shared;
    for (size_t li = launch0; li < run.launches.size(); li++) {
        MergedProduct* m = run.launches[li].merged.get();
        if (!m || m->self_read) continue;
        for (int side = 0; side < 2; side++) {
            if (side == 0 ? m->cache_a : m->cache_b) continue;
            auto& bucket = seen[digest(*m, side == 0)];
            bool found = false;
            for (auto& e : bucket)
                if (same(*e.first, e.second, *m, side == 0)) {
                    shared.push_back({{m, side == 0}, e});
                    found = true;
                    break;
                }
            if (found) continue;
            bucket.push_back({m, side == 0});
            Dest d;
            d.m = m;
            d.a = side == 0;
            d.rows_p = kern::split_rows_pad(side == 0 ? m->M : m->N);
            d.kpad = kern::split_k_pad(m->K, kern::SLICE_INT8);
            d.soff = slice_bytes;
            d.roff = aux_rows;
            slice_bytes += (5ll * d.rows_p * d.kpad + 255) / 256 * 256;
            aux_rows += d.rows_p;
            ds.push_back(d);
        }
    }
    if (ds.size() < 3 || host_only) return;
    const int64_t aux_bytes = aux_rows * 2 * (int64_t)sizeof(double);   // scales, then row maxima
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    if ((double)(slice_bytes + aux_bytes) > 0.25 * (double)free_b) return;
    uint8_t* sl = (uint8_t*)dmalloc(slice_bytes);
    double* aux = (double*)dmalloc(aux_bytes);
    CCSD_CUDA(cudaMemsetAsync(sl, 0, slice_bytes, stream));
    CCSD_CUDA(cudaMemsetAsync(aux, 0, aux_bytes, stream));
    unsigned long long* rmax = reinterpret_cast<unsigned long long*>(aux + aux_rows);
    std::vector<kern::RectDesc> rects;
    std::vector<int64_t> ts;
    int64_t tiles = 0;
    for (const Dest& d : ds) {
        kern::SlicedOperand v;
        v.data = sl + d.soff;
        v.scale = aux + d.roff;
        v.rowmax = reinterpret_cast<double*>(rmax + d.roff);
        v.rows = d.rows_p;
        v.kpad = d.kpad;
        v.kind = kern::SLICE_INT8;
        v.bytes = 5ll * d.rows_p * d.kpad;
        for (kern::RectDesc r : d.a ? d.m->hA : d.m->hB) {
            r.out = v.data;
            r.scale = v.scale;
            r.rowmax = rmax + d.roff;
            r.rows_p = d.rows_p;
            r.kpad = d.kpad;
            ts.push_back(tiles);
            tiles += (int64_t)r.tiles_r * ((r.nk + 63) / 64);
            rects.push_back(r);
        }
        (d.a ? d.m->batched_a : d.m->batched_b) = true;
        (d.a ? d.m->pa : d.m->pb) = v;
    }
    for (auto& sh : shared) {   // the operands sliced once for several products
        const kern::SlicedOperand& v = sh.second.second ? sh.second.first->pa : sh.second.first->pb;
        (sh.first.second ? sh.first.first->batched_a : sh.first.first->batched_b) = true;
        (sh.first.second ? sh.first.first->pa : sh.first.first->pb) = v;
    }
    GemmLaunch l;
    l.kind = GemmLaunch::MERGED_SLICE;
    l.gemm = run.launches[launch0].merged->first_gemm;   // the statement's slice count
    l.nprob = (int)rects.size();
    l.chunks = tiles;
    l.desc_bytes = rects.size() * sizeof(kern::RectDesc);
    l.d_desc = dmalloc(l.desc_bytes);
    l.d_chunks = (int64_t*)dmalloc(ts.size() * sizeof(int64_t));
    stage_h2d(l.d_desc, rects.data(), l.desc_bytes);
    stage_h2d(l.d_chunks, ts.data(), ts.size() * sizeof(int64_t));
    l.arena = sl;
    l.arena_bytes = slice_bytes;
    l.aux = aux;
    l.aux_bytes = aux_bytes;
    run.launches.insert(run.launches.begin() + launch0, l);
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
        if (is_a ? m.batched_a : m.batched_b) {   // sliced by the statement's batched launch
            kern::SlicedOperand v = is_a ? m.pa : m.pb;
            v.nslices = ns;
            return v;
        }
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
