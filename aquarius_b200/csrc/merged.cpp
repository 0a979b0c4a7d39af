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
    // block products that would run on the FP64 kernels, GEMM-shaped
    std::vector<Cand> cands;
    for (int i = first; i < end; i++) {
        const GemmStep& g = p.gemms[p.steps[i].idx];
        if (g.mkey.empty() || routes_split(g) || std::min(g.M, g.N) <= 8 || g.K <= 0) continue;
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
    // the grids to merge: a component that is a full grid, else the row classes of it (rows
    // that meet the same column blocks over the same k blocks) that are.  A ring statement's
    // component joins rows of several spin sectors and antisymmetriser terms through shared
    // k and column blocks; each sector alone is a full grid.
    std::vector<std::vector<int>> grids;
    for (auto& kv : comp) {
        const std::vector<int>& js = kv.second;
        if (js.size() < 2) continue;
        std::set<int> Rs, Cs, Ks;
        std::set<std::tuple<int, int, int>> cells;
        for (int j : js) {
            Rs.insert(cands[j].r);
            Cs.insert(cands[j].c);
            Ks.insert(cands[j].k);
            cells.insert(std::make_tuple(cands[j].r, cands[j].c, cands[j].k));
        }
        if (cells.size() == js.size() && cells.size() == Rs.size() * Cs.size() * Ks.size()) {
            grids.push_back(js);
            continue;
        }
        std::map<int, std::pair<std::set<int>, std::set<int>>> sig;   // row -> (column blocks, k blocks)
        std::map<int, std::vector<int>> of_row;
        for (int j : js) {
            sig[cands[j].r].first.insert(cands[j].c);
            sig[cands[j].r].second.insert(cands[j].k);
            of_row[cands[j].r].push_back(j);
        }
        std::map<std::pair<std::set<int>, std::set<int>>, std::vector<int>> cls;
        for (auto& rs : sig) cls[rs.second].push_back(rs.first);
        for (auto& cl : cls) {
            std::vector<int> sub;
            for (int r : cl.second) sub.insert(sub.end(), of_row[r].begin(), of_row[r].end());
            if (sub.size() < 2) continue;
            std::sort(sub.begin(), sub.end());   // plan order
            if (sub.size() == cl.second.size() * cl.first.first.size() * cl.first.second.size()) grids.push_back(sub);
            else reject(sub, "row class not a full grid", cl.second.size(), cl.first.first.size(), cl.first.second.size());
        }
    }
    for (const std::vector<int>& js : grids) {
        std::vector<int> R, C, Kb;
        std::map<std::tuple<int, int, int>, int> at;
        std::map<int, int> Mr, Nc, Kl;
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
            if (!Mr.count(c.r)) R.push_back(c.r), Mr[c.r] = g.M;
            if (!Nc.count(c.c)) C.push_back(c.c), Nc[c.c] = g.N;
            if (!Kl.count(c.k)) Kb.push_back(c.k), Kl[c.k] = g.K;
            ok &= Mr[c.r] == g.M && Nc[c.c] == g.N && Kl[c.k] == g.K;
        }
        // a full grid only: every row block with every column block over every k block
        if (!ok || at.size() != R.size() * C.size() * Kb.size()) {
            reject(js, !ok ? "repeated or mismatched extents" : "not a full grid", R.size(), C.size(), Kb.size());
            continue;
        }
        auto J = [&](int r, int c, int k) { return at.at(std::make_tuple(r, c, k)); };
        // the rectangles of A depend on (rows, k) only, of B on (k, columns), of C on (rows,
        // columns): the products that share them must agree on their tables
        for (int r : R)
            for (int k : Kb) {
                const GemmStep& a = G(J(r, C[0], k));
                for (int c : C) {
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
                const GemmStep& a = G(J(R[0], c, k));
                for (int r : R) {
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
        for (int k : Kb) ratio[k] = G(J(R[0], C[0], k)).alpha / G(J(R[0], C[0], Kb[0])).alpha;
        for (int r : R)
            for (int c : C) {
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
        // a class worth one tensor-core GEMM (its slicing reads the operands once; below this
        // the grouped FP64 launch is cheaper)
        if (M < 64 || N < 32 || K < 128 || 2.0 * M * N * K < 2e7 || M > (1 << 28) || N > (1 << 28) || K > (1 << 28)) {
            reject(js, "below the size bar", R.size(), C.size(), Kb.size());
            continue;
        }
        if (report)
            std::fprintf(stderr, "[merged] %-48s %5zu products  M=%-6lld N=%-6lld K=%-6lld\n", G(js[0]).label.c_str(),
                         js.size(), (long long)M, (long long)N, (long long)K);

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
                const GemmStep& g = G(J(r, C[0], k));
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
                const GemmStep& g = G(J(R[0], c, k));
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
        for (int r : R)
            for (int c : C) {
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
                for (int k : Kb) constA &= G(J(r, C[0], k)).tA != kScratch && is_constant(G(J(r, C[0], k)).tA);
            for (int c : C)
                for (int k : Kb) constB &= G(J(R[0], c, k)).tB != kScratch && is_constant(G(J(R[0], c, k)).tB);
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

void Context::run_merged(Plan& p, MergedProduct& m) {
    const int ns = step_slices(p.gemms[m.first_gemm]), kind = slice_kind();
    split_launches++;
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
                kern::rect_slice(d, ts, n, tiles, ns, c, stream);
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
        kern::rect_slice(d, ts, n, tiles, ns, v, stream);
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
    kern::gemm_split(va, vb, m.M, m.N, m.K, a, stream, ks);
    for (auto& L : m.levels)
        kern::rect_scatter(L.d, L.cs, L.n, L.chunks, merged_ws, m.N, (int64_t)m.M * m.N, ks, stream);
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
