// Host side of the split-BF16 contraction path: which block contractions use it, slicing
// of their operands (cached for the constant H blocks, per call for the amplitudes and
// intermediates), and the tcgen05 GEMM launch.
#include <algorithm>
#include <cstdlib>

#include "engine.hpp"

namespace ccsd {

// Which block contractions take the split kernel.  Small contractions stay on the FP64
// kernels: a 128x128 tile would be mostly padding and the slicing passes would cost more
// than the product.  CCSD_SPLIT_ROUTE_ALL sends every contraction through the split
// kernel (coverage tests).
bool Context::split_eligible(const GemmStep& g) const {
    if (split_routing == CCSD_SPLIT_ROUTE_ALL) return g.M > 0 && g.N > 0 && g.K > 0;
    if (g.K < 256 || g.flops() < 5e8) return false;
    // few-tile products take the split kernel only when splitting K fills the machine (a
    // 1024-k chunk per range)
    const int64_t tiles = (int64_t)((g.M + 127) / 128) * ((g.N + 127) / 128);
    const int64_t ctas = tiles * kern::split_ksplit(g.M, g.N, g.K, 3, slice_kind());
    if (ctas < 148) return false;
    // Skinny products (an extent of a few tens) stay on the FP64 kernels even when the long
    // operand is a constant H block: each statement gathers that block in its own row / k
    // split, so its slices could not be shared, and slicing per call costs more than the
    // FP64 product
    return g.M >= 128 && g.N >= 64;
}

namespace {

// bytes of the ns slices (and row scales) of a rows x K operand
int64_t slice_bytes(int rows, int K, int ns, int kind) {
    return kern::split_slice_bytes(rows, K, ns, kind) + 2 * (int64_t)kern::split_rows_pad(rows) * 8;
}

// workspace bytes per padded row x k element: enough for any scheme (4 BF16 slices at
// 2 bytes, or 5 INT8 slices at 1 byte over a k padded to 128)
constexpr int64_t kWsBytesPerElem = 8;
int64_t ws_k_pad(int K) { return kern::split_k_pad(K, kern::SLICE_INT8); }   // the wider padding

}  // namespace

// device bytes the sliced constant operands may occupy (CCSD_SPLIT_CACHE_GB, default 50)
int64_t split_cache_budget() {
    const char* e = std::getenv("CCSD_SPLIT_CACHE_GB");
    double gb = e ? std::atof(e) : 50.0;
    return (int64_t)(gb * 1e9);
}

bool Context::routes_split(const GemmStep& g) const {
    return split_precision() && kern::split_supported() && split_eligible(g);
}

kern::SlicedOperand Context::alloc_sliced(int rows, int K, int ns, int kind) {
    kern::SlicedOperand s;
    s.rows = kern::split_rows_pad(rows);
    s.kpad = kern::split_k_pad(K, kind);
    s.nslices = ns;
    s.kind = kind;
    s.bytes = kern::split_slice_bytes(rows, K, ns, kind);
    s.data = (uint8_t*)dmalloc(s.bytes);
    s.scale = (double*)dmalloc(s.rows * sizeof(double));
    s.rowmax = (double*)dmalloc((s.rows + 2) * sizeof(double));   // + the slicing kernels' tile counters
    return s;
}

void Context::free_sliced(kern::SlicedOperand& s) {
    dfree(s.data, s.bytes);
    dfree(s.scale, s.rows * sizeof(double));
    dfree(s.rowmax, (s.rows + 2) * sizeof(double));
    s = kern::SlicedOperand();
}

// make the per-call workspace hold a rows x K operand in any scheme (never shrinks); the
// rows, kpad, kind and slice count of a view are set per call
void Context::ensure_ws(kern::SlicedOperand& w, int rows, int K) {
    const int rp = kern::split_rows_pad(rows);
    const int64_t need = (int64_t)rp * ws_k_pad(K) * kWsBytesPerElem;
    if (w.data && w.bytes >= need && w.rows >= rp) return;
    const int keep_rows = std::max(rp, w.rows);
    const int64_t keep_bytes = std::max(need, w.bytes);
    if (w.data) free_sliced(w);
    w.rows = keep_rows;
    w.bytes = keep_bytes;
    w.data = (uint8_t*)dmalloc(keep_bytes);
    w.scale = (double*)dmalloc(keep_rows * sizeof(double));
    w.rowmax = (double*)dmalloc((keep_rows + 2) * sizeof(double));
}

// Decide, for every split contraction of a plan, which constant operands keep cached
// slices (largest contractions first, within the byte budget), and size the per-call
// workspace for the rest (called before any capture).
void Context::reserve_split(Plan& p) {
    std::vector<GemmStep*> order;
    for (auto& g : p.gemms)
        if (split_eligible(g)) order.push_back(&g);
    std::stable_sort(order.begin(), order.end(), [](GemmStep* a, GemmStep* b) { return a->flops() > b->flops(); });
    int64_t base = merged_cache_bytes;
    for (auto& kv : split_cache) base += kv.second.bytes;
    const int64_t budget = split_cache_budget();
    auto choose = [&](int ns) {
        int64_t used = base;
        for (GemmStep* g : order) {
            for (int side = 0; side < 2; side++) {
                const int h = side == 0 ? g->tA : g->tB;
                const int rows = side == 0 ? g->M : g->N;
                bool& cache = side == 0 ? g->cache_a : g->cache_b;
                cache = false;
                if (h == kScratch || !is_constant(h)) continue;
                const int64_t b = slice_bytes(rows, g->K, ns, slice_kind());
                if (used + b <= budget) {
                    cache = true;
                    used += b;
                }
            }
        }
        return used;
    };
    // a solve that refines to more slices re-slices its cached operands within the same
    // budget: a planning query accounts the largest selection the refinement can reach
    // (the flags of the current slice count are chosen last)
    int64_t used = 0;
    if (plan_refine && host_only)
        for (int ns = split_slices() + 1; kern::slice_scheme_ok(slice_kind(), ns); ns++) used = std::max(used, choose(ns));
    used = std::max(used, choose(split_slices()));
    int64_t need_a = 0, need_b = 0, rows_a = 0, rows_b = 0;
    for (GemmStep* g : order) {
        if (!g->cache_a) {
            need_a = std::max<int64_t>(need_a, (int64_t)kern::split_rows_pad(g->M) * ws_k_pad(g->K));
            rows_a = std::max<int64_t>(rows_a, kern::split_rows_pad(g->M));
        }
        if (!g->cache_b) {
            need_b = std::max<int64_t>(need_b, (int64_t)kern::split_rows_pad(g->N) * ws_k_pad(g->K));
            rows_b = std::max<int64_t>(rows_b, kern::split_rows_pad(g->N));
        }
    }
    if (host_only) {
        // account the cached slices and the workspace as if they were allocated
        dmalloc(used + 1);
        dmalloc(kWsBytesPerElem * (need_a + need_b) + 16 * (rows_a + rows_b) + 1);
        return;
    }
    for (GemmStep* g : order) {
        if (!g->cache_a) ensure_ws(split_ws.a, g->M, g->K);
        if (!g->cache_b) ensure_ws(split_ws.b, g->N, g->K);
    }
}

void Context::drop_split_cache(GemmStep& g) {
    for (int64_t* key : {&g.split_cache_a, &g.split_cache_b}) {
        auto it = *key >= 0 ? split_cache.find(*key) : split_cache.end();
        if (it != split_cache.end()) {
            free_sliced(it->second);
            split_owner.erase(it->first);
            split_cache.erase(it);
        }
        *key = -1;
    }
}

void Context::refresh_split(Plan& p) {
    CCSD_CUDA(cudaStreamSynchronize(stream));
    for (auto& g : p.gemms) drop_split_cache(g);
    reserve_split(p);
}

void Context::run_split_gemm(GemmStep& g, kern::GemmArgs& a) {
    if (!split_eligible(g)) {
        kern::gemm_fp64(a, stream);
        return;
    }
    split_launches++;
    const int ns = step_slices(g), kind = slice_kind();
    auto prepare = [&](bool is_a, int64_t& key, kern::SlicedOperand& ws) -> kern::SlicedOperand* {
        const int rows = is_a ? g.M : g.N;
        const double* X = is_a ? a.A : a.B;
        const int64_t* R = is_a ? a.Am : a.Bn;
        const int64_t* Kt = is_a ? a.Ak : a.Bk;
        const bool kc = is_a ? a.a_kcontig : a.b_kcontig;
        const int h = is_a ? g.tA : g.tB;
        bool& cached = is_a ? g.cache_a : g.cache_b;
        // the first ns slices of a deeper slicing are the ns-slice slicing (each slice is the
        // rounded remainder of the ones before): a cached operand with more slices serves
        // a contraction that the autotuner runs with fewer
        if (cached && key >= 0 && split_cache[key].kind == kind && split_cache[key].nslices > ns) {
            kern::SlicedOperand& v = ws_view[is_a ? 0 : 1];
            v = split_cache[key];
            v.nslices = ns;
            return &v;
        }
        if (cached && key >= 0 && (split_cache[key].nslices != ns || split_cache[key].kind != kind)) {
            // the scheme changed (refinement): re-slice within the budget, or stop caching
            free_sliced(split_cache[key]);
            split_cache.erase(key);
            split_owner.erase(key);
            key = -1;
            int64_t used = 0;
            for (auto& kv : split_cache) used += kv.second.bytes;
            if (used + slice_bytes(rows, g.K, ns, kind) > split_cache_budget()) cached = false;
        }
        if (cached) {
            if (key < 0) {
                key = split_cache_next++;
                split_cache[key] = alloc_sliced(rows, g.K, ns, kind);
                split_owner[key] = h;
                kern::slice_rows(X, R, Kt, rows, g.K, kc, split_cache[key], stream);
            }
            return &split_cache[key];
        }
        ensure_ws(ws, rows, g.K);
        kern::SlicedOperand view = ws;
        view.rows = kern::split_rows_pad(rows);
        view.kpad = kern::split_k_pad(g.K, kind);
        view.nslices = ns;
        view.kind = kind;
        ws_view[is_a ? 0 : 1] = view;
        kern::slice_rows(X, R, Kt, rows, g.K, kc, ws_view[is_a ? 0 : 1], stream);
        return &ws_view[is_a ? 0 : 1];
    };
    kern::SlicedOperand* sa = prepare(true, g.split_cache_a, split_ws.a);
    kern::SlicedOperand* sb = prepare(false, g.split_cache_b, split_ws.b);
    kern::gemm_split(*sa, *sb, g.M, g.N, g.K, a, stream, kern::split_ksplit(g.M, g.N, g.K, ns, kind));
}

}  // namespace ccsd
