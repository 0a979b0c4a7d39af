// Context, device tensors and the step executor.
//
// Tensor layout follows the reference's SpinorbitalTensor / SymmetryBlockedTensor:
// spin cases are the alpha counts of the four index groups with alpha indices first
// (src/tensor/spinorbital_tensor.cxx:166-272, 387-432); inside a case, blocks are the
// totally symmetric irrep tuples (src/tensor/symblocked_tensor.cxx:551-690), each a
// dense array with the first index fastest (src/tensor/ctf_tensor.hpp:221-226).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include "engine.hpp"

namespace ccsd {

Context::Context(int dev, cudaStream_t s) : device(dev), stream(s) {
    host_only = device < 0;
    if (const char* e = std::getenv("CCSD_SPLIT_ALL")) split_routing = e[0] == '1' ? CCSD_SPLIT_ROUTE_ALL : split_routing;
    // CCSD_FP64_TILED=1: every FP64 product on the tiled DMMA kernel (coverage tests)
    if (const char* e = std::getenv("CCSD_FP64_TILED")) fp64_tiled_only = e[0] == '1';
    // CCSD_GROUP_GEMMS=0: every block contraction in a launch of its own (coverage tests)
    if (const char* e = std::getenv("CCSD_GROUP_GEMMS")) group_gemms = e[0] != '0';
    if (!host_only) {
        CCSD_CUDA(cudaSetDevice(device));
        if (!stream) {
            CCSD_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
            own_stream = true;
        }
    }
    d_scalar = (double*)dmalloc(64 * sizeof(double));
}

Context::~Context() {
    if (host_only) return;
    cudaSetDevice(device);
    cudaStreamSynchronize(stream);
    for (auto& kv : plan_cache) release(*kv.second);
    plan_cache.clear();
    for (auto& kv : split_cache) {
        cudaFree(kv.second.data);
        cudaFree(kv.second.scale);
        cudaFree(kv.second.rowmax);
    }
    for (auto* w : {&split_ws.a, &split_ws.b}) {
        cudaFree(w->data);
        cudaFree(w->scale);
        cudaFree(w->rowmax);
    }
    for (auto& kv : tensors)
        if (!kv.second->view_of) cudaFree(kv.second->data);   // views alias their base
    cudaFree(d_scalar);
    cudaFree(splitk_ws);
    cudaFree(merged_ws);
    for (double* q : merged_retired) cudaFree(q);
    for (auto& p : pending) {
        cudaEventDestroy(p.second.first);
        cudaEventDestroy(p.second.second);
    }
    for (auto e : event_pool) cudaEventDestroy(e);
    kern::release_stream_buffers(stream);
    if (pin_buf) cudaFreeHost(pin_buf);
    if (own_stream) cudaStreamDestroy(stream);
}

void Context::stage_h2d(void* dst, const void* src, size_t bytes) {
    if (host_only || bytes == 0) return;
    constexpr size_t kArena = 64ull << 20;
    if (bytes > kArena / 4) {   // large copies go direct (pageable: the driver stages them)
        CCSD_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream));
        return;
    }
    if (!pin_buf) {
        CCSD_CUDA(cudaMallocHost((void**)&pin_buf, kArena));
        pin_cap = kArena;
        pin_off = 0;
    }
    if (pin_off + bytes > pin_cap) {
        CCSD_CUDA(cudaStreamSynchronize(stream));   // every staged copy has left the arena
        pin_off = 0;
    }
    std::memcpy(pin_buf + pin_off, src, bytes);
    CCSD_CUDA(cudaMemcpyAsync(dst, pin_buf + pin_off, bytes, cudaMemcpyHostToDevice, stream));
    pin_off += (bytes + 255) & ~(size_t)255;
}

void* Context::dmalloc(size_t bytes) {
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    if (host_only) {
        // planning only: account the bytes, hand out a distinct never-dereferenced address
        static uintptr_t next = 0x1000;
        next += (bytes + 255) & ~(size_t)255;
        device_bytes += bytes;
        peak_bytes = std::max(peak_bytes, device_bytes);
        return reinterpret_cast<void*>(next);
    }
    cudaError_t e = cudaMallocAsync(&p, bytes, stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(CCSD_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
    device_bytes += bytes;
    peak_bytes = std::max(peak_bytes, device_bytes);
    return p;
}

void Context::dfree(void* p, size_t bytes) {
    if (!p) return;
    if (!host_only) cudaFreeAsync(p, stream);
    device_bytes -= bytes;
}

Tensor& Context::tensor(int h) {
    auto it = tensors.find(h);
    if (it == tensors.end()) throw Error(CCSD_ERR_ARG, "unknown tensor handle " + std::to_string(h));
    return *it->second;
}

bool Context::is_constant(int h) const {
    return std::find(constant_tensors.begin(), constant_tensors.end(), h) != constant_tensors.end();
}

int Context::create_tensor(const std::string& name, const int nout[2], const int nin[2], int flags) {
    if (!spaces_set) throw Error(CCSD_ERR_ARG, "spaces not set on this context");
    auto T = std::make_unique<Tensor>();
    T->name = name;
    T->flags = flags;
    for (int s = 0; s < 2; s++) {
        if (nout[s] < 0 || nin[s] < 0 || nout[s] > 4 || nin[s] > 4) throw Error(CCSD_ERR_ARG, "bad tensor shape");
        T->nout[s] = nout[s];
        T->nin[s] = nin[s];
    }
    const int gsize[4] = {nout[0], nout[1], nin[0], nin[1]};
    for (int g = 0; g < 4; g++)
        for (int k = 0; k < gsize[g]; k++) T->group.push_back(g);
    T->ndim = (int)T->group.size();
    if (T->ndim > 8) throw Error(CCSD_ERR_ARG, "tensor rank above 8");
    const int nouttot = nout[0] + nout[1], nintot = nin[0] + nin[1];
    if ((nintot - nouttot) % 2) throw Error(CCSD_ERR_ARG, "odd spin imbalance");
    if (T->plain() && T->packed()) throw Error(CCSD_ERR_ARG, "a plain tensor has no antisymmetric pairs to pack");
    if (T->plain() && nintot != nouttot) throw Error(CCSD_ERR_ARG, "plain tensors need as many lower as upper indices");
    const int nirr = spaces.nirrep;
    int64_t offset = 0;
    // spin cases: #alpha(lower) = #alpha(upper) + (nin - nout)/2  (spinorbital_tensor.cxx:183);
    // a plain tensor has the one all-alpha case (spatial orbitals)
    for (int a0 = 0; a0 <= gsize[0]; a0++)
        for (int a1 = 0; a1 <= gsize[1]; a1++)
            for (int a2 = 0; a2 <= gsize[2]; a2++)
                for (int a3 = 0; a3 <= gsize[3]; a3++) {
                    if (a2 + a3 != a0 + a1 + (nintot - nouttot) / 2) continue;
                    if (T->plain() && (a0 != gsize[0] || a1 != gsize[1] || a2 != gsize[2] || a3 != gsize[3])) continue;
                    SpinCase sc;
                    sc.alpha[0] = a0;
                    sc.alpha[1] = a1;
                    sc.alpha[2] = a2;
                    sc.alpha[3] = a3;
                    for (int g = 0; g < 4; g++)
                        for (int k = 0; k < gsize[g]; k++) sc.spin.push_back(k < sc.alpha[g] ? ALPHA : BETA);
                    // irrep tuples with XOR 0
                    std::vector<int> irr(T->ndim, 0);
                    while (true) {
                        int x = 0;
                        for (int h : irr) x ^= h;
                        if (x == 0) {
                            Block b;
                            b.irrep = irr;
                            b.len.resize(T->ndim);
                            b.stride.assign(T->ndim, 0);
                            bool stored = true;
                            for (int p = 0; p < T->ndim; p++)
                                b.len[p] = spaces.n[group_space(T->group[p])][sc.spin[p]][irr[p]];
                            // packed same-spin pairs
                            if (T->packed()) {
                                for (int g = 0; g < 4; g++) {
                                    if (gsize[g] != 2) continue;
                                    int p = 0;
                                    while (T->group[p] != g) p++;
                                    if (sc.spin[p] != sc.spin[p + 1]) continue;
                                    Block::Pair pr;
                                    pr.p = p;
                                    pr.q = p + 1;
                                    if (irr[p] == irr[p + 1]) pr.kind = 1;
                                    else if (irr[p] < irr[p + 1]) pr.kind = 2;
                                    else stored = false;
                                    b.pairs.push_back(pr);
                                }
                            }
                            if (stored) {
                                int64_t st = 1;
                                for (int p = 0; p < T->ndim; p++) {
                                    int pi = b.pair_of(p);
                                    if (pi >= 0) {
                                        auto& pr = b.pairs[pi];
                                        if (pr.p != p) continue;
                                        pr.stride = st;
                                        int64_t n0 = b.len[pr.p], n1 = b.len[pr.q];
                                        st *= pr.kind == 1 ? n0 * (n0 - 1) / 2 : n0 * n1;
                                    } else {
                                        b.stride[p] = st;
                                        st *= b.len[p];
                                    }
                                }
                                b.size = st;
                                b.offset = offset;
                                offset += st;
                                sc.block_of[irr] = (int)sc.blocks.size();
                                sc.blocks.push_back(b);
                            }
                        }
                        int i = 0;
                        for (; i < T->ndim; i++) {
                            if (++irr[i] < nirr) break;
                            irr[i] = 0;
                        }
                        if (i == T->ndim) break;
                    }
                    T->cases.push_back(sc);
                }
    T->total = offset;
    T->data = (double*)dmalloc(std::max<int64_t>(offset, 1) * sizeof(double));
    if (!host_only) CCSD_CUDA(cudaMemsetAsync(T->data, 0, std::max<int64_t>(offset, 1) * sizeof(double), stream));
    int h = next_handle++;
    tensors[h] = std::move(T);
    return h;
}

void Context::destroy_tensor(int h) {
    Tensor& T = tensor(h);
    // drop cached plans that mention this tensor
    for (auto it = plan_cache.begin(); it != plan_cache.end();) {
        bool uses = false;
        for (auto& g : it->second->gemms) uses |= g.tA == h || g.tB == h || g.tC == h;
        for (auto& g : it->second->sums) uses |= g.tA == h || g.tC == h;
        for (auto& g : it->second->scales) uses |= g.tC == h;
        for (auto& g : it->second->dots) uses |= g.tA == h || g.tB == h;
        if (uses) {
            release(*it->second);
            it = plan_cache.erase(it);
        } else {
            ++it;
        }
    }
    // drop cached slices of this tensor
    for (auto it = split_cache.begin(); it != split_cache.end();) {
        if (split_owner[it->first] == h) {
            free_sliced(it->second);
            split_owner.erase(it->first);
            it = split_cache.erase(it);
        } else {
            ++it;
        }
    }
    constant_tensors.erase(std::remove(constant_tensors.begin(), constant_tensors.end(), h), constant_tensors.end());
    for (auto& kv : tensors)
        if (kv.second->view_of == h && kv.first != h)
            throw Error(CCSD_ERR_ARG, "tensor " + T.name + " still has views (" + kv.second->name + ")");
    if (!T.view_of) dfree(T.data, std::max<int64_t>(T.total, 1) * sizeof(double));
    tensors.erase(h);
}

int Context::create_view(const std::string& name, int hb, const int nout[2], const int nin[2], const int* perm) {
    Tensor& Bt = tensor(hb);
    if (Bt.view_of) throw Error(CCSD_ERR_ARG, "a view of a view is not supported");
    if (Bt.packed()) throw Error(CCSD_ERR_ARG, "views of packed tensors are not supported");
    auto T = std::make_unique<Tensor>();
    T->name = name;
    const int gsize[4] = {nout[0], nout[1], nin[0], nin[1]};
    for (int g = 0; g < 4; g++)
        for (int k = 0; k < gsize[g]; k++) T->group.push_back(g);
    T->ndim = (int)T->group.size();
    if (T->ndim != Bt.ndim) throw Error(CCSD_ERR_ARG, "view rank differs from its base");
    for (int s = 0; s < 2; s++) {
        T->nout[s] = nout[s];
        T->nin[s] = nin[s];
    }
    for (int p = 0; p < T->ndim; p++)
        if (group_space(T->group[p]) != group_space(Bt.group[perm[p]]))
            throw Error(CCSD_ERR_ARG, "view permutation mixes occupied and virtual positions");
    // every view group must map, in order, onto one base group (alpha-first order is kept)
    for (int p = 0; p + 1 < T->ndim; p++)
        if (T->group[p] == T->group[p + 1] &&
            (Bt.group[perm[p]] != Bt.group[perm[p + 1]] || perm[p + 1] != perm[p] + 1))
            throw Error(CCSD_ERR_ARG, "view permutation splits an antisymmetric group");
    for (auto& bc : Bt.cases) {
        SpinCase sc;
        sc.spin.resize(T->ndim);
        for (int p = 0; p < T->ndim; p++) {
            sc.spin[p] = bc.spin[perm[p]];
            if (sc.spin[p] == ALPHA) sc.alpha[T->group[p]]++;
        }
        for (auto& bb : bc.blocks) {
            Block b;
            b.irrep.resize(T->ndim);
            b.len.resize(T->ndim);
            b.stride.resize(T->ndim);
            for (int p = 0; p < T->ndim; p++) {
                b.irrep[p] = bb.irrep[perm[p]];
                b.len[p] = bb.len[perm[p]];
                b.stride[p] = bb.stride[perm[p]];
            }
            b.offset = bb.offset;
            b.size = bb.size;
            sc.block_of[b.irrep] = (int)sc.blocks.size();
            sc.blocks.push_back(b);
        }
        T->cases.push_back(sc);
    }
    T->data = Bt.data;
    T->total = Bt.total;
    T->view_of = hb;
    int h = next_handle++;
    tensors[h] = std::move(T);
    return h;
}

// ---------------------------------------------------------------------------
// executor
// ---------------------------------------------------------------------------

std::pair<cudaEvent_t, cudaEvent_t> Context::prof_begin() {
    cudaEvent_t e0, e1;
    if (event_pool.size() >= 2) {
        e0 = event_pool.back();
        event_pool.pop_back();
        e1 = event_pool.back();
        event_pool.pop_back();
    } else {
        CCSD_CUDA(cudaEventCreate(&e0));
        CCSD_CUDA(cudaEventCreate(&e1));
    }
    CCSD_CUDA(cudaEventRecord(e0, stream));
    return {e0, e1};
}

void Context::prof_end(std::pair<cudaEvent_t, cudaEvent_t> ev, const std::string& label, double flops) {
    CCSD_CUDA(cudaEventRecord(ev.second, stream));
    pending.push_back({label, ev});
    pending_flops.push_back(flops);
}

// fold recorded event pairs into per-statement totals (synchronises the stream)
void Context::collect_profile() {
    CCSD_CUDA(cudaStreamSynchronize(stream));
    for (size_t i = 0; i < pending.size(); i++) {
        float ms = 0;
        CCSD_CUDA(cudaEventElapsedTime(&ms, pending[i].second.first, pending[i].second.second));
        auto& e = profile[pending[i].first];
        e.launches++;
        e.ms += ms;
        e.flops += pending_flops[i];
        event_pool.push_back(pending[i].second.first);
        event_pool.push_back(pending[i].second.second);
    }
    pending.clear();
    pending_flops.clear();
}

void Context::upload(Plan& p) {
    bool any = false;
    if (p.scratch_elems > 0 && !p.scratch) p.scratch = (double*)dmalloc(p.scratch_elems * sizeof(double));
    // split-K workspace of the FP64 GEMM, grown before any capture
    int64_t need = 0;
    for (auto& g : p.gemms) {
        int ks = kern::fp64_ksplit(g.M, g.N, g.K, !fp64_tiled_only);
        if (ks > 1) need = std::max<int64_t>(need, (int64_t)ks * g.M * g.N);
        // split-precision GEMMs share the space (every scheme a refinement may reach)
        for (int kind : {kern::SLICE_BF16, kern::SLICE_INT8})
            for (int ns = 3; ns <= 5; ns++) {
                if (!kern::slice_scheme_ok(kind, ns)) continue;
                const int kss = kern::split_ksplit(g.M, g.N, g.K, ns, kind);
                if (kss > 1) need = std::max<int64_t>(need, (int64_t)kss * g.M * g.N);
            }
    }
    if (need > splitk_elems) {
        if (splitk_ws) dfree(splitk_ws, splitk_elems * sizeof(double));
        splitk_ws = (double*)dmalloc(need * sizeof(double));
        splitk_elems = need;
    }
    // every table of the steps not yet uploaded goes into ONE device buffer with one copy:
    // a symmetry-blocked plan has hundreds of thousands of tables, and an allocation and a
    // copy per table cost seconds alone and minutes when several solves share the driver
    {
        int64_t total = 0;
        auto count = [&](const std::vector<int64_t>& h) { total += (int64_t)h.size(); };
        for (auto& g : p.gemms) {
            if (g.dAm) continue;
            count(g.hAm);
            count(g.hAk);
            count(g.hBk);
            count(g.hBn);
            for (int v = 0; v < g.nvm; v++) count(g.hCm[v]);
            for (int v = 0; v < g.nvn; v++) count(g.hCn[v]);
        }
        if (total > 0) {
            int64_t* d = (int64_t*)dmalloc(total * sizeof(int64_t));
            p.table_pool.push_back({d, total * sizeof(int64_t)});
            std::vector<int64_t> host;
            host.reserve(total);
            auto place = [&](const std::vector<int64_t>& h) -> int64_t* {
                if (h.empty()) return nullptr;
                int64_t* at = d + host.size();
                host.insert(host.end(), h.begin(), h.end());
                return at;
            };
            for (auto& g : p.gemms) {
                if (g.dAm) continue;
                g.dAm = place(g.hAm);
                g.dAk = place(g.hAk);
                g.dBk = place(g.hBk);
                g.dBn = place(g.hBn);
                for (int v = 0; v < g.nvm; v++) g.dCm[v] = place(g.hCm[v]);
                for (int v = 0; v < g.nvn; v++) g.dCn[v] = place(g.hCn[v]);
            }
            if (!host_only) {
                CCSD_CUDA(cudaMemcpyAsync(d, host.data(), total * sizeof(int64_t), cudaMemcpyHostToDevice, stream));
                CCSD_CUDA(cudaStreamSynchronize(stream));   // the staging vector goes out of scope
            }
        }
    }
    for (auto& g : p.gemms) {
        if (g.uploaded) continue;
        g.uploaded = true;
        any = true;
        // k tables that are arithmetic progressions let the kernels compute the offsets
        auto affine = [](const std::vector<int64_t>& t, int64_t& b0, int64_t& st) {
            if (t.empty()) return false;
            b0 = t[0];
            st = t.size() > 1 ? t[1] - t[0] : 0;
            for (size_t k = 2; k < t.size(); k++)
                if (t[k] - t[k - 1] != st) return false;
            return true;
        };
        g.ak_affine = affine(g.hAk, g.ak0, g.ak_step);
        g.bk_affine = affine(g.hBk, g.bk0, g.bk_step);
    }
    // tables are uploaded from pageable host memory; make sure the copies have been
    // staged before the host vectors could change
    if (split_precision() && !p.split_reserved && (host_only || kern::split_supported())) {
        reserve_split(p);
        p.split_reserved = true;
    }
    (void)any;   // staged copies need no synchronisation (the host tables stay with the plan)
}

void Context::release(Plan& p) {
    if (p.scratch) dfree(p.scratch, p.scratch_elems * sizeof(double));
    p.scratch = nullptr;
    for (auto& t : p.table_pool) dfree(t.first, t.second);
    p.table_pool.clear();
    for (auto& g : p.gemms) {
        g.dAm = g.dAk = g.dBk = g.dBn = nullptr;
        for (int v = 0; v < 2; v++) g.dCm[v] = g.dCn[v] = nullptr;
        g.uploaded = false;
        // cached slices belong to the plan's contraction, not to the operand tensor alone
        drop_split_cache(g);
    }
    for (auto& kv : p.schedules)
        for (auto& r : kv.second.runs)
            for (auto& l : r.launches) {
                if (l.d_probs) dfree(l.d_probs, l.nprob * sizeof(kern::GemmArgs));
                if (l.d_part) dfree(l.d_part, l.part_elems * sizeof(double));
                if (l.d_tile_start)
                    dfree(l.d_tile_start, (l.kind == GemmLaunch::FOLD_GROUPS ? l.ngroups + 1 : l.nprob) * sizeof(int));
                if (l.d_desc) dfree(l.d_desc, l.desc_bytes);
                if (l.d_chunks) dfree(l.d_chunks, l.nprob * sizeof(int64_t));
                if (l.arena) dfree(l.arena, l.arena_bytes);
                if (l.aux) dfree(l.aux, l.aux_bytes);
                if (l.merged) free_merged(*l.merged);
            }
    p.schedules.clear();
}

double* Context::data_of(Plan& p, int h) {
    if (h == kScratch) {
        if (!p.scratch) throw Error(CCSD_ERR_PLAN, "plan scratch not allocated");
        return p.scratch;
    }
    return tensor(h).data;
}

void Context::run_gemm(Plan& p, GemmStep& g) {
    kern::GemmArgs a = gemm_args(p, g);
    if (split_precision() && kern::split_supported()) {
        run_split_gemm(g, a);
    } else {
        kern::gemm_fp64(a, stream);
    }
}

kern::GemmArgs Context::gemm_args(Plan& p, const GemmStep& g) {
    kern::GemmArgs a;
    a.A = data_of(p, g.tA);
    a.B = data_of(p, g.tB);
    a.C = data_of(p, g.tC);
    a.M = g.M;
    a.N = g.N;
    a.K = g.K;
    a.alpha = g.alpha;
    a.Am = g.dAm;
    a.Ak = g.dAk;
    a.Bk = g.dBk;
    a.Bn = g.dBn;
    a.Cm[0] = g.dCm[0];
    a.Cm[1] = g.dCm[1];
    a.Cn[0] = g.dCn[0];
    a.Cn[1] = g.dCn[1];
    a.nvm = g.nvm;
    a.nvn = g.nvn;
    for (int i = 0; i < 4; i++) a.vsign[i] = g.vsign[i];
    a.a_kcontig = g.a_kcontig;
    a.b_kcontig = g.b_kcontig;
    a.ws = splitk_ws;
    a.ws_elems = splitk_elems;
    a.skinny_ok = !fp64_tiled_only;
    a.ak_affine = g.ak_affine;
    a.bk_affine = g.bk_affine;
    a.ak0 = g.ak0;
    a.ak_step = g.ak_step;
    a.bk0 = g.bk0;
    a.bk_step = g.bk_step;
    return a;
}

// Grouped schedule of a plan under the current routing.  A run is a maximal sequence of
// GEMM steps of one statement: they read only the statement's operands and write its
// output (or the plan scratch), so the only hazard among them is two writes to one
// output block.  Each step gets a level one above the last level that wrote any of its
// output blocks; within a level the small FP64 products (fewer than a wave of tiles, no
// split-K) become one grouped launch per operand contiguity, the rest launch alone.
// Every output block thus receives its contributions in plan order.  Runs of permuted
// sums (antisymmetriser images, copies) and of block scalings of one statement are
// batched the same way, one launch per level.
RunSchedule& Context::schedule(Plan& p) {
    const int key = (split_precision() ? 1 : 0) | (split_routing << 1) | (fp64_tiled_only ? 4 : 0) |
                    (group_gemms ? 8 : 0) | (precision == CCSD_PREC_SPLIT_I8 ? 16 : 0);
    auto it = p.schedules.find(key);
    if (it != p.schedules.end()) return it->second;
    RunSchedule& rs = p.schedules[key];
    rs.run_at.assign(p.steps.size(), -1);
    if (!group_gemms || host_only) return rs;
    auto label_of = [&](const Step& st) -> const std::string& {
        switch (st.kind) {
            case Step::GEMM: return p.gemms[st.idx].label;
            case Step::SUM: return p.sums[st.idx].label;
            case Step::SCALE: return p.scales[st.idx].label;
            default: {
                static const std::string none;
                return none;
            }
        }
    };
    size_t s = 0;
    while (s < p.steps.size()) {
        const Step::Kind kind = p.steps[s].kind;
        if (kind == Step::DOT) {
            size_t e = s;
            while (e < p.steps.size() && p.steps[e].kind == Step::DOT) e++;
            if (e - s >= 2) build_dot_run(p, rs, (int)s, (int)e);
            s = e;
            continue;
        }
        const std::string& lab = label_of(p.steps[s]);
        size_t e = s;
        while (e < p.steps.size() && p.steps[e].kind == kind && label_of(p.steps[e]) == lab) e++;
        if (e - s >= 2) {
            if (kind == Step::GEMM) build_run(p, rs, (int)s, (int)e);
            else build_elementwise_run(p, rs, (int)s, (int)e);
        }
        s = e;
    }
    return rs;
}

void Context::build_run(Plan& p, RunSchedule& rs, int first, int end) {
    // output block of an element offset: (buffer, start of the block containing it)
    std::map<int, std::vector<int64_t>> starts;
    auto block_of = [&](int h, int64_t off) -> std::pair<int, int64_t> {
        if (h == kScratch) return {h, off};   // a product region starts at its lowest offset
        auto& v = starts[h];
        if (v.empty()) {
            for (auto& sc : tensor(h).cases)
                for (auto& b : sc.blocks) v.push_back(b.offset);
            std::sort(v.begin(), v.end());
        }
        auto ub = std::upper_bound(v.begin(), v.end(), off);
        return {h, ub == v.begin() ? 0 : *(ub - 1)};
    };
    // small products (less than a wave of tiles; either little work or no split-K on
    // their own) gain from sharing a launch; larger ones keep their own kernel choice
    auto groupable = [&](const GemmStep& g) {
        if (routes_split(g) || g.M <= 0 || g.N <= 0 || g.K <= 0) return false;
        if (kern::fp64_tiles(g.M, g.N) >= 148) return false;
        // a skinny product (one extent <= 32) with a long operand of 4M elements or more is
        // bandwidth work for the skinny kernel: on a 128 x 64 tile it would use 1/64 to 1/2
        // of every tile (F(ae) += <am||ef> t(fm) at o=16 v=128: 2.3 ms grouped)
        if (!fp64_tiled_only && std::min(g.M, g.N) <= 32 && (int64_t)std::max(g.M, g.N) * g.K >= (int64_t)1 << 22)
            return false;
        // and so is a skinny product with a long side of a tile or more: the grouped skinny
        // launch streams it (the tiles would stay 1/8 to 1/2 empty and walk it at a fraction
        // of the rate: W~(am,ei) += <am||ef> t(fi) at o=48 v=336 D2h took 16 ms on tiles)
        if (!fp64_tiled_only && std::min(g.M, g.N) <= 32 && std::max(g.M, g.N) >= 128) return false;
        // a grouped tile walks the whole K range: long-K products keep their split-K launch
        if (g.flops() < 4e8 && g.K <= 4096) return true;
        return kern::fp64_ksplit(g.M, g.N, g.K, !fp64_tiled_only) == 1 && kern::fp64_ksplit(g.M, g.N, g.K, false) == 1;
    };
    // short products (both extents <= 64, long K) compute partials on the short kernel and
    // join the fold below, whatever their levels
    // (CCSD_SHORT_MIN_K: the shortest K that takes them, default 512; coverage tests lower it)
    const int short_min_k = std::getenv("CCSD_SHORT_MIN_K") ? std::atoi(std::getenv("CCSD_SHORT_MIN_K")) : 512;
    auto shortable = [&](const GemmStep& g) {
        return !fp64_tiled_only && !routes_split(g) && g.K >= short_min_k && kern::short_shape(g.M, g.N).first > 0;
    };
    // skinny products without a K split share one launch per level and shape
    auto skinny_groupable = [&](const GemmStep& g) {
        return !fp64_tiled_only && !routes_split(g) && !groupable(g) && kern::skinny_groups(g.M, g.N) > 0 &&
               kern::fp64_ksplit(g.M, g.N, g.K, true) == 1;
    };
    int nskinny = 0;
    std::map<std::pair<int, int64_t>, int> last;
    std::vector<int> level(end - first, 0);
    std::vector<std::pair<int, int64_t>> key1(end - first, {0, -1});   // the block of a one-destination step
    std::vector<std::vector<std::pair<int, int64_t>>> keys_of(end - first);   // every output block of a step
    int nshort = 0;
    int maxlvl = 0;
    int ngroupable = 0;
    for (int i = first; i < end; i++) {
        const GemmStep& g = p.gemms[p.steps[i].idx];
        std::vector<std::pair<int, int64_t>> keys;
        for (int v = 0; v < g.nvm; v++)
            for (int w = 0; w < g.nvn; w++) {
                if (g.hCm[v].empty() || g.hCn[w].empty()) continue;
                const int64_t lo = *std::min_element(g.hCm[v].begin(), g.hCm[v].end()) +
                                   *std::min_element(g.hCn[w].begin(), g.hCn[w].end());
                keys.push_back(block_of(g.tC, lo));
            }
        int lvl = 0;
        for (auto& k : keys) {
            auto f = last.find(k);
            if (f != last.end()) lvl = std::max(lvl, f->second + 1);
        }
        for (auto& k : keys) last[k] = lvl;
        level[i - first] = lvl;
        if (keys.size() == 1) key1[i - first] = keys[0];
        keys_of[i - first] = keys;
        maxlvl = std::max(maxlvl, lvl);
        if (groupable(g)) ngroupable++;
        if (shortable(g)) nshort++;
        if (!fp64_tiled_only && !routes_split(g) && kern::skinny_groups(g.M, g.N) > 0) nskinny++;
    }
    GemmRun run;
    run.first = first;
    run.end = end;
    bool any_group = false;
    // the block products of one irrep class as one split GEMM (symmetry-blocked statements)
    std::vector<char> merged(end - first, 0);
    // CCSD_MERGED=0: no merged products (coverage tests)
    const bool merge_on = !std::getenv("CCSD_MERGED") || std::getenv("CCSD_MERGED")[0] != '0';
    if (merge_on && precision == CCSD_PREC_SPLIT_I8 && kern::split_supported() && spaces.nirrep > 1 &&
        split_routing != CCSD_SPLIT_ROUTE_ALL) {
        build_merged(p, run, first, end, merged, block_of);
        any_group = !run.launches.empty();
        ngroupable = 0;
        for (int i = first; i < end; i++)
            if (!merged[i - first] && groupable(p.gemms[p.steps[i].idx])) ngroupable++;
    }
    if (!any_group && ngroupable < 2 && nshort == 0 && nskinny < 2) return;

    // Shared-output groups.  Small one-destination products that several levels would
    // serialise (block contractions of a symmetry-blocked statement summing into the same
    // output blocks over their internal irreps) run as one grouped launch per operand
    // contiguity writing dense partial products, and the short products as one launch per
    // fragment shape writing a partial per CTA; then one fold launch: a CTA per group of
    // output blocks (products that share a block, antisymmetriser variants included, fall in
    // one group) adds its products in plan order (deterministic).
    std::vector<char> in_fold(end - first, 0);   // 1: tile partial, 2: short partials
    {
        int nfold = 0;
        bool multi = false;
        int64_t part = 0;
        for (int i = first; i < end; i++) {
            const GemmStep& g = p.gemms[p.steps[i].idx];
            if (merged[i - first] || shortable(g) || !groupable(g) || g.nvm != 1 || g.nvn != 1 ||
                key1[i - first].second < 0)
                continue;
            if ((int64_t)g.M * g.N > 65536) continue;
            in_fold[i - first] = 1;
            nfold++;
            multi |= level[i - first] > 0;
            part += (int64_t)g.M * g.N;
        }
        if (nfold < 2 || !multi || part > (32ll << 20)) {
            std::fill(in_fold.begin(), in_fold.end(), 0);
            part = 0;
        }
        std::vector<int> sctas(end - first, 0), skper(end - first, 0);
        for (int i = first; i < end; i++) {
            const GemmStep& g = p.gemms[p.steps[i].idx];
            if (merged[i - first] || !shortable(g) || keys_of[i - first].empty()) continue;
            in_fold[i - first] = 2;
            sctas[i - first] = kern::short_ctas(g.K, &skper[i - first]);
            part += (int64_t)sctas[i - first] * g.M * g.N;
        }
        // skinny products that split K write their K ranges' partials for the fold too (one
        // grouped launch instead of a skinny launch and a fold launch per product), within a
        // partial buffer of 64M elements
        int64_t skpart = 0;
        for (int i = first; i < end; i++) {
            const GemmStep& g = p.gemms[p.steps[i].idx];
            if (in_fold[i - first] || merged[i - first] || fp64_tiled_only || routes_split(g) ||
                kern::skinny_groups(g.M, g.N) == 0 || keys_of[i - first].empty())
                continue;
            // (small outputs only: one CTA folds a group, so a large partial stays with the
            // product's own launch and its parallel fold)
            const int ks = kern::fp64_ksplit(g.M, g.N, g.K, true);
            const int64_t mn = (int64_t)g.M * g.N;
            if (ks < 2 || mn > 16384 || ks * mn > 262144 || skpart + ks * mn > (64ll << 20)) continue;
            in_fold[i - first] = 3;
            sctas[i - first] = ks;
            skpart += (int64_t)ks * g.M * g.N;
        }
        part += skpart;
        if (std::any_of(in_fold.begin(), in_fold.end(), [](char c) { return c != 0; })) {
            double* d_part = (double*)dmalloc(std::max<int64_t>(part, 1) * sizeof(double));
            bool owner = true;   // the partial buffer is owned by the first launch
            auto own = [&](GemmLaunch& l) {
                if (!owner) return;
                l.d_part = d_part;
                l.part_elems = std::max<int64_t>(part, 1);
                owner = false;
            };
            int64_t off = 0;
            std::vector<kern::GemmArgs> probs[4];
            std::vector<int> tstart[4];
            int tiles[4] = {0, 0, 0, 0};
            double fl[4] = {0, 0, 0, 0};
            std::map<std::pair<int, int>, std::vector<kern::ShortDesc>> sprobs;
            std::map<std::pair<int, int>, std::vector<int>> sstart;
            std::map<std::pair<int, int>, int> sctas_total;
            std::map<std::pair<int, int>, double> sfl;
            std::map<std::pair<int, bool>, std::vector<kern::SkinnyArgs>> kprobs;
            std::map<std::pair<int, bool>, std::vector<int>> kstart;
            std::map<std::pair<int, bool>, int> ktiles;
            std::map<std::pair<int, bool>, double> kfl;
            std::vector<kern::FoldDesc> fdesc(end - first);
            for (int i = first; i < end; i++) {
                if (!in_fold[i - first]) continue;
                const GemmStep& g = p.gemms[p.steps[i].idx];
                kern::GemmArgs a = gemm_args(p, g);
                kern::FoldDesc& f = fdesc[i - first];
                f.part = d_part + off;
                f.C = a.C;
                for (int v = 0; v < 2; v++) {
                    f.Cm[v] = a.Cm[v];
                    f.Cn[v] = a.Cn[v];
                }
                f.nvm = a.nvm;
                f.nvn = a.nvn;
                for (int v = 0; v < 4; v++) f.vsign[v] = a.vsign[v];
                f.M = g.M;
                f.N = g.N;
                f.scale = a.alpha;
                if (in_fold[i - first] == 1) {
                    a.ws = d_part + off;
                    a.ws_elems = (int64_t)g.M * g.N;
                    a.partial_out = true;
                    off += (int64_t)g.M * g.N;
                    const int c = (g.a_kcontig ? 2 : 0) + (g.b_kcontig ? 1 : 0);
                    probs[c].push_back(a);
                    tstart[c].push_back(tiles[c]);
                    tiles[c] += kern::fp64_tiles(g.M, g.N);
                    fl[c] += g.flops();
                } else if (in_fold[i - first] == 3) {
                    bool lk;
                    kern::SkinnyArgs k = kern::skinny_args(a, &lk);
                    k.nz = sctas[i - first];
                    k.partial = true;
                    k.ws = d_part + off;
                    // the partials are [z][long extent][short extent]: fold in that orientation
                    f.M = k.R;
                    f.N = k.NS;
                    for (int v = 0; v < 2; v++) {
                        f.Cm[v] = k.Cr[v];
                        f.Cn[v] = k.Cs[v];
                    }
                    f.nvm = k.nvr;
                    f.nvn = k.nvs;
                    for (int v = 0; v < 4; v++) f.vsign[v] = k.vsign[v];
                    f.scale = k.alpha;
                    f.ks = k.nz;
                    off += (int64_t)k.nz * k.R * k.NS;
                    const std::pair<int, bool> cls{kern::skinny_groups(g.M, g.N), lk};
                    kstart[cls].push_back(ktiles[cls]);
                    ktiles[cls] += kern::skinny_tiles(k.R) * k.nz;
                    kprobs[cls].push_back(k);
                    kfl[cls] += g.flops();
                } else {
                    const auto shape = kern::short_shape(g.M, g.N);
                    kern::ShortDesc d;
                    d.A = a.A;
                    d.B = a.B;
                    d.Am = a.Am;
                    d.Ak = a.Ak;
                    d.Bk = a.Bk;
                    d.Bn = a.Bn;
                    d.ak_affine = a.ak_affine;
                    d.bk_affine = a.bk_affine;
                    d.ak0 = a.ak0;
                    d.ak_step = a.ak_step;
                    d.bk0 = a.bk0;
                    d.bk_step = a.bk_step;
                    d.M = g.M;
                    d.N = g.N;
                    d.K = g.K;
                    d.kper = skper[i - first];
                    d.part = d_part + off;
                    f.ks = sctas[i - first];
                    off += (int64_t)f.ks * g.M * g.N;
                    sstart[shape].push_back(sctas_total[shape]);
                    sctas_total[shape] += f.ks;
                    sprobs[shape].push_back(d);
                    sfl[shape] += g.flops();
                }
            }
            for (int c = 0; c < 4; c++) {
                if (probs[c].empty()) continue;
                GemmLaunch l;
                l.kind = GemmLaunch::GEMM_GROUPED;
                l.ak = (c & 2) != 0;
                l.bk = (c & 1) != 0;
                l.nprob = (int)probs[c].size();
                l.tiles = tiles[c];
                l.flops = fl[c];
                own(l);
                l.d_probs = (kern::GemmArgs*)dmalloc(probs[c].size() * sizeof(kern::GemmArgs));
                l.d_tile_start = (int*)dmalloc(tstart[c].size() * sizeof(int));
                stage_h2d(l.d_probs, probs[c].data(), probs[c].size() * sizeof(kern::GemmArgs));
                stage_h2d(l.d_tile_start, tstart[c].data(), tstart[c].size() * sizeof(int));
                run.launches.push_back(l);
            }
            for (auto& kv : sprobs) {
                GemmLaunch l;
                l.kind = GemmLaunch::SHORT_GROUPED;
                l.mt = kv.first.first;
                l.nt = kv.first.second;
                l.nprob = (int)kv.second.size();
                l.tiles = sctas_total[kv.first];
                l.flops = sfl[kv.first];
                own(l);
                l.desc_bytes = kv.second.size() * sizeof(kern::ShortDesc);
                l.d_desc = dmalloc(l.desc_bytes);
                l.d_tile_start = (int*)dmalloc(kv.second.size() * sizeof(int));
                stage_h2d(l.d_desc, kv.second.data(), l.desc_bytes);
                stage_h2d(l.d_tile_start, sstart[kv.first].data(), kv.second.size() * sizeof(int));
                run.launches.push_back(l);
            }
            for (auto& kv : kprobs) {
                GemmLaunch l;
                l.kind = GemmLaunch::SKINNY_GROUPED;
                l.nt = kv.first.first;
                l.ak = kv.first.second;
                l.nprob = (int)kv.second.size();
                l.tiles = ktiles[kv.first];
                l.flops = kfl[kv.first];
                own(l);
                l.desc_bytes = kv.second.size() * sizeof(kern::SkinnyArgs);
                l.d_desc = dmalloc(l.desc_bytes);
                l.d_tile_start = (int*)dmalloc(kv.second.size() * sizeof(int));
                stage_h2d(l.d_desc, kv.second.data(), l.desc_bytes);
                stage_h2d(l.d_tile_start, kstart[kv.first].data(), kv.second.size() * sizeof(int));
                run.launches.push_back(l);
            }
            // groups: products connected through a shared output block, in plan order
            std::map<std::pair<int, int64_t>, int> bid;
            std::vector<int> par;
            auto find = [&](int x) {
                while (par[x] != x) x = par[x] = par[par[x]];
                return x;
            };
            for (int i = first; i < end; i++) {
                if (!in_fold[i - first]) continue;
                int root = -1;
                for (auto& k : keys_of[i - first]) {
                    auto it = bid.find(k);
                    int b;
                    if (it == bid.end()) {
                        b = (int)par.size();
                        par.push_back(b);
                        bid.emplace(k, b);
                    } else {
                        b = it->second;
                    }
                    if (root < 0) root = find(b);
                    else {
                        const int rb = find(b);
                        if (rb != root) par[rb] = root;
                    }
                }
            }
            std::map<int, std::vector<int>> members;
            std::vector<int> group_order;
            for (int i = first; i < end; i++) {
                if (!in_fold[i - first]) continue;
                const int r = find(bid.at(keys_of[i - first][0]));
                if (!members.count(r)) group_order.push_back(r);
                members[r].push_back(i - first);
            }
            std::vector<kern::FoldDesc> descs;
            std::vector<int> gstart;
            for (int r : group_order) {
                gstart.push_back((int)descs.size());
                for (int j : members[r]) descs.push_back(fdesc[j]);
            }
            gstart.push_back((int)descs.size());
            GemmLaunch fl_l;
            fl_l.kind = GemmLaunch::FOLD_GROUPS;
            fl_l.nprob = (int)descs.size();
            fl_l.ngroups = (int)group_order.size();
            fl_l.desc_bytes = descs.size() * sizeof(kern::FoldDesc);
            fl_l.d_desc = dmalloc(fl_l.desc_bytes);
            fl_l.d_tile_start = (int*)dmalloc(gstart.size() * sizeof(int));
            stage_h2d(fl_l.d_desc, descs.data(), fl_l.desc_bytes);
            stage_h2d(fl_l.d_tile_start, gstart.data(), gstart.size() * sizeof(int));
            run.launches.push_back(fl_l);
            any_group = true;
        }
    }

    for (int L = 0; L <= maxlvl; L++) {
        std::vector<int> grp[4];
        std::map<std::pair<int, bool>, std::vector<int>> sk;
        for (int i = first; i < end; i++) {
            if (level[i - first] != L || in_fold[i - first] || merged[i - first]) continue;
            const int gi = p.steps[i].idx;
            const GemmStep& g = p.gemms[gi];
            if (groupable(g)) {
                grp[(g.a_kcontig ? 2 : 0) + (g.b_kcontig ? 1 : 0)].push_back(gi);
            } else if (skinny_groupable(g)) {
                const bool lk = g.M >= g.N ? g.a_kcontig : g.b_kcontig;
                sk[{kern::skinny_groups(g.M, g.N), lk}].push_back(gi);
            } else {
                GemmLaunch l;
                l.gemm = gi;
                l.flops = g.flops();
                run.launches.push_back(l);
            }
        }
        for (int c = 0; c < 4; c++) {
            if (grp[c].empty()) continue;
            if (grp[c].size() == 1) {
                GemmLaunch l;
                l.gemm = grp[c][0];
                l.flops = p.gemms[grp[c][0]].flops();
                run.launches.push_back(l);
                continue;
            }
            GemmLaunch l;
            l.kind = GemmLaunch::GEMM_GROUPED;
            l.ak = (c & 2) != 0;
            l.bk = (c & 1) != 0;
            std::vector<kern::GemmArgs> probs;
            std::vector<int> tstart;
            int tiles = 0;
            for (int gi : grp[c]) {
                const GemmStep& g = p.gemms[gi];
                kern::GemmArgs a = gemm_args(p, g);
                a.ws = nullptr;
                a.ws_elems = 0;
                probs.push_back(a);
                tstart.push_back(tiles);
                tiles += kern::fp64_tiles(g.M, g.N);
                l.flops += g.flops();
            }
            l.nprob = (int)probs.size();
            l.tiles = tiles;
            l.d_probs = (kern::GemmArgs*)dmalloc(probs.size() * sizeof(kern::GemmArgs));
            l.d_tile_start = (int*)dmalloc(tstart.size() * sizeof(int));
            stage_h2d(l.d_probs, probs.data(), probs.size() * sizeof(kern::GemmArgs));
            stage_h2d(l.d_tile_start, tstart.data(), tstart.size() * sizeof(int));
            run.launches.push_back(l);
            any_group = true;
        }
        for (auto& kv : sk) {
            if (kv.second.size() == 1) {
                GemmLaunch l;
                l.gemm = kv.second[0];
                l.flops = p.gemms[kv.second[0]].flops();
                run.launches.push_back(l);
                continue;
            }
            GemmLaunch l;
            l.kind = GemmLaunch::SKINNY_GROUPED;
            l.nt = kv.first.first;
            l.ak = kv.first.second;
            std::vector<kern::SkinnyArgs> probs;
            std::vector<int> tstart;
            int tiles = 0;
            for (int gi : kv.second) {
                const GemmStep& g = p.gemms[gi];
                bool lk;
                kern::SkinnyArgs a = kern::skinny_args(gemm_args(p, g), &lk);
                a.ws = nullptr;
                probs.push_back(a);
                tstart.push_back(tiles);
                tiles += kern::skinny_tiles(a.R);
                l.flops += g.flops();
            }
            l.nprob = (int)probs.size();
            l.tiles = tiles;
            l.desc_bytes = probs.size() * sizeof(kern::SkinnyArgs);
            l.d_desc = dmalloc(l.desc_bytes);
            l.d_tile_start = (int*)dmalloc(tstart.size() * sizeof(int));
            stage_h2d(l.d_desc, probs.data(), l.desc_bytes);
            stage_h2d(l.d_tile_start, tstart.data(), tstart.size() * sizeof(int));
            run.launches.push_back(l);
            any_group = true;
        }
    }
    if (!any_group) return;
    rs.run_at[first] = (int)rs.runs.size();
    rs.runs.push_back(std::move(run));
}

// A run of permuted sums or of scalings of one statement.  Sums read their A blocks (an
// operand or a product region, never written in the run) and write C blocks: each gets a
// level above the last sum into the same C block, and every level is one batched launch.
// Scalings touch distinct blocks: one launch.
void Context::build_elementwise_run(Plan& p, RunSchedule& rs, int first, int end) {
    const bool is_sum = p.steps[first].kind == Step::SUM;
    std::map<int, std::vector<int64_t>> starts;
    auto block_of = [&](int h, int64_t off) -> std::pair<int, int64_t> {
        if (h == kScratch) return {h, off};
        auto& v = starts[h];
        if (v.empty()) {
            for (auto& sc : tensor(h).cases)
                for (auto& b : sc.blocks) v.push_back(b.offset);
            std::sort(v.begin(), v.end());
        }
        auto ub = std::upper_bound(v.begin(), v.end(), off);
        return {h, ub == v.begin() ? 0 : *(ub - 1)};
    };
    std::vector<int> level(end - first, 0);
    int maxlvl = 0;
    if (is_sum) {
        std::map<std::pair<int, int64_t>, int> last;
        for (int i = first; i < end; i++) {
            const SumStep& s = p.sums[p.steps[i].idx];
            auto k = block_of(s.tC, s.offC);
            auto f = last.find(k);
            const int lvl = f == last.end() ? 0 : f->second + 1;
            last[k] = lvl;
            level[i - first] = lvl;
            maxlvl = std::max(maxlvl, lvl);
        }
    }
    GemmRun run;
    run.first = first;
    run.end = end;
    for (int L = 0; L <= maxlvl; L++) {
        std::vector<int> idx;
        for (int i = first; i < end; i++)
            if (level[i - first] == L) idx.push_back(p.steps[i].idx);
        if (idx.empty()) continue;
        GemmLaunch l;
        std::vector<int64_t> cs;
        int64_t chunks = 0;
        auto nchunks = [](int64_t n) { return (n + kern::kBatchChunk - 1) / kern::kBatchChunk; };
        if (is_sum) {
            l.kind = GemmLaunch::SUM_BATCHED;
            std::vector<kern::SumDesc> d;
            for (int k : idx) {
                const SumStep& s = p.sums[k];
                kern::SumDesc x;
                x.A = data_of(p, s.tA) + s.offA;
                x.C = data_of(p, s.tC) + s.offC;
                x.alpha = s.alpha;
                x.ndim = s.ndim;
                x.total = 1;
                for (int q = 0; q < s.ndim; q++) {
                    x.len[q] = s.len[q];
                    x.sA[q] = s.sA[q];
                    x.sC[q] = s.sC[q];
                    x.total *= s.len[q];
                }
                if (x.total <= 0) continue;
                kern::sum_plan_tiles(x);
                d.push_back(x);
                cs.push_back(chunks);
                chunks += kern::sum_chunks(x);
            }
            if (d.empty()) continue;
            l.desc_bytes = d.size() * sizeof(kern::SumDesc);
            l.d_desc = dmalloc(l.desc_bytes);
            stage_h2d(l.d_desc, d.data(), l.desc_bytes);
            l.nprob = (int)d.size();
        } else {
            l.kind = GemmLaunch::SCALE_BATCHED;
            std::vector<kern::ScaleDesc> d;
            for (int k : idx) {
                const ScaleStep& s = p.scales[k];
                if (s.n <= 0) continue;
                kern::ScaleDesc x;
                x.X = data_of(p, s.tC) + s.off;
                x.n = s.n;
                x.beta = s.beta;
                d.push_back(x);
                cs.push_back(chunks);
                chunks += nchunks(x.n);
            }
            if (d.empty()) continue;
            l.desc_bytes = d.size() * sizeof(kern::ScaleDesc);
            l.d_desc = dmalloc(l.desc_bytes);
            stage_h2d(l.d_desc, d.data(), l.desc_bytes);
            l.nprob = (int)d.size();
        }
        if (chunks > INT32_MAX) throw Error(CCSD_ERR_PLAN, "batched launch too large");
        l.chunks = chunks;
        l.d_chunks = (int64_t*)dmalloc(cs.size() * sizeof(int64_t));
        stage_h2d(l.d_chunks, cs.data(), cs.size() * sizeof(int64_t));
        run.launches.push_back(l);
    }
    rs.run_at[first] = (int)rs.runs.size();
    rs.runs.push_back(std::move(run));
}

// A run of dots (the energy and other scalars): one launch of per-chunk partial dots and
// one fixed-order fold into the run's accumulator.
void Context::build_dot_run(Plan& p, RunSchedule& rs, int first, int end) {
    std::vector<kern::DotDesc> descs;
    std::vector<int64_t> cs;
    int64_t chunks = 0;
    for (int i = first; i < end; i++) {
        const DotStep& d = p.dots[p.steps[i].idx];
        kern::DotDesc x;
        x.A = tensor(d.tA).data + d.offA;
        x.B = tensor(d.tB).data + d.offB;
        x.ndim = d.ndim;
        x.total = 1;
        for (int k = 0; k < d.ndim; k++) {
            x.len[k] = d.len[k];
            x.sA[k] = d.sA[k];
            x.sB[k] = d.sB[k];
            x.total *= d.len[k];
        }
        x.alpha = d.alpha;
        if (x.total <= 0) continue;
        kern::plan_divisors(x.len, x.ndim, x.total, x.fast, x.dmul, x.dshr);
        descs.push_back(x);
        cs.push_back(chunks);
        chunks += (x.total + kern::kBatchChunk - 1) / kern::kBatchChunk;
    }
    if (descs.size() < 2) return;
    GemmLaunch l;
    l.kind = GemmLaunch::DOT_BATCHED;
    l.nprob = (int)descs.size();
    l.chunks = chunks;
    l.desc_bytes = descs.size() * sizeof(kern::DotDesc);
    l.d_desc = dmalloc(l.desc_bytes);
    l.d_chunks = (int64_t*)dmalloc(cs.size() * sizeof(int64_t));
    l.d_part = (double*)dmalloc(chunks * sizeof(double));
    l.part_elems = chunks;
    stage_h2d(l.d_desc, descs.data(), l.desc_bytes);
    stage_h2d(l.d_chunks, cs.data(), cs.size() * sizeof(int64_t));
    GemmRun run;
    run.first = first;
    run.end = end;
    run.launches.push_back(l);
    rs.run_at[first] = (int)rs.runs.size();
    rs.runs.push_back(std::move(run));
}

void Context::launch(Plan& p, const GemmLaunch& l, const std::string& label, double* dot_acc) {
    auto ev = profiling ? prof_begin() : std::make_pair((cudaEvent_t) nullptr, (cudaEvent_t) nullptr);
    switch (l.kind) {
        case GemmLaunch::MERGED_SPLIT: run_merged(p, *l.merged, label); break;
        case GemmLaunch::GEMM: run_gemm(p, p.gemms[l.gemm]); break;
        case GemmLaunch::GEMM_GROUPED:
            kern::gemm_fp64_grouped(l.d_probs, l.d_tile_start, l.nprob, l.tiles, l.ak, l.bk, stream);
            break;
        case GemmLaunch::DOT_BATCHED:
            kern::dot_batched((const kern::DotDesc*)l.d_desc, l.d_chunks, l.nprob, l.chunks, l.d_part, dot_acc, stream);
            break;
        case GemmLaunch::MERGED_SLICE:
            kern::rect_slice_batched((const kern::RectDesc*)l.d_desc, l.d_chunks, l.nprob, l.chunks,
                                     step_slices(p.gemms[l.gemm]), (uint8_t*)l.aux + l.aux_bytes / 2, l.aux_bytes / 2,
                                     stream);
            break;
        case GemmLaunch::SKINNY_GROUPED:
            kern::skinny_grouped((const kern::SkinnyArgs*)l.d_desc, l.d_tile_start, l.nprob, l.tiles, l.nt, l.ak, stream);
            break;
        case GemmLaunch::SHORT_GROUPED:
            kern::short_grouped((const kern::ShortDesc*)l.d_desc, l.d_tile_start, l.nprob, l.tiles, l.mt, l.nt, stream);
            break;
        case GemmLaunch::FOLD_GROUPS:
            kern::fold_groups((const kern::FoldDesc*)l.d_desc, l.d_tile_start, l.ngroups, stream);
            break;
        case GemmLaunch::SUM_BATCHED:
            kern::sum_batched((const kern::SumDesc*)l.d_desc, l.d_chunks, l.nprob, l.chunks, stream);
            break;
        case GemmLaunch::SCALE_BATCHED:
            kern::scale_batched((const kern::ScaleDesc*)l.d_desc, l.d_chunks, l.nprob, l.chunks, stream);
            break;
        default: throw Error(CCSD_ERR_PLAN, "bad launch record");
    }
    if (profiling) {
        // CCSD_PROFILE_KINDS=1: totals per statement and launch kind
        static const bool kinds = std::getenv("CCSD_PROFILE_KINDS") != nullptr;
        static const char* names[] = {"gemm", "grouped", "fold", "sum", "sum-batched", "scale", "scale-batched",
                                      "dot-batched", "merged", "short", "skinny-grouped", "merged-slice"};
        if (kinds) {
            std::string k = names[l.kind];
            if (l.kind == GemmLaunch::GEMM) k = routes_split(p.gemms[l.gemm]) ? "gemm-split" : "gemm-fp64";
            prof_end(ev, label + " {" + k + "}", l.flops);
        } else {
            prof_end(ev, label, l.flops);
        }
    }
}

void Context::run(Plan& p, double* scalar_out, double* dot_target) {
    upload(p);
    if (host_only) return;   // planning only: account the tables, launch nothing
    bool zeroed = dot_target != nullptr;
    double* acc = dot_target ? dot_target : d_scalar;
    RunSchedule* rs = host_only ? nullptr : &schedule(p);
    for (size_t si = 0; si < p.steps.size(); si++) {
        const Step& st = p.steps[si];
        if (rs && rs->run_at[si] >= 0) {
            GemmRun& r = rs->runs[rs->run_at[si]];
            std::string lab;
            switch (st.kind) {
                case Step::GEMM: lab = p.gemms[st.idx].label.empty() ? "gemm" : p.gemms[st.idx].label; break;
                case Step::SUM: lab = p.sums[st.idx].label.empty() ? "sum" : p.sums[st.idx].label; break;
                case Step::DOT: lab = "dot"; break;
                default: lab = p.scales[st.idx].label.empty() ? "scale" : p.scales[st.idx].label; break;
            }
            if (st.kind == Step::DOT && !zeroed) {
                CCSD_CUDA(cudaMemsetAsync(d_scalar, 0, sizeof(double), stream));
                zeroed = true;
            }
            for (auto& l : r.launches) launch(p, l, lab, acc);
            si = r.end - 1;
            continue;
        }
        switch (st.kind) {
            case Step::GEMM: {
                GemmStep& g = p.gemms[st.idx];
                if (profiling) {
                    auto ev = prof_begin();
                    run_gemm(p, g);
                    prof_end(ev, g.label.empty() ? std::string("gemm") : g.label, g.flops());
                } else {
                    run_gemm(p, g);
                }
                break;
            }
            case Step::SUM: {
                auto& s = p.sums[st.idx];
                kern::StridedArgs a;
                a.ndim = s.ndim;
                a.total = 1;
                for (int d = 0; d < s.ndim; d++) {
                    a.len[d] = s.len[d];
                    a.sA[d] = s.sA[d];
                    a.sB[d] = s.sC[d];
                    a.total *= s.len[d];
                }
                auto ev = profiling ? prof_begin() : std::make_pair((cudaEvent_t) nullptr, (cudaEvent_t) nullptr);
                kern::sum_strided(data_of(p, s.tA) + s.offA, data_of(p, s.tC) + s.offC, a, s.alpha, stream);
                if (profiling) prof_end(ev, s.label.empty() ? std::string("sum") : s.label, 0.0);
                break;
            }
            case Step::SCALE: {
                auto& s = p.scales[st.idx];
                auto ev = profiling ? prof_begin() : std::make_pair((cudaEvent_t) nullptr, (cudaEvent_t) nullptr);
                kern::scale(data_of(p, s.tC) + s.off, s.n, s.beta, stream);
                if (profiling) prof_end(ev, s.label.empty() ? std::string("scale") : s.label, 0.0);
                break;
            }
            case Step::DOT: {
                auto& d = p.dots[st.idx];
                if (!zeroed) {
                    CCSD_CUDA(cudaMemsetAsync(d_scalar, 0, sizeof(double), stream));
                    zeroed = true;
                }
                kern::StridedArgs a;
                a.ndim = d.ndim;
                a.total = 1;
                for (int k = 0; k < d.ndim; k++) {
                    a.len[k] = d.len[k];
                    a.sA[k] = d.sA[k];
                    a.sB[k] = d.sB[k];
                    a.total *= d.len[k];
                }
                kern::dot_strided(tensor(d.tA).data + d.offA, tensor(d.tB).data + d.offB, a, d.alpha, acc, stream);
                break;
            }
        }
    }
    if (scalar_out) {
        if (!zeroed) CCSD_CUDA(cudaMemsetAsync(d_scalar, 0, sizeof(double), stream));
        CCSD_CUDA(cudaMemcpyAsync(scalar_out, d_scalar, sizeof(double), cudaMemcpyDeviceToHost, stream));
        CCSD_CUDA(cudaStreamSynchronize(stream));
    }
    CCSD_CUDA(cudaGetLastError());
}

}  // namespace ccsd
