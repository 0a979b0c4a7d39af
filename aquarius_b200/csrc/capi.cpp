// extern "C" entry points (declared in include/ccsd_b200.h).  Every call converts
// engine exceptions into status codes; nothing throws across the ABI.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <sstream>

#include "diis.hpp"
#include "engine.hpp"
#include "hbuild.hpp"
#include "solver.hpp"

struct ccsd_ctx_s {
    ccsd::Context* c = nullptr;
};

struct ccsd_solver_s {
    ccsd_ctx_s* ctx = nullptr;
    ccsd::Solver* s = nullptr;
};

namespace {
thread_local std::string g_global_error;
}

namespace ccsd {
Context* from_handle(ccsd_ctx c) {
    if (!c || !c->c) throw Error(CCSD_ERR_ARG, "null context");
    return c->c;
}
// a context whose tensors have device data (not a planning-only context)
Context* device_handle(ccsd_ctx c) {
    Context* x = from_handle(c);
    if (x->host_only) throw Error(CCSD_ERR_UNSUPPORTED, "planning-only context: tensors hold no data");
    return x;
}
// message for entry points that have no context (ccsd_last_error(NULL))
void set_global_error(const std::string& msg) { g_global_error = msg; }
// an output argument of the ABI: NULL is a caller error, reported as CCSD_ERR_ARG
template <class T>
T& need(T* p) {
    if (!p) throw Error(CCSD_ERR_ARG, "null output argument");
    return *p;
}
}  // namespace ccsd

using namespace ccsd;

namespace {

template <class F>
int guarded(ccsd_ctx ctx, F f) {
    try {
        if (ctx && ctx->c && ctx->c->device >= 0) CCSD_CUDA(cudaSetDevice(ctx->c->device));
        f();
        return CCSD_OK;
    } catch (const Error& e) {
        if (ctx && ctx->c) ctx->c->last_error = e.what();
        else g_global_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        if (ctx && ctx->c) ctx->c->last_error = e.what();
        else g_global_error = e.what();
        return CCSD_ERR_ARG;
    }
}

const Block& block_at(Tensor& T, const int alpha[4], const int* irreps, int& cs) {
    cs = T.find_case(alpha);
    if (cs < 0) throw Error(CCSD_ERR_ARG, "no such spin case in " + T.name);
    std::vector<int> irr(T.ndim, 0);
    if (irreps)
        for (int p = 0; p < T.ndim; p++) irr[p] = irreps[p];
    auto it = T.cases[cs].block_of.find(irr);
    if (it == T.cases[cs].block_of.end()) throw Error(CCSD_ERR_ARG, "block not stored in " + T.name);
    return T.cases[cs].blocks[it->second];
}

// Expand a key (first index fastest, full block index) into the storage offsets of all
// its images under permutations inside same-spin groups, with signs; for packed pairs
// only the canonical image is stored.
void key_images(const Tensor& T, int cs, const Block& b, int64_t key, std::vector<std::pair<int64_t, double>>& out) {
    out.clear();
    const int nd = T.ndim;
    std::vector<int64_t> x(nd);
    int64_t r = key;
    for (int p = 0; p < nd; p++) {
        if (b.len[p] == 0) return;
        x[p] = r % b.len[p];
        r /= b.len[p];
    }
    if (r != 0) throw Error(CCSD_ERR_ARG, "key out of range");
    const SpinCase& sc = T.cases[cs];
    // same-spin pairs inside a group with equal irreps can be swapped (AS symmetry);
    // plain tensors have no antisymmetric images
    std::vector<std::pair<int, int>> swaps;
    for (int p = 0; p + 1 < nd && !T.plain(); p++)
        if (T.group[p] == T.group[p + 1] && sc.spin[p] == sc.spin[p + 1] && b.irrep[p] == b.irrep[p + 1])
            swaps.push_back({p, p + 1});
    const int ns = (int)swaps.size();
    for (int mask = 0; mask < (1 << ns); mask++) {
        std::vector<int64_t> y = x;
        double sign = 1;
        for (int i = 0; i < ns; i++)
            if (mask & (1 << i)) {
                std::swap(y[swaps[i].first], y[swaps[i].second]);
                sign = -sign;
            }
        bool skip = false;
        int64_t off = b.offset;
        for (int p = 0; p < nd; p++) {
            int pi = b.pair_of(p);
            if (pi >= 0) {
                const auto& pr = b.pairs[pi];
                if (pr.p != p) continue;
                int64_t u = y[pr.p], v = y[pr.q];
                if (pr.kind == 1) {
                    if (u >= v) {
                        skip = true;
                        break;
                    }
                    off += pr.stride * (v * (v - 1) / 2 + u);
                } else {
                    off += pr.stride * (u + (int64_t)b.len[pr.p] * v);
                }
            } else {
                off += b.stride[p] * y[p];
            }
        }
        bool diag = false;
        for (auto& s : swaps) diag |= x[s.first] == x[s.second];
        if (diag) {
            // antisymmetric diagonal elements are zero: store nothing but a zero
            if (mask == 0 && !skip) out.push_back({off, 0.0});
            continue;
        }
        if (!skip) out.push_back({off, sign});
    }
}

}  // namespace

extern "C" {

int ccsd_ctx_create(int device, void* stream, ccsd_ctx* out) {
    if (!out) return CCSD_ERR_ARG;
    *out = nullptr;
    return guarded(nullptr, [&] {
        if (device >= 0) CCSD_CUDA(cudaSetDevice(device));   // < 0: planning only
        auto* h = new ccsd_ctx_s;
        try {
            h->c = new Context(device, (cudaStream_t)stream);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int ccsd_ctx_destroy(ccsd_ctx ctx) {
    if (!ctx) return CCSD_ERR_ARG;
    int st = guarded(ctx, [&] { delete ctx->c; });
    ctx->c = nullptr;
    delete ctx;
    return st;
}

const char* ccsd_last_error(ccsd_ctx ctx) {
    if (ctx && ctx->c) return ctx->c->last_error.c_str();
    return g_global_error.c_str();
}

int ccsd_ctx_plan_flops(ccsd_ctx ctx, double* flops) {
    return guarded(ctx, [&] {
        if (!flops) throw Error(CCSD_ERR_ARG, "null output");
        *flops = from_handle(ctx)->last_plan_flops;
    });
}

int ccsd_ctx_plan_export(ccsd_ctx ctx, const char* path) {
    return guarded(ctx, [&] {
        if (!path) throw Error(CCSD_ERR_ARG, "null path");
        Context* c = from_handle(ctx);
        auto it = c->plan_cache.find(c->last_plan_key);
        if (c->last_plan_key.empty() || it == c->plan_cache.end())
            throw Error(CCSD_ERR_ARG, "no statement planned on this context");
        export_plan(*c, *it->second, path);
    });
}

int ccsd_ctx_synchronize(ccsd_ctx ctx) {
    return guarded(ctx, [&] { CCSD_CUDA(cudaStreamSynchronize(from_handle(ctx)->stream)); });
}

int ccsd_ctx_device_bytes(ccsd_ctx ctx, int64_t* bytes) {
    return guarded(ctx, [&] { need(bytes) = from_handle(ctx)->device_bytes; });
}

int ccsd_ctx_launch_count(ccsd_ctx ctx, int64_t* count) {
    return guarded(ctx, [&] {
        from_handle(ctx);
        need(count) = kern::launch_count();
    });
}

int ccsd_ctx_set_precision(ccsd_ctx ctx, int precision, int slices) {
    return guarded(ctx, [&] {
        Context* c = from_handle(ctx);
        if (precision != CCSD_PREC_FP64 && precision != CCSD_PREC_SPLIT && precision != CCSD_PREC_SPLIT_I8)
            throw Error(CCSD_ERR_ARG, "bad precision");
        if (precision != CCSD_PREC_FP64 && !kern::split_supported())
            throw Error(CCSD_ERR_UNSUPPORTED, "split GEMMs need an sm_100 device");
        const int kind = precision == CCSD_PREC_SPLIT_I8 ? kern::SLICE_INT8 : kern::SLICE_BF16;
        if (slices != 0 && !kern::slice_scheme_ok(kind, slices))
            throw Error(CCSD_ERR_ARG, "slices must be 0 (default) or 3, 4 (BF16) / 3, 4, 5 (INT8)");
        c->precision = precision;
        c->slices = slices;
    });
}

int ccsd_ctx_set_split_routing(ccsd_ctx ctx, int mode) {
    return guarded(ctx, [&] {
        if (mode != CCSD_SPLIT_ROUTE_AUTO && mode != CCSD_SPLIT_ROUTE_ALL) throw Error(CCSD_ERR_ARG, "bad routing mode");
        from_handle(ctx)->split_routing = mode;
    });
}

int ccsd_ctx_split_launches(ccsd_ctx ctx, int64_t* launches) {
    return guarded(ctx, [&] {
        if (!launches) throw Error(CCSD_ERR_ARG, "null output");
        *launches = from_handle(ctx)->split_launches;
    });
}

int ccsd_ctx_set_profiling(ccsd_ctx ctx, int on) {
    return guarded(ctx, [&] {
        Context* c = from_handle(ctx);
        c->collect_profile();
        c->profiling = on != 0;
    });
}

int ccsd_ctx_profile_report(ccsd_ctx ctx, char* buf, int64_t buflen, int64_t* needed) {
    return guarded(ctx, [&] {
        Context* c = from_handle(ctx);
        c->collect_profile();
        std::ostringstream o;
        o.precision(10);
        o << "{";
        bool first = true;
        for (auto& kv : c->profile) {
            if (!first) o << ",";
            first = false;
            o << "\"";
            for (char ch : kv.first) {
                if (ch == '"' || ch == '\\') o << '\\';
                o << ch;
            }
            o << "\":{\"launches\":" << kv.second.launches << ",\"ms\":" << kv.second.ms
              << ",\"flops\":" << kv.second.flops << "}";
        }
        o << "}";
        std::string s = o.str();
        if (needed) *needed = (int64_t)s.size() + 1;
        if (buf && buflen > (int64_t)s.size()) {
            std::memcpy(buf, s.c_str(), s.size() + 1);
            c->profile.clear();
        } else if (buf) {
            throw Error(CCSD_ERR_ARG, "profile buffer too small");
        }
    });
}

int ccsd_ctx_set_spaces(ccsd_ctx ctx, int nirrep, const int* vrt_alpha, const int* vrt_beta, const int* occ_alpha,
                        const int* occ_beta) {
    return guarded(ctx, [&] {
        Context* c = from_handle(ctx);
        if (nirrep != 1 && nirrep != 2 && nirrep != 4 && nirrep != 8) throw Error(CCSD_ERR_ARG, "nirrep must be 1,2,4,8");
        if (!c->tensors.empty()) throw Error(CCSD_ERR_ARG, "spaces cannot change while tensors exist");
        if (!vrt_alpha || !occ_alpha) throw Error(CCSD_ERR_ARG, "null alpha orbital counts");
        Spaces S;
        S.nirrep = nirrep;
        // NULL beta counts: closed shell, the same orbitals for both spins
        const int* src[2][2] = {{vrt_alpha, vrt_beta ? vrt_beta : vrt_alpha}, {occ_alpha, occ_beta ? occ_beta : occ_alpha}};
        for (int sp = 0; sp < 2; sp++)
            for (int s = 0; s < 2; s++) {
                int off = 0;
                for (int h = 0; h < nirrep; h++) {
                    int v = src[sp][s][h];
                    if (v < 0) throw Error(CCSD_ERR_ARG, "negative orbital count");
                    S.n[sp][s][h] = v;
                    S.off[sp][s][h] = off;
                    off += v;
                }
            }
        c->spaces = S;
        c->spaces_set = true;
    });
}

int ccsd_tensor_create(ccsd_ctx ctx, const char* name, const int nout[2], const int nin[2], int flags,
                       ccsd_tensor* out) {
    return guarded(ctx, [&] {
        if (!nout || !nin || !out) throw Error(CCSD_ERR_ARG, "null argument");
        *out = from_handle(ctx)->create_tensor(name ? name : "", nout, nin, flags);
    });
}

int ccsd_tensor_destroy(ccsd_ctx ctx, ccsd_tensor t) {
    return guarded(ctx, [&] { from_handle(ctx)->destroy_tensor(t); });
}

int ccsd_tensor_ndim(ccsd_ctx ctx, ccsd_tensor t, int* ndim) {
    return guarded(ctx, [&] { need(ndim) = from_handle(ctx)->tensor(t).ndim; });
}

int ccsd_tensor_spin_cases(ccsd_ctx ctx, ccsd_tensor t, int* ncases, int* alpha) {
    return guarded(ctx, [&] {
        Tensor& T = from_handle(ctx)->tensor(t);
        need(ncases) = (int)T.cases.size();
        if (alpha)
            for (size_t c = 0; c < T.cases.size(); c++)
                for (int g = 0; g < 4; g++) alpha[4 * c + g] = T.cases[c].alpha[g];
    });
}

int ccsd_tensor_block_size(ccsd_ctx ctx, ccsd_tensor t, const int alpha[4], const int* irreps, int64_t* n) {
    return guarded(ctx, [&] {
        Tensor& T = from_handle(ctx)->tensor(t);
        if (!alpha) throw Error(CCSD_ERR_ARG, "null spin case");
        int cs = T.find_case(alpha);
        need(n) = 0;
        if (cs < 0) return;
        std::vector<int> irr(T.ndim, 0);
        if (irreps)
            for (int p = 0; p < T.ndim; p++) irr[p] = irreps[p];
        auto it = T.cases[cs].block_of.find(irr);
        if (it != T.cases[cs].block_of.end()) *n = T.cases[cs].blocks[it->second].size;
    });
}

// storage offset (relative to the block) of every element of a block in first-index-fastest
// order; the identity for ordinary blocks, a permutation for views
static std::vector<int64_t> block_order(const Block& b) {
    std::vector<int64_t> off(b.size);
    const int nd = (int)b.len.size();
    for (int64_t l = 0; l < b.size; l++) {
        int64_t r = l, o = 0;
        for (int p = 0; p < nd; p++) {
            int64_t x = r % b.len[p];
            r /= b.len[p];
            o += x * b.stride[p];
        }
        off[l] = o;
    }
    return off;
}

int ccsd_tensor_write_block(ccsd_ctx ctx, ccsd_tensor t, const int alpha[4], const int* irreps, const double* host) {
    return guarded(ctx, [&] {
        Context* c = device_handle(ctx);
        Tensor& T = c->tensor(t);
        int cs;
        const Block& b = block_at(T, alpha, irreps, cs);
        if (T.view_of) {
            std::vector<int64_t> ord = block_order(b);
            std::vector<double> buf(b.size);
            for (int64_t l = 0; l < b.size; l++) buf[ord[l]] = host[l];
            CCSD_CUDA(cudaMemcpy(T.data + b.offset, buf.data(), b.size * sizeof(double), cudaMemcpyHostToDevice));
            return;
        }
        CCSD_CUDA(cudaMemcpyAsync(T.data + b.offset, host, b.size * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        CCSD_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int ccsd_tensor_read_block(ccsd_ctx ctx, ccsd_tensor t, const int alpha[4], const int* irreps, double* host) {
    return guarded(ctx, [&] {
        Context* c = device_handle(ctx);
        Tensor& T = c->tensor(t);
        int cs;
        const Block& b = block_at(T, alpha, irreps, cs);
        CCSD_CUDA(cudaStreamSynchronize(c->stream));
        if (T.view_of) {
            std::vector<int64_t> ord = block_order(b);
            std::vector<double> buf(b.size);
            CCSD_CUDA(cudaMemcpy(buf.data(), T.data + b.offset, b.size * sizeof(double), cudaMemcpyDeviceToHost));
            for (int64_t l = 0; l < b.size; l++) host[l] = buf[ord[l]];
            return;
        }
        CCSD_CUDA(cudaMemcpyAsync(host, T.data + b.offset, b.size * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CCSD_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int ccsd_tensor_write(ccsd_ctx ctx, ccsd_tensor t, const int alpha_spin[4], const int* irreps, int64_t n,
                      const int64_t* keys, const double* vals, double alpha, double beta) {
    return guarded(ctx, [&] {
        Context* c = device_handle(ctx);
        Tensor& T = c->tensor(t);
        int cs;
        const Block& b = block_at(T, alpha_spin, irreps, cs);
        std::vector<int64_t> offs;
        std::vector<double> v;
        std::vector<std::pair<int64_t, double>> img;
        for (int64_t i = 0; i < n; i++) {
            key_images(T, cs, b, keys[i], img);
            for (auto& im : img) {
                offs.push_back(im.first);
                v.push_back(im.second * vals[i]);
            }
        }
        if (offs.empty()) return;
        int64_t* dk = (int64_t*)c->dmalloc(offs.size() * sizeof(int64_t));
        double* dv = (double*)c->dmalloc(v.size() * sizeof(double));
        CCSD_CUDA(cudaMemcpyAsync(dk, offs.data(), offs.size() * sizeof(int64_t), cudaMemcpyHostToDevice, c->stream));
        CCSD_CUDA(cudaMemcpyAsync(dv, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        kern::kv_write(T.data, dk, dv, (int64_t)offs.size(), alpha, beta, c->stream);
        CCSD_CUDA(cudaStreamSynchronize(c->stream));
        c->dfree(dk, offs.size() * sizeof(int64_t));
        c->dfree(dv, v.size() * sizeof(double));
    });
}

int ccsd_tensor_read(ccsd_ctx ctx, ccsd_tensor t, const int alpha_spin[4], const int* irreps, int64_t n,
                     const int64_t* keys, double* vals) {
    return guarded(ctx, [&] {
        Context* c = device_handle(ctx);
        Tensor& T = c->tensor(t);
        int cs;
        const Block& b = block_at(T, alpha_spin, irreps, cs);
        std::vector<int64_t> offs(n);
        std::vector<double> sign(n, 1.0);
        std::vector<std::pair<int64_t, double>> img;
        for (int64_t i = 0; i < n; i++) {
            key_images(T, cs, b, keys[i], img);
            if (img.empty()) throw Error(CCSD_ERR_ARG, "key maps to no stored element");
            offs[i] = img[0].first;
            sign[i] = img[0].second;
        }
        if (n == 0) return;
        int64_t* dk = (int64_t*)c->dmalloc(n * sizeof(int64_t));
        double* dv = (double*)c->dmalloc(n * sizeof(double));
        CCSD_CUDA(cudaMemcpyAsync(dk, offs.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice, c->stream));
        kern::kv_read(T.data, dk, dv, n, c->stream);
        CCSD_CUDA(cudaMemcpyAsync(vals, dv, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CCSD_CUDA(cudaStreamSynchronize(c->stream));
        for (int64_t i = 0; i < n; i++) vals[i] *= sign[i] == 0.0 ? 0.0 : sign[i];
        c->dfree(dk, n * sizeof(int64_t));
        c->dfree(dv, n * sizeof(double));
    });
}

int ccsd_tensor_fill(ccsd_ctx ctx, ccsd_tensor t, double val) {
    return guarded(ctx, [&] {
        Context* c = device_handle(ctx);
        Tensor& T = c->tensor(t);
        kern::fill(T.data, T.total, val, c->stream);
    });
}

static std::string plan_key(const char* kind, double alpha, int A, const char* iA, int B, const char* iB, double beta,
                            int C, const char* iC, int prec) {
    std::ostringstream o;
    o.precision(17);
    o << kind << '|' << alpha << '|' << A << ':' << iA << '|' << B << ':' << (iB ? iB : "") << '|' << beta << '|' << C
      << ':' << (iC ? iC : "") << '|' << prec;
    return o.str();
}

int ccsd_contract(ccsd_ctx ctx, double alpha, ccsd_tensor A, const char* idxA, ccsd_tensor B, const char* idxB,
                  double beta, ccsd_tensor C, const char* idxC) {
    return guarded(ctx, [&] {
        Context* c = from_handle(ctx);
        if (!idxA || !idxB || !idxC) throw Error(CCSD_ERR_ARG, "null index string");
        std::string key = plan_key("mult", alpha, A, idxA, B, idxB, beta, C, idxC, 0);
        auto it = c->plan_cache.find(key);
        if (it == c->plan_cache.end()) {
            auto p = std::make_unique<Plan>(plan_contract(*c, alpha, A, idxA, B, idxB, beta, C, idxC));
            it = c->plan_cache.emplace(key, std::move(p)).first;
        }
        c->last_plan_flops = it->second->flops();
        c->last_plan_key = key;
        c->run(*it->second);
    });
}

int ccsd_sum(ccsd_ctx ctx, double alpha, ccsd_tensor A, const char* idxA, double beta, ccsd_tensor B,
             const char* idxB) {
    return guarded(ctx, [&] {
        Context* c = from_handle(ctx);
        if (!idxA || !idxB) throw Error(CCSD_ERR_ARG, "null index string");
        std::string key = plan_key("sum", alpha, A, idxA, 0, nullptr, beta, B, idxB, 0);
        auto it = c->plan_cache.find(key);
        if (it == c->plan_cache.end()) {
            auto p = std::make_unique<Plan>(plan_sum(*c, alpha, A, idxA, beta, B, idxB));
            it = c->plan_cache.emplace(key, std::move(p)).first;
        }
        c->last_plan_key = key;
        c->run(*it->second);
    });
}

int ccsd_scale(ccsd_ctx ctx, ccsd_tensor A, double alpha) {
    return guarded(ctx, [&] {
        Context* c = device_handle(ctx);
        Tensor& T = c->tensor(A);
        kern::scale(T.data, T.total, alpha, c->stream);
    });
}

int ccsd_dot(ccsd_ctx ctx, ccsd_tensor A, const char* idxA, ccsd_tensor B, const char* idxB, double* out) {
    return guarded(ctx, [&] {
        Context* c = device_handle(ctx);
        if (!idxA || !idxB || !out) throw Error(CCSD_ERR_ARG, "null argument");
        std::string key = plan_key("dot", 1.0, A, idxA, B, idxB, 0.0, 0, nullptr, 0);
        auto it = c->plan_cache.find(key);
        if (it == c->plan_cache.end()) {
            auto p = std::make_unique<Plan>(plan_dot(*c, A, idxA, B, idxB));
            it = c->plan_cache.emplace(key, std::move(p)).first;
        }
        c->run(*it->second, out);
    });
}

// SpinorbitalTensor::norm (spinorbital_tensor.cxx:1077-1109): p=0 max over spin cases;
// p=1,2 weight each case by the number of spin-orbital arrangements it stands for.
// Inside a case each antisymmetric same-spin element counts once (packed semantics).
int ccsd_norm(ccsd_ctx ctx, ccsd_tensor A, int p, double* out) {
    return guarded(ctx, [&] {
        Context* c = device_handle(ctx);
        need(out);
        if (p != 0 && p != 1 && p != 2) throw Error(CCSD_ERR_ARG, "p must be 0, 1 or 2");
        Tensor& T = c->tensor(A);
        CCSD_CUDA(cudaMemsetAsync(c->d_scalar, 0, sizeof(double), c->stream));
        const int gs[4] = {T.nout[0], T.nout[1], T.nin[0], T.nin[1]};
        for (auto& sc : T.cases) {
            double factor = 1, perms = 1;
            for (int g = 0; g < 4; g++) {
                double b = 1;
                for (int k = 0; k < sc.alpha[g]; k++) b = b * (gs[g] - k) / (k + 1);
                factor *= b;
                // unpacked storage holds every order of a same-spin run: a! * (n-a)!
                int na = sc.alpha[g], nb = gs[g] - sc.alpha[g];
                double f = 1;
                for (int k = 2; k <= na; k++) f *= k;
                for (int k = 2; k <= nb; k++) f *= k;
                if (!T.packed()) perms *= f;
            }
            for (auto& b : sc.blocks) {
                if (b.size == 0) continue;
                kern::norm_accum(T.data + b.offset, b.size, p, factor / perms, c->d_scalar, c->stream);
            }
        }
        double h = 0;
        CCSD_CUDA(cudaMemcpyAsync(&h, c->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CCSD_CUDA(cudaStreamSynchronize(c->stream));
        need(out) = p == 2 ? std::sqrt(h) : h;
    });
}

int ccsd_weight(ccsd_ctx ctx, ccsd_tensor A, const double* dvrt_a, const double* dvrt_b, const double* docc_a,
                const double* docc_b, double shift) {
    return guarded(ctx, [&] {
        Context* c = device_handle(ctx);
        Tensor& T = c->tensor(A);
        const Spaces& S = c->spaces;
        const double* src[2][2] = {{dvrt_a, dvrt_b}, {docc_a, docc_b}};
        double* dev[2][2];
        for (int sp = 0; sp < 2; sp++)
            for (int s = 0; s < 2; s++) {
                int n = std::max(1, S.total(sp, s));
                dev[sp][s] = (double*)c->dmalloc(n * sizeof(double));
                if (S.total(sp, s) > 0)
                    CCSD_CUDA(cudaMemcpyAsync(dev[sp][s], src[sp][s], S.total(sp, s) * sizeof(double),
                                              cudaMemcpyHostToDevice, c->stream));
            }
        for (auto& sc : T.cases)
            for (auto& b : sc.blocks) {
                if (b.size == 0) continue;
                if (!b.pairs.empty()) throw Error(CCSD_ERR_UNSUPPORTED, "weight of a packed tensor");
                if (T.view_of) throw Error(CCSD_ERR_UNSUPPORTED, "weight of a view tensor");
                kern::WeightArgs w;
                w.ndim = T.ndim;
                w.total = b.size;
                for (int p = 0; p < T.ndim; p++) {
                    int sp = group_space(T.group[p]);
                    w.len[p] = b.len[p];
                    w.d[p] = dev[sp][sc.spin[p]] + S.off[sp][sc.spin[p]][b.irrep[p]];
                }
                kern::weight_block(T.data + b.offset, w, shift, c->stream);
            }
        CCSD_CUDA(cudaStreamSynchronize(c->stream));
        for (int sp = 0; sp < 2; sp++)
            for (int s = 0; s < 2; s++) c->dfree(dev[sp][s], std::max(1, S.total(sp, s)) * sizeof(double));
    });
}

void ccsd_options_default(ccsd_options* opts) {
    if (opts) options_default(opts);
}

int ccsd_hamiltonian_from_factor(ccsd_ctx ctx, int naux, const double* B, const double* eps,
                                 const int* aux_per_irrep, int pack_vvvv, ccsd_hamiltonian* H) {
    return guarded(ctx, [&] {
        if (!B || !eps || !H || naux <= 0) throw Error(CCSD_ERR_ARG, "bad factor arguments");
        build_hamiltonian(*device_handle(ctx), naux, B, eps, aux_per_irrep, pack_vvvv != 0, H);
    });
}

int ccsd_hamiltonian_create(ccsd_ctx ctx, int pack_vvvv, ccsd_hamiltonian* H) {
    return guarded(ctx, [&] {
        if (!H) throw Error(CCSD_ERR_ARG, "null hamiltonian");
        Context* c = from_handle(ctx);
        if (!c->spaces_set) throw Error(CCSD_ERR_ARG, "set the orbital spaces first");
        create_hamiltonian_tensors(*c, pack_vvvv != 0, H);
    });
}

int ccsd_hamiltonian_from_integrals(ccsd_ctx ctx, int n, const double* fock, const double* eri, int pack_vvvv,
                                    ccsd_hamiltonian* H) {
    return guarded(ctx, [&] {
        if (!fock || !eri || !H || n <= 0) throw Error(CCSD_ERR_ARG, "bad integral arguments");
        Context* c = device_handle(ctx);
        if (!c->spaces_set) throw Error(CCSD_ERR_ARG, "set the orbital spaces first");
        build_hamiltonian_dense(*c, n, fock, eri, pack_vvvv != 0, H);
    });
}

int ccsd_fcidump_read(const char* path, int flags, int* norb, int* nelec, double* ecore, double* h, double* eri) {
    return guarded(nullptr, [&] {
        if (!path) throw Error(CCSD_ERR_ARG, "null path");
        Fcidump d = read_fcidump(path, (flags & CCSD_FCIDUMP_FULL_FOCK) != 0, !h && !eri);
        if (norb) *norb = d.norb;
        if (nelec) *nelec = d.nelec;
        if (ecore) *ecore = d.ecore;
        if (h && !d.h.empty()) std::memcpy(h, d.h.data(), d.h.size() * sizeof(double));
        if (eri && !d.eri.empty()) std::memcpy(eri, d.eri.data(), d.eri.size() * sizeof(double));
    });
}

int ccsd_hamiltonian_from_fcidump(ccsd_ctx ctx, const char* path, int flags, int pack_vvvv, ccsd_hamiltonian* H,
                                  double* escf) {
    return guarded(ctx, [&] {
        if (!path || !H) throw Error(CCSD_ERR_ARG, "bad FCIDUMP arguments");
        Context* c = device_handle(ctx);
        Fcidump d = read_fcidump(path, (flags & CCSD_FCIDUMP_FULL_FOCK) != 0, false);
        const int n = d.norb, no = d.nelec / 2, nv = n - no;
        if (!c->tensors.empty()) {
            const Spaces& S = c->spaces;
            bool same = c->spaces_set && S.nirrep == 1;
            for (int s = 0; s < 2 && same; s++) same = S.n[VRT][s][0] == nv && S.n[OCC][s][0] == no;
            if (!same) throw Error(CCSD_ERR_ARG, "context has tensors over other spaces than the FCIDUMP's");
        } else {
            int v[1] = {nv}, o[1] = {no};
            const int st = ccsd_ctx_set_spaces(ctx, 1, v, v, o, o);
            if (st != CCSD_OK) throw Error(st, "setting the FCIDUMP spaces failed");
        }
        std::vector<double> f((size_t)n * n);
        const double e = closed_shell_fock(n, no, d.h.data(), d.eri.data(), f.data());
        if (flags & CCSD_FCIDUMP_SEMICANONICAL) semicanonicalize(n, no, f.data(), d.eri.data());
        build_hamiltonian_dense(*c, n, f.data(), d.eri.data(), pack_vvvv != 0, H);
        if (escf) *escf = d.ecore + e;
    });
}

namespace {
// C1 closed-shell spaces for nocc of nmo orbitals on a context without tensors (or check them)
void set_closed_shell_spaces(ccsd_ctx ctx, Context* c, int nmo, int nocc) {
    const int nv = nmo - nocc;
    if (!c->tensors.empty() || c->spaces_set) {
        const Spaces& S = c->spaces;
        bool same = c->spaces_set && S.nirrep == 1;
        for (int s = 0; s < 2 && same; s++) same = S.n[VRT][s][0] == nv && S.n[OCC][s][0] == nocc;
        if (!same) throw Error(CCSD_ERR_ARG, "context spaces differ from the AO problem's (C1, nocc, nmo - nocc)");
        return;
    }
    int v[1] = {nv}, o[1] = {nocc};
    const int st = ccsd_ctx_set_spaces(ctx, 1, v, v, o, o);
    if (st != CCSD_OK) throw Error(st, "setting the AO problem's spaces failed");
}

// device MO integrals of an AO problem, freed with the object
struct MoIntegrals {
    Context& c;
    double* d = nullptr;
    int64_t bytes = 0;
    std::vector<double> fock;
    double e = 0;
    MoIntegrals(Context& ctx, int nao, int nmo, int nocc, const double* hcore, const double* eri, const double* C)
        : c(ctx) {
        bytes = (int64_t)nmo * nmo * nmo * nmo * (int64_t)sizeof(double);
        d = (double*)c.dmalloc(bytes);
        fock.resize((size_t)nmo * nmo);
        e = ao_to_mo(c, nao, nmo, nocc, hcore, eri, C, d, fock.data());
    }
    ~MoIntegrals() {
        cudaStreamSynchronize(c.stream);
        c.dfree(d, bytes);
    }
};
}  // namespace

int ccsd_hamiltonian_from_ao(ccsd_ctx ctx, int nao, int nmo, int nocc, const double* hcore, const double* eri_ao,
                             const double* C, int pack_vvvv, ccsd_hamiltonian* H, double* e_elec) {
    return guarded(ctx, [&] {
        if (!hcore || !eri_ao || !C || !H) throw Error(CCSD_ERR_ARG, "bad AO arguments");
        Context* c = device_handle(ctx);
        set_closed_shell_spaces(ctx, c, nmo, nocc);
        MoIntegrals mo(*c, nao, nmo, nocc, hcore, eri_ao, C);
        build_hamiltonian_device(*c, nmo, mo.fock.data(), mo.d, pack_vvvv != 0, H);
        if (e_elec) *e_elec = mo.e;
    });
}

int ccsd_rhf_hamiltonian_from_ao(ccsd_ctx ctx, int nao, int nmo, int nocc, const double* hcore,
                                 const double* eri_ao, const double* C, ccsd_rhf_hamiltonian* H, double* e_elec) {
    return guarded(ctx, [&] {
        if (!hcore || !eri_ao || !C || !H) throw Error(CCSD_ERR_ARG, "bad AO arguments");
        Context* c = device_handle(ctx);
        set_closed_shell_spaces(ctx, c, nmo, nocc);
        MoIntegrals mo(*c, nao, nmo, nocc, hcore, eri_ao, C);
        build_rhf_hamiltonian_device(*c, nmo, mo.fock.data(), mo.d, H);
        if (e_elec) *e_elec = mo.e;
    });
}

int ccsd_hamiltonian_destroy(ccsd_ctx ctx, ccsd_hamiltonian* H) {
    return guarded(ctx, [&] {
        Context* c = from_handle(ctx);
        // views first, then the tensors they alias
        for (ccsd_tensor* t : {&H->VMNEJ, &H->VABIJ, &H->VABEJ, &H->fAI, &H->fME, &H->fAE, &H->fMI, &H->VMNIJ,
                               &H->VAMIJ, &H->VMNEF, &H->VAMEI, &H->VAMEF, &H->VABEF}) {
            if (*t && c->tensors.count(*t)) c->destroy_tensor(*t);
            *t = 0;
        }
    });
}

int ccsd_rhf_hamiltonian_from_factor(ccsd_ctx ctx, int naux, const double* B, const double* eps,
                                     const int* aux_per_irrep, ccsd_rhf_hamiltonian* H) {
    return guarded(ctx, [&] {
        if (!B || !eps || !H || naux <= 0) throw Error(CCSD_ERR_ARG, "bad factor arguments");
        Context* c = device_handle(ctx);
        if (!c->spaces_set) throw Error(CCSD_ERR_ARG, "set the orbital spaces first");
        build_rhf_hamiltonian(*c, naux, B, eps, aux_per_irrep, H);
    });
}

int ccsd_rhf_hamiltonian_from_integrals(ccsd_ctx ctx, int n, const double* fock, const double* eri,
                                        ccsd_rhf_hamiltonian* H) {
    return guarded(ctx, [&] {
        if (!fock || !eri || !H || n <= 0) throw Error(CCSD_ERR_ARG, "bad integral arguments");
        Context* c = device_handle(ctx);
        if (!c->spaces_set) throw Error(CCSD_ERR_ARG, "set the orbital spaces first");
        build_rhf_hamiltonian_dense(*c, n, fock, eri, H);
    });
}

int ccsd_rhf_hamiltonian_destroy(ccsd_ctx ctx, ccsd_rhf_hamiltonian* H) {
    return guarded(ctx, [&] {
        if (!H) throw Error(CCSD_ERR_ARG, "null hamiltonian");
        Context* c = from_handle(ctx);
        for (ccsd_tensor* t : {&H->fAI, &H->fAB, &H->fIJ, &H->VABCD, &H->VABCI, &H->VABIJ, &H->VAIBJ, &H->VAIJB,
                               &H->VAIJK, &H->VIJKL}) {
            if (*t && c->tensors.count(*t)) c->destroy_tensor(*t);
            *t = 0;
        }
    });
}

int ccsd_rhf_solver_create(ccsd_ctx ctx, const ccsd_rhf_hamiltonian* H, const ccsd_options* opts, ccsd_solver* out) {
    if (!out) return CCSD_ERR_ARG;
    *out = nullptr;
    return guarded(ctx, [&] {
        if (!H) throw Error(CCSD_ERR_ARG, "null hamiltonian");
        Context* c = device_handle(ctx);
        ccsd_options o;
        options_default(&o);
        if (opts) o = *opts;
        if (o.precision != CCSD_PREC_FP64 && !kern::split_supported())
            throw Error(CCSD_ERR_UNSUPPORTED, "split GEMMs need an sm_100 device");
        auto* h = new ccsd_solver_s;
        h->ctx = ctx;
        try {
            h->s = new Solver(*c, *H, o);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

namespace {
// orbital counts per irrep; the beta counts default to the alpha ones (closed shell)
Spaces query_spaces(int nirrep, const int* vrt, const int* occ, int& n, const int* vrt_b = nullptr,
                    const int* occ_b = nullptr) {
    if (nirrep != 1 && nirrep != 2 && nirrep != 4 && nirrep != 8) throw Error(CCSD_ERR_ARG, "nirrep must be 1,2,4,8");
    if (!vrt || !occ) throw Error(CCSD_ERR_ARG, "null orbital counts");
    Spaces S;
    S.nirrep = nirrep;
    n = 0;
    for (int s = 0; s < 2; s++) {
        const int* v = (s == 1 && vrt_b) ? vrt_b : vrt;
        const int* o = (s == 1 && occ_b) ? occ_b : occ;
        int ov = 0, oo = 0;
        for (int h = 0; h < nirrep; h++) {
            S.n[VRT][s][h] = v[h];
            S.n[OCC][s][h] = o[h];
            S.off[VRT][s][h] = ov;
            S.off[OCC][s][h] = oo;
            ov += v[h];
            oo += o[h];
        }
        n = ov + oo;
    }
    return S;
}
}  // namespace

int ccsd_rhf_plan_query(int nirrep, const int* vrt, const int* occ, const ccsd_options* opts,
                        double* flops_per_iter, int64_t* device_bytes) {
    return guarded(nullptr, [&] {
        Context host(-1, nullptr);
        int n = 0;
        host.spaces = query_spaces(nirrep, vrt, occ, n);
        host.spaces_set = true;
        ccsd_rhf_hamiltonian H;
        create_rhf_hamiltonian_tensors(host, &H);
        const int64_t build_peak = host.device_bytes + (int64_t)3 * n * n * n * 8;
        ccsd_options o;
        options_default(&o);
        if (opts) o = *opts;
        Solver s(host, H, o);
        if (flops_per_iter) *flops_per_iter = s.flops_per_iter;
        if (device_bytes) *device_bytes = std::max(host.peak_bytes, build_peak);
    });
}

int ccsd_plan_query(int nirrep, const int* vrt, const int* occ, const ccsd_options* opts, int pack_vvvv,
                    double* flops_per_iter, int64_t* device_bytes) {
    return guarded(nullptr, [&] {
        if (nirrep != 1 && nirrep != 2 && nirrep != 4 && nirrep != 8) throw Error(CCSD_ERR_ARG, "nirrep must be 1,2,4,8");
        Context host(-1, nullptr);
        Spaces S;
        S.nirrep = nirrep;
        int n = 0;
        for (int s = 0; s < 2; s++) {
            int ov = 0, oo = 0;
            for (int h = 0; h < nirrep; h++) {
                S.n[VRT][s][h] = vrt[h];
                S.n[OCC][s][h] = occ[h];
                S.off[VRT][s][h] = ov;
                S.off[OCC][s][h] = oo;
                ov += vrt[h];
                oo += occ[h];
            }
            n = ov + oo;
        }
        host.spaces = S;
        host.spaces_set = true;
        ccsd_hamiltonian H;
        create_hamiltonian_tensors(host, pack_vvvv != 0, &H);
        const int64_t h_bytes = host.device_bytes;
        // factor build: B (3n x n x n) plus two 256 MiB chunk buffers for packed blocks
        const int64_t build_peak = h_bytes + (int64_t)3 * n * n * n * 8 + (int64_t)2 * (256ll << 20) * 8 / 8;
        ccsd_options o;
        options_default(&o);
        if (opts) o = *opts;
        Solver s(host, H, o);
        if (flops_per_iter) *flops_per_iter = s.flops_per_iter;
        if (device_bytes) *device_bytes = std::max(host.peak_bytes, build_peak);
    });
}

int ccsd_lambda_plan_query(int nirrep, const int* vrt, const int* occ, const ccsd_options* opts,
                           double* hbar_flops, double* flops_per_iter, int64_t* device_bytes) {
    return guarded(nullptr, [&] {
        Context host(-1, nullptr);
        int n = 0;
        host.spaces = query_spaces(nirrep, vrt, occ, n);
        host.spaces_set = true;
        ccsd_hamiltonian H;
        create_hamiltonian_tensors(host, false, &H);
        ccsd_options o;
        options_default(&o);
        if (opts) o = *opts;
        Solver cc(host, H, o);
        cc.hbar_so();
        Solver lam(host, cc, cc.HB, o);
        if (hbar_flops) *hbar_flops = cc.hbar_plan.flops();
        if (flops_per_iter) *flops_per_iter = lam.flops_per_iter;
        if (device_bytes) *device_bytes = host.peak_bytes;
    });
}

int ccsd_plan_export_solver(int method, int nirrep, const int* vrt, const int* occ, const int* vrt_beta,
                            const int* occ_beta, int which, const char* path) {
    return guarded(nullptr, [&] {
        if (!path) throw Error(CCSD_ERR_ARG, "null path");
        if (method == CCSD_METHOD_RHF && (vrt_beta || occ_beta))
            throw Error(CCSD_ERR_ARG, "the closed-shell solver has one set of spatial orbitals");
        if (method < CCSD_METHOD_CCSD || method > CCSD_METHOD_LAMBDA) throw Error(CCSD_ERR_ARG, "bad method");
        if (which < CCSD_PLAN_ITERATION || which > CCSD_PLAN_ENERGY) throw Error(CCSD_ERR_ARG, "bad plan");
        if (which == CCSD_PLAN_HBAR && method == CCSD_METHOD_LAMBDA) throw Error(CCSD_ERR_ARG, "Lambda forms no Hbar");
        Context host(-1, nullptr);
        int n = 0;
        host.spaces = query_spaces(nirrep, vrt, occ, n, vrt_beta, occ_beta);
        host.spaces_set = true;
        ccsd_options o;
        options_default(&o);
        Plan out;
        auto take = [&](const Plan& p) {
            Plan c = p;
            out.append(std::move(c));
        };
        // the iteration plan starts from Tau = T2 + 1/2 P(ab)P(ij) t t, which the fused Tau
        // kernel forms on the device; its statement form (the Tau plan) is exported first
        auto pick = [&](Solver& s) {
            if (which == CCSD_PLAN_ITERATION) {
                take(s.tau_plan);
                take(s.iter_plan);
            } else if (which == CCSD_PLAN_ENERGY) {
                take(s.energy_plan);
            } else {
                take(s.hbar_plan);
            }
        };
        if (method == CCSD_METHOD_RHF) {
            ccsd_rhf_hamiltonian H;
            create_rhf_hamiltonian_tensors(host, &H);
            Solver s(host, H, o);
            if (which == CCSD_PLAN_HBAR) s.hbar_rhf();
            pick(s);
            export_plan(host, out, path);
            return;
        }
        ccsd_hamiltonian H;
        create_hamiltonian_tensors(host, false, &H);
        Solver cc(host, H, o);
        if (method == CCSD_METHOD_CCSD) {
            if (which == CCSD_PLAN_HBAR) cc.hbar_so();
            pick(cc);
            export_plan(host, out, path);
            return;
        }
        cc.hbar_so();
        Solver lam(host, cc, cc.HB, o);
        pick(lam);
        export_plan(host, out, path);
    });
}

int ccsd_solver_create(ccsd_ctx ctx, const ccsd_hamiltonian* H, const ccsd_options* opts, ccsd_solver* out) {
    if (!out) return CCSD_ERR_ARG;
    *out = nullptr;
    return guarded(ctx, [&] {
        if (!H) throw Error(CCSD_ERR_ARG, "null hamiltonian");
        Context* c = device_handle(ctx);
        ccsd_options o;
        options_default(&o);
        if (opts) o = *opts;
        if (o.precision != CCSD_PREC_FP64 && !kern::split_supported())
            throw Error(CCSD_ERR_UNSUPPORTED, "split GEMMs need an sm_100 device");
        auto* h = new ccsd_solver_s;
        h->ctx = ctx;
        try {
            h->s = new Solver(*c, *H, o);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int ccsd_lambda_solver_create(ccsd_ctx ctx, const ccsd_hamiltonian* hbar, ccsd_solver ccsd, const ccsd_options* opts,
                              ccsd_solver* out) {
    if (!out) return CCSD_ERR_ARG;
    *out = nullptr;
    return guarded(ctx, [&] {
        if (!hbar || !ccsd || !ccsd->s) throw Error(CCSD_ERR_ARG, "null Hbar or CCSD solver");
        Context* c = device_handle(ctx);
        if (ccsd->ctx != ctx) throw Error(CCSD_ERR_ARG, "the CCSD solver belongs to another context");
        ccsd_options o;
        options_default(&o);
        if (opts) o = *opts;
        if (o.precision != CCSD_PREC_FP64 && !kern::split_supported())
            throw Error(CCSD_ERR_UNSUPPORTED, "split GEMMs need an sm_100 device");
        auto* h = new ccsd_solver_s;
        h->ctx = ctx;
        try {
            h->s = new Solver(*c, *ccsd->s, *hbar, o);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

// ---- DIIS over caller tensors (diis.hpp:36-228) ----------------------------------------

struct ccsd_diis_s {
    ccsd_ctx ctx = nullptr;
    DiisRing* d = nullptr;
};

int ccsd_diis_create(ccsd_ctx ctx, int order, int start, double damping, ccsd_diis* out) {
    if (!out) return CCSD_ERR_ARG;
    *out = nullptr;
    return guarded(ctx, [&] {
        Context* c = device_handle(ctx);
        auto* h = new ccsd_diis_s;
        h->ctx = ctx;
        try {
            h->d = new DiisRing(*c, order, start, damping);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int ccsd_diis_extrapolate(ccsd_diis d, int n, const ccsd_tensor* x, const ccsd_tensor* dx, const double* weights) {
    if (!d) return CCSD_ERR_ARG;
    return guarded(d->ctx, [&] {
        if (n < 1 || !x || !dx) throw Error(CCSD_ERR_ARG, "DIIS: n >= 1 pieces and non-null x, dx needed");
        d->d->extrapolate(std::vector<int>(x, x + n), std::vector<int>(dx, dx + n), weights);
    });
}

int ccsd_diis_coefficients(ccsd_diis d, int* nvec, double* c) {
    if (!d) return CCSD_ERR_ARG;
    return guarded(d->ctx, [&] { need(nvec) = d->d->coefficients(c); });
}

int ccsd_diis_destroy(ccsd_diis d) {
    if (!d) return CCSD_ERR_ARG;
    int st = guarded(d->ctx, [&] { delete d->d; });
    delete d;
    return st;
}

int ccsd_solver_destroy(ccsd_solver s) {
    if (!s) return CCSD_ERR_ARG;
    if (s->s && s->s->lambda_users > 0)
        return guarded(s->ctx, [&] {
            throw Error(CCSD_ERR_ARG, "a Lambda solver still reads this solver's amplitudes and Hbar: destroy it first");
        });
    int st = guarded(s->ctx, [&] { delete s->s; });
    delete s;
    return st;
}

int ccsd_solver_mp2(ccsd_solver s, double* mp2) {
    if (!s) return CCSD_ERR_ARG;
    return guarded(s->ctx, [&] { need(mp2) = s->s->mp2; });
}

int ccsd_solver_iterate(ccsd_solver s, double* energy, double* conv) {
    if (!s) return CCSD_ERR_ARG;
    return guarded(s->ctx, [&] { s->s->iterate(energy, conv); });
}

int ccsd_solver_iterate_async(ccsd_solver s) {
    if (!s) return CCSD_ERR_ARG;
    return guarded(s->ctx, [&] { s->s->iterate_async(); });
}

int ccsd_solver_status(ccsd_solver s, double* energy, double* conv, int* iterations) {
    if (!s) return CCSD_ERR_ARG;
    return guarded(s->ctx, [&] {
        s->s->read_status();
        if (energy) *energy = s->s->energy;
        if (conv) *conv = s->s->conv;
        if (iterations) *iterations = s->s->iterations;
    });
}

int ccsd_solver_run(ccsd_solver s, double* energy, double* conv, int* iterations) {
    if (!s) return CCSD_ERR_ARG;
    int status = CCSD_OK;
    int g = guarded(s->ctx, [&] { status = s->s->run(energy, conv, iterations); });
    return g != CCSD_OK ? g : status;
}

int ccsd_solver_amplitudes(ccsd_solver s, ccsd_tensor* T1, ccsd_tensor* T2) {
    if (!s) return CCSD_ERR_ARG;
    return guarded(s->ctx, [&] {
        if (T1) *T1 = s->s->T1;
        if (T2) *T2 = s->s->T2;
    });
}

int ccsd_rhf_solver_hbar(ccsd_solver s, ccsd_rhf_hbar* out) {
    if (!s || !out) return CCSD_ERR_ARG;
    return guarded(s->ctx, [&] {
        Solver& v = *s->s;
        v.hbar_rhf();
        out->FME = v.FME;
        out->FMI = v.FMI;
        out->FAE = v.FAE;
        out->WMNIJ = v.WMNIJ;
        out->WMNEJ = v.WMNEJ;
        out->WAMIJ = v.WAMIJ;
        out->WAMIE = v.WAMIE;
        out->WAMEI = v.WAMEI;
        out->WABEJ = v.WABEJ;
    });
}

int ccsd_solver_hbar(ccsd_solver s, ccsd_hamiltonian* out) {
    if (!s || !out) return CCSD_ERR_ARG;
    return guarded(s->ctx, [&] {
        s->s->hbar_so();
        *out = s->s->HB;
    });
}

int ccsd_solver_flops(ccsd_solver s, double* flops) {
    if (!s) return CCSD_ERR_ARG;
    return guarded(s->ctx, [&] { need(flops) = s->s->flops_per_iter; });
}

int ccsd_slice_choice(int n, const double* dE, double budget, int* drop) {
    return guarded(nullptr, [&] {
        if (n < 0 || (n > 0 && (!dE || !drop))) throw Error(CCSD_ERR_ARG, "ccsd_slice_choice: bad arguments");
        const std::vector<int> d = slice_choice(std::vector<double>(dE, dE + n), budget);
        for (int i = 0; i < n; i++) drop[i] = d[i];
    });
}

int ccsd_solver_slice_report(ccsd_solver s, char* buf, int64_t len, int64_t* needed) {
    if (!s) return CCSD_ERR_ARG;
    return guarded(s->ctx, [&] {
        Solver& v = *s->s;
        const int base = v.mode_slices >= 3 ? v.mode_slices : 3;
        std::string out;
        std::vector<std::string> seen;
        auto line = [&](const std::string& label, int slices, double dE) {
            char head[64];
            std::snprintf(head, sizeof(head), "%d\t%.6e\t", slices, dE);
            out += head + label + "\n";
        };
        if (!v.tune_report.empty()) {
            for (auto& e : v.tune_report) line(e.label, std::max(3, base + e.delta), e.dE);
        } else if (v.ctx.split_precision() || v.mode_precision != CCSD_PREC_FP64) {
            const int saved_p = v.ctx.precision, saved_s = v.ctx.slices;
            v.use_mode();
            for (auto& g : v.iter_plan.gemms)
                if (v.ctx.routes_split(g) && std::find(seen.begin(), seen.end(), g.label) == seen.end()) {
                    seen.push_back(g.label);
                    line(g.label, base, 0.0);
                }
            v.ctx.precision = saved_p;
            v.ctx.slices = saved_s;
        }
        need(needed) = (int64_t)out.size() + 1;
        if (buf && len > 0) {
            const size_t n = std::min<size_t>(out.size(), (size_t)len - 1);
            std::memcpy(buf, out.data(), n);
            buf[n] = 0;
        }
    });
}

int ccsd_solver_mode(ccsd_solver s, int* precision, int* slices) {
    if (!s) return CCSD_ERR_ARG;
    return guarded(s->ctx, [&] {
        if (precision) *precision = s->s->mode_precision;
        if (slices) *slices = s->s->mode_slices >= 3 ? s->s->mode_slices : 3;
    });
}

}  // extern "C"
