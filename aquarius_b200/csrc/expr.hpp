// Indexed-tensor expression layer with the reference's surface syntax
// (src/tensor/indexable_tensor.hpp:133-155, 330-337; src/tensor/tensor.hpp:328-360):
//
//     Z2["abij"] += 0.5*VABEF["abef"]*Tau["efij"];
//
// Each statement is planned once (spin cases, irrep blocks, gather tables) and
// appended to a Plan that the solver replays every iteration.
#pragma once
#include <exception>
#include <functional>
#include <string>
#include <vector>

#include "engine.hpp"

namespace ccsd {

// With `defer` set, statements are collected and planned by run_deferred(), in parallel
// (planning reads the context's tensors only), and appended to the plan in statement order.
struct Recorder {
    Context* ctx;
    Plan* plan;
    std::vector<std::function<Plan()>>* defer = nullptr;
};

inline void run_deferred(Recorder& r) {
    if (!r.defer) return;
    auto& jobs = *r.defer;
    std::vector<Plan> out(jobs.size());
    std::vector<std::exception_ptr> err(jobs.size());
    const int nt = r.ctx->plan_threads > 0 ? r.ctx->plan_threads : 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (long i = 0; i < (long)jobs.size(); i++) {
        try {
            out[i] = jobs[i]();
        } catch (...) {
            err[i] = std::current_exception();
        }
    }
    for (auto& e : err)
        if (e) std::rethrow_exception(e);
    // one allocation per step list for the merged plan (a D2h iteration has ~10^5 GEMMs)
    size_t ng = r.plan->gemms.size(), nsu = r.plan->sums.size(), nsc = r.plan->scales.size(),
           nd = r.plan->dots.size(), nst = r.plan->steps.size();
    for (auto& p : out) {
        ng += p.gemms.size();
        nsu += p.sums.size();
        nsc += p.scales.size();
        nd += p.dots.size();
        nst += p.steps.size();
    }
    r.plan->gemms.reserve(ng);
    r.plan->sums.reserve(nsu);
    r.plan->scales.reserve(nsc);
    r.plan->dots.reserve(nd);
    r.plan->steps.reserve(nst);
    for (auto& p : out) r.plan->append(std::move(p));
    jobs.clear();
}

struct Indexed {
    Recorder* r = nullptr;
    int h = 0;
    std::string idx;
    double f = 1.0;
};

struct IndexedMult {
    Indexed a, b;
    double f = 1.0;
};

inline Indexed operator*(double f, Indexed x) {
    x.f *= f;
    return x;
}
inline IndexedMult operator*(const Indexed& a, const Indexed& b) { return IndexedMult{a, b, a.f * b.f}; }
inline IndexedMult operator*(double f, IndexedMult m) {
    m.f *= f;
    return m;
}

struct Lhs {
    Recorder* r;
    int h;
    std::string idx;
    void sum(double alpha, const Indexed& x, double beta) {
        Context* ctx = r->ctx;
        const int hc = h, ha = x.h;
        const std::string ic = idx, ia = x.idx;
        auto job = [=]() {
            Plan p = plan_sum(*ctx, alpha, ha, ia, beta, hc, ic);
            std::string label = ctx->tensor(hc).name + "[" + ic + "] += " + ctx->tensor(ha).name + "[" + ia + "]";
            for (auto& g : p.sums) g.label = label;
            for (auto& g : p.scales) g.label = label + " (scale)";
            return p;
        };
        if (r->defer) r->defer->push_back(job);
        else r->plan->append(job());
    }
    void mult(double alpha, const IndexedMult& m, double beta) {
        Context* ctx = r->ctx;
        const int hc = h, ha = m.a.h, hb = m.b.h;
        const std::string ic = idx, ia = m.a.idx, ib = m.b.idx;
        auto job = [=]() {
            Plan p = plan_contract(*ctx, alpha, ha, ia, hb, ib, beta, hc, ic);
            std::string label = ctx->tensor(hc).name + "[" + ic + "] += " + ctx->tensor(ha).name + "[" + ia + "]*" +
                                ctx->tensor(hb).name + "[" + ib + "]";
            for (auto& g : p.gemms) g.label = label;
            for (auto& g : p.sums) g.label = label + " (images)";
            for (auto& g : p.scales) g.label = label + " (scale)";
            return p;
        };
        if (r->defer) r->defer->push_back(job);
        else r->plan->append(job());
    }
    void operator=(const Indexed& x) { sum(x.f, x, 0.0); }
    void operator+=(const Indexed& x) { sum(x.f, x, 1.0); }
    void operator-=(const Indexed& x) { sum(-x.f, x, 1.0); }
    void operator=(const IndexedMult& m) { mult(m.f, m, 0.0); }
    void operator+=(const IndexedMult& m) { mult(m.f, m, 1.0); }
    void operator-=(const IndexedMult& m) { mult(-m.f, m, 1.0); }
};

// A tensor handle bound to a recorder: T["abij"] yields an Indexed on the RHS and an
// Lhs target on the left.
struct TensorRef {
    Recorder* r = nullptr;
    int h = 0;
    struct Proxy {
        Recorder* r;
        int h;
        std::string idx;
        operator Indexed() const { return Indexed{r, h, idx, 1.0}; }
        void operator=(const Indexed& x) { Lhs{r, h, idx} = x; }
        void operator+=(const Indexed& x) { Lhs{r, h, idx} += x; }
        void operator-=(const Indexed& x) { Lhs{r, h, idx} -= x; }
        void operator=(const IndexedMult& m) { Lhs{r, h, idx} = m; }
        void operator+=(const IndexedMult& m) { Lhs{r, h, idx} += m; }
        void operator-=(const IndexedMult& m) { Lhs{r, h, idx} -= m; }
        void operator=(const Proxy& x) { Lhs{r, h, idx} = Indexed(x); }
        void operator+=(const Proxy& x) { Lhs{r, h, idx} += Indexed(x); }
        void operator-=(const Proxy& x) { Lhs{r, h, idx} -= Indexed(x); }
    };
    Proxy operator[](const char* idx) const { return Proxy{r, h, idx}; }
};

inline Indexed operator*(double f, const TensorRef::Proxy& p) { return f * Indexed(p); }
inline IndexedMult operator*(const TensorRef::Proxy& a, const TensorRef::Proxy& b) { return Indexed(a) * Indexed(b); }
inline IndexedMult operator*(const Indexed& a, const TensorRef::Proxy& b) { return a * Indexed(b); }
inline IndexedMult operator*(const TensorRef::Proxy& a, const Indexed& b) { return Indexed(a) * b; }

}  // namespace ccsd
