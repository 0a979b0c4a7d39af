// Indexed-tensor expression layer with the reference's surface syntax
// (src/tensor/indexable_tensor.hpp:133-155, 330-337; src/tensor/tensor.hpp:328-360):
//
//     Z2["abij"] += 0.5*VABEF["abef"]*Tau["efij"];
//
// Each statement is planned once (spin cases, irrep blocks, gather tables) and
// appended to a Plan that the solver replays every iteration.
#pragma once
#include <string>

#include "engine.hpp"

namespace ccsd {

struct Recorder {
    Context* ctx;
    Plan* plan;
};

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
        Plan p = plan_sum(*r->ctx, alpha, x.h, x.idx, beta, h, idx);
        std::string label = r->ctx->tensor(h).name + "[" + idx + "] += " + r->ctx->tensor(x.h).name + "[" + x.idx + "]";
        for (auto& g : p.sums) g.label = label;
        for (auto& g : p.scales) g.label = label + " (scale)";
        r->plan->append(std::move(p));
    }
    void mult(double alpha, const IndexedMult& m, double beta) {
        Plan p = plan_contract(*r->ctx, alpha, m.a.h, m.a.idx, m.b.h, m.b.idx, beta, h, idx);
        std::string label = r->ctx->tensor(h).name + "[" + idx + "] += " + r->ctx->tensor(m.a.h).name + "[" + m.a.idx +
                            "]*" + r->ctx->tensor(m.b.h).name + "[" + m.b.idx + "]";
        for (auto& g : p.gemms) g.label = label;
        for (auto& g : p.sums) g.label = label + " (images)";
        for (auto& g : p.scales) g.label = label + " (scale)";
        r->plan->append(std::move(p));
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
