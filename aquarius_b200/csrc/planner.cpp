// Statement planner.
//
// A spin-orbital statement  C[idxC] = beta*C + alpha*A[idxA]*B[idxB]  is expanded into
// block contractions exactly as the reference's spin-orbital layer does
// (src/tensor/spinorbital_tensor.cxx:455-790 for mult, :793-1018 for sum):
//
//  1. external lines of C are split, per orbital space and separately for upper and
//     lower indices, into the lines coming from A, from B and from neither; when more
//     than one of those sets is non-empty the result is antisymmetrised over them
//     (the P(ab|c)-type operator built by Diagram::antisymmetrize, :637-669; for sum
//     only when both "in A" and "not in A" are present, :910-932);
//  2. every spin assignment of the lines is enumerated (Diagram::convert(UHF)); a
//     factor whose indices are not in the alpha-first order of its stored spin case
//     is reordered with the sign of the permutation (all groups are antisymmetric);
//  3. every irrep assignment with totally symmetric blocks is enumerated
//     (SymmetryBlockedTensor::mult, src/tensor/symblocked_tensor.cxx:1031-1088);
//  4. beta is applied once to each block of C that receives a contribution
//     (:1058-1062), before its first contribution.
//
// Tensors are stored unpacked, so step 2 sums over full spin-orbital ranges and no
// overcounting factor is needed.  Two pair restrictions recover the reference's packed
// flop counts: an internal pair antisymmetric in both factors is summed over e<f
// with a factor 2, and an external pair antisymmetric in one factor and in C is
// computed for x<y only and written to C twice with opposite signs.  Tensors created
// packed (V_abcd) are only ever read through such restricted pairs.
#include <algorithm>
#include <numeric>
#include <set>
#include <sstream>
#include <cstring>

#include "engine.hpp"

namespace ccsd {

void Plan::append(Plan&& o) {
    for (auto& s : o.steps) {
        Step t = s;
        switch (s.kind) {
            case Step::GEMM: t.idx += (int)gemms.size(); break;
            case Step::SUM: t.idx += (int)sums.size(); break;
            case Step::SCALE: t.idx += (int)scales.size(); break;
            case Step::DOT: t.idx += (int)dots.size(); break;
        }
        steps.push_back(t);
    }
    for (auto& g : o.gemms) gemms.push_back(std::move(g));
    for (auto& g : o.sums) sums.push_back(g);
    for (auto& g : o.scales) scales.push_back(g);
    for (auto& g : o.dots) dots.push_back(g);
    scratch_elems = std::max(scratch_elems, o.scratch_elems);
}

namespace {

[[noreturn]] void fail(int code, const std::string& msg) { throw Error(code, msg); }

int perm_parity(const std::vector<int>& p) {
    std::vector<int> q = p;
    int par = 0;
    for (size_t i = 0; i < q.size(); i++) {
        while (q[i] != (int)i) {
            std::swap(q[i], q[q[i]]);
            par ^= 1;
        }
    }
    return par;
}

// A "variable" of a block einsum: either C position p (external) or an internal letter.
struct Var {
    int space = 0, spin = 0, irrep = 0;
    int len = 0;
};

struct Operand {
    const Tensor* t = nullptr;
    int cs = -1;                       // spin case
    const Block* blk = nullptr;
    std::vector<int> var;              // variable per canonical position
};

// Canonical (alpha-first within each group) reordering of a factor's positions.
// spin_of_pos: spin per original position. Returns false if no such spin case.
bool canonical(const Tensor& T, const std::vector<int>& spin_of_pos, std::vector<int>& order, int& sign,
               int& cs) {
    int alpha[4] = {0, 0, 0, 0};
    for (int p = 0; p < T.ndim; p++)
        if (spin_of_pos[p] == ALPHA) alpha[T.group[p]]++;
    cs = T.find_case(alpha);
    if (cs < 0) return false;
    order.clear();
    for (int g = 0; g < 4; g++) {
        for (int pass = 0; pass < 2; pass++)
            for (int p = 0; p < T.ndim; p++)
                if (T.group[p] == g && spin_of_pos[p] == (pass == 0 ? ALPHA : BETA)) order.push_back(p);
    }
    sign = perm_parity(order) ? -1 : 1;
    return true;
}

struct Letters {
    // letter -> positions in A, B, C (-1 if absent)
    std::map<char, int> inA, inB, inC;
    std::map<char, int> space;
};

void index_check(const Tensor& T, const std::string& idx, const char* which, std::map<char, int>& pos,
                 std::map<char, int>& space) {
    if ((int)idx.size() != T.ndim)
        fail(CCSD_ERR_ARG, std::string("index string '") + idx + "' does not match the rank of " + T.name);
    for (int p = 0; p < T.ndim; p++) {
        char c = idx[p];
        if (pos.count(c)) fail(CCSD_ERR_PLAN, std::string("repeated index '") + c + "' in " + which);
        pos[c] = p;
        int sp = group_space(T.group[p]);
        auto it = space.find(c);
        if (it != space.end() && it->second != sp)
            fail(CCSD_ERR_ARG, std::string("index '") + c + "' used for both occupied and virtual lines");
        space[c] = sp;
    }
}

// Shuffles of one group of C positions over sub-groups (letters keep their relative order
// inside a sub-group).  Output: list of (mapping letter-slot -> C position, sign).
struct Shuffle {
    std::vector<int> target;   // for k-th position of the group (in C order), the C position its letter maps to
    int sign;
};

std::vector<Shuffle> group_shuffles(const std::vector<int>& positions, const std::vector<int>& sub) {
    int n = (int)positions.size();
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    std::vector<Shuffle> out;
    int nsub = 0;
    for (int s : sub) nsub = std::max(nsub, s + 1);
    std::set<int> distinct(sub.begin(), sub.end());
    if (distinct.size() <= 1) {
        out.push_back({positions, 1});
        return out;
    }
    do {
        bool ok = true;
        for (int a = 0; a < n && ok; a++)
            for (int b = a + 1; b < n && ok; b++)
                if (sub[a] == sub[b] && perm[a] > perm[b]) ok = false;
        if (!ok) continue;
        Shuffle sh;
        sh.target.resize(n);
        for (int a = 0; a < n; a++) sh.target[a] = positions[perm[a]];
        sh.sign = perm_parity(perm) ? -1 : 1;
        out.push_back(sh);
    } while (std::next_permutation(perm.begin(), perm.end()));
    return out;
}

// all combinations of per-group shuffles -> letter -> C position map with total sign
void combine_shuffles(const std::vector<std::vector<int>>& grp_pos, const std::vector<std::vector<Shuffle>>& grp_sh,
                      const std::string& idxC, std::vector<std::pair<std::map<char, int>, int>>& out) {
    std::vector<size_t> sel(grp_sh.size(), 0);
    while (true) {
        std::map<char, int> m;
        int sign = 1;
        for (size_t g = 0; g < grp_sh.size(); g++) {
            const Shuffle& sh = grp_sh[g][sel[g]];
            for (size_t a = 0; a < grp_pos[g].size(); a++) m[idxC[grp_pos[g][a]]] = sh.target[a];
            sign *= sh.sign;
        }
        out.push_back({m, sign});
        size_t g = 0;
        for (; g < sel.size(); g++) {
            if (++sel[g] < grp_sh[g].size()) break;
            sel[g] = 0;
        }
        if (g == sel.size()) break;
    }
}

// enumerate all assignments of values in [0,base) to n slots
template <class F>
void for_each_assignment(int n, int base, F f) {
    std::vector<int> a(n, 0);
    while (true) {
        f(a);
        int i = 0;
        for (; i < n; i++) {
            if (++a[i] < base) break;
            a[i] = 0;
        }
        if (i == n) break;
    }
}

const Block* find_block(const Tensor& T, int cs, const std::vector<int>& irr) {
    auto& sc = T.cases[cs];
    auto it = sc.block_of.find(irr);
    if (it == sc.block_of.end()) return nullptr;
    return &sc.blocks[it->second];
}

// offset contribution of canonical position q of a block given value x (unpacked dims only)
inline int64_t pos_off(const Block& b, int q, int64_t x) { return b.stride[q] * x; }

// pair offset for a packed block pair (x at position p, y at position q, canonical order)
inline int64_t pair_off(const Block& b, const Block::Pair& pr, int64_t x, int64_t y) {
    if (pr.kind == 1) return pr.stride * (y * (y - 1) / 2 + x);
    return pr.stride * (x + (int64_t)b.len[pr.p] * y);
}

// A GEMM dimension: ordered units, each a single variable or a restricted pair
struct Unit {
    int v0 = -1, v1 = -1;     // variables (v1 >= 0 for a pair)
    bool tri = false;         // pair with equal irreps: x<y triangle; else full rectangle
    int64_t size = 0;
};

// enumerate a dimension: calls f(k, values-per-var map) for k = 0..size-1 (first unit fastest)
template <class F>
void enumerate_dim(const std::vector<Unit>& units, const std::vector<Var>& vars, F f) {
    int64_t total = 1;
    for (auto& u : units) total *= u.size;
    std::vector<int64_t> val(vars.size(), 0);
    // precompute triangle decode tables lazily per unit
    std::vector<std::vector<std::pair<int, int>>> tri(units.size());
    for (size_t i = 0; i < units.size(); i++) {
        if (units[i].v1 >= 0 && units[i].tri) {
            int n = vars[units[i].v0].len;
            for (int y = 0; y < n; y++)
                for (int x = 0; x < y; x++) tri[i].push_back({x, y});
        }
    }
    for (int64_t k = 0; k < total; k++) {
        int64_t r = k;
        for (size_t i = 0; i < units.size(); i++) {
            const Unit& u = units[i];
            int64_t c = r % u.size;
            r /= u.size;
            if (u.v1 < 0) {
                val[u.v0] = c;
            } else if (u.tri) {
                val[u.v0] = tri[i][c].first;
                val[u.v1] = tri[i][c].second;
            } else {
                int64_t n0 = vars[u.v0].len;
                val[u.v0] = c % n0;
                val[u.v1] = c / n0;
            }
        }
        f(k, val);
    }
}

constexpr int kMaxVars = 32;   // C positions + internal letters of one statement (at most 8 + 8)

// Offset table of a GEMM dimension: out[k] = base + f(values at point k), points ordered as
// enumerate_dim orders them (first unit fastest).  Every offset this planner tabulates is a
// sum of one term per unit: an operand position depends on one variable, and a packed or
// swapped pair on the two variables of one restricted-pair unit.  So each unit's terms are
// evaluated once (f at that unit's values, all other variables 0, minus f at all zeros) and
// the table is their Kronecker sum: O(points) additions instead of O(points x positions).
template <class F>
void fill_table(std::vector<int64_t>& out, const std::vector<Unit>& units, const std::vector<Var>& vars, int64_t base,
                F f) {
    // per-thread scratch: planning runs statements on several threads, and the tables of a
    // large plan are filled a few million times
    thread_local std::vector<int64_t> val, cur, next, term;
    val.assign(vars.size(), 0);
    const int64_t f0 = f(val);
    cur.assign(1, base + f0);
    for (const Unit& u : units) {
        term.resize(u.size);
        // the unit's points in enumerate_dim's order: a value, a rectangle pair (first
        // variable fastest) or a triangle pair x < y (y outer, x inner)
        if (u.v1 < 0) {
            for (int64_t c = 0; c < u.size; c++) {
                val[u.v0] = c;
                term[c] = f(val) - f0;
            }
        } else if (u.tri) {
            int64_t c = 0;
            for (int64_t y = 0; y < vars[u.v0].len; y++)
                for (int64_t x = 0; x < y; x++) {
                    val[u.v0] = x;
                    val[u.v1] = y;
                    term[c++] = f(val) - f0;
                }
        } else {
            const int64_t n0 = vars[u.v0].len;
            for (int64_t c = 0; c < u.size; c++) {
                val[u.v0] = c % n0;
                val[u.v1] = c / n0;
                term[c] = f(val) - f0;
            }
        }
        val[u.v0] = 0;
        if (u.v1 >= 0) val[u.v1] = 0;
        next.resize(cur.size() * term.size());
        for (size_t j = 0; j < term.size(); j++)
            for (size_t t = 0; t < cur.size(); t++) next[j * cur.size() + t] = cur[t] + term[j];
        cur.swap(next);
    }
    out.assign(cur.begin(), cur.end());
}

int64_t operand_offset(const Operand& op, const std::vector<int64_t>& val, const std::vector<int>& only_vars) {
    // offset of the operand element for the subset of variables `only_vars` (others 0)
    const Block& b = *op.blk;
    int64_t off = 0;
    char use[kMaxVars] = {0};   // per element: no heap allocation on the planning hot path
    for (int v : only_vars) use[v] = 1;
    int np = (int)op.var.size();
    for (int q = 0; q < np; q++) {
        if (b.pair_of(q) >= 0) continue;
        int v = op.var[q];
        if (use[v]) off += pos_off(b, q, val[v]);
    }
    for (auto& pr : b.pairs) {
        int vp = op.var[pr.p], vq = op.var[pr.q];
        bool up = use[vp], uq = use[vq];
        if (up != uq) fail(CCSD_ERR_PLAN, "packed pair split between GEMM dimensions");
        if (up) off += pair_off(b, pr, val[vp], val[vq]);
    }
    return off;
}

struct Term {
    int cC, cA, cB;
    const Block *bC, *bA, *bB;
    Operand A, B;
    std::vector<int> cvar;          // variable per C position
    std::vector<Var> vars;
    std::vector<int> mvars, nvars, kvars;
    double coef;
};

// same group and same spin in canonical case of operand
bool same_group_spin(const Operand& op, int va, int vb, const std::vector<Var>& vars) {
    int qa = -1, qb = -1;
    for (size_t q = 0; q < op.var.size(); q++) {
        if (op.var[q] == va) qa = (int)q;
        if (op.var[q] == vb) qb = (int)q;
    }
    if (qa < 0 || qb < 0) return false;
    return op.t->group[qa] == op.t->group[qb] && vars[va].spin == vars[vb].spin;
}

int pos_in(const Operand& op, int v) {
    for (size_t q = 0; q < op.var.size(); q++)
        if (op.var[q] == v) return (int)q;
    return -1;
}

// Build units for a list of variables following `order_op`'s position order, pairing
// variables listed in `pairs`.
std::vector<Unit> make_units(const std::vector<int>& vlist, const std::vector<std::pair<int, int>>& pairs,
                             const Operand& order_op, const std::vector<Var>& vars) {
    std::vector<int> sorted = vlist;
    std::sort(sorted.begin(), sorted.end(), [&](int a, int b) { return pos_in(order_op, a) < pos_in(order_op, b); });
    std::vector<Unit> units;
    std::set<int> done;
    for (int v : sorted) {
        if (done.count(v)) continue;
        Unit u;
        u.v0 = v;
        for (auto& pr : pairs) {
            if (pr.first == v || pr.second == v) {
                int a = pr.first, b = pr.second;
                if (pos_in(order_op, a) > pos_in(order_op, b)) std::swap(a, b);
                u.v0 = a;
                u.v1 = b;
            }
        }
        if (u.v1 >= 0) {
            done.insert(u.v0);
            done.insert(u.v1);
            u.tri = vars[u.v0].irrep == vars[u.v1].irrep;
            int64_t n0 = vars[u.v0].len, n1 = vars[u.v1].len;
            u.size = u.tri ? n0 * (n0 - 1) / 2 : n0 * n1;
        } else {
            done.insert(v);
            u.size = vars[v].len;
        }
        units.push_back(u);
    }
    return units;
}

bool unit_ok(const std::vector<Unit>& units, const std::vector<Var>& vars) {
    for (auto& u : units)
        if (u.v1 >= 0 && vars[u.v0].irrep > vars[u.v1].irrep) return false;
    for (auto& u : units)
        if (u.size == 0) return false;
    return true;
}

// Destination of a lowered block contraction: a block of C (external pair restrictions
// allowed), or the plan's scratch product X with the given strides per C position.
struct Dest {
    int handle = 0;
    bool scratch = false;
    std::vector<int64_t> stride;   // per C position (scratch only)
};

void lower_gemm(Context& ctx, Term& t, int hA, int hB, int hC, int cc, std::set<std::pair<int, int>>& touched,
                Plan& plan, const Dest* dest_x = nullptr) {
    const auto& vars = t.vars;
    if ((int)vars.size() > kMaxVars) fail(CCSD_ERR_PLAN, "too many index letters in one statement");
    // pair restrictions
    std::vector<std::pair<int, int>> kpairs, mpairs, npairs;
    double factor = 1.0;
    auto find_pairs = [&](const std::vector<int>& vl, const Operand& op1, const Operand* op2,
                          std::vector<std::pair<int, int>>& out, bool external) {
        if (op1.t->plain()) return;   // no antisymmetric pairs in plain tensors
        std::set<int> used;
        for (size_t i = 0; i < vl.size(); i++)
            for (size_t j = i + 1; j < vl.size(); j++) {
                int a = vl[i], b = vl[j];
                if (used.count(a) || used.count(b)) continue;
                if (!same_group_spin(op1, a, b, vars)) continue;
                if (op2 && !same_group_spin(*op2, a, b, vars)) continue;
                if (external) {
                    // C positions a,b must be in the same group of C with equal spin
                    const Tensor& C = *ctx.tensors.at(hC);
                    int pa = -1, pb = -1;
                    for (size_t p = 0; p < t.cvar.size(); p++) {
                        if (t.cvar[p] == a) pa = (int)p;
                        if (t.cvar[p] == b) pb = (int)p;
                    }
                    if (C.group[pa] != C.group[pb]) continue;
                }
                // only restrict groups that are exactly a pair of this spin in op1
                int q1 = pos_in(op1, a);
                int cnt = 0;
                for (size_t q = 0; q < op1.var.size(); q++)
                    if (op1.t->group[q] == op1.t->group[q1] && vars[op1.var[q]].spin == vars[a].spin) cnt++;
                if (cnt != 2) continue;
                used.insert(a);
                used.insert(b);
                out.push_back({a, b});
            }
    };
    find_pairs(t.kvars, t.A, &t.B, kpairs, false);
    if (!dest_x) {
        find_pairs(t.mvars, t.A, nullptr, mpairs, true);
        find_pairs(t.nvars, t.B, nullptr, npairs, true);
    }
    for (size_t i = 0; i < kpairs.size(); i++) factor *= 2.0;

    // packed operands must be read through restricted pairs only
    for (const Operand* op : {&t.A, &t.B}) {
        const Block& b = *op->blk;
        for (auto& bp : b.pairs) {
            int va = op->var[bp.p], vb = op->var[bp.q];
            bool ok = false;
            for (auto* pl : {&kpairs, &mpairs, &npairs})
                for (auto& pr : *pl)
                    if ((pr.first == va && pr.second == vb) || (pr.first == vb && pr.second == va)) ok = true;
            if (!ok) fail(CCSD_ERR_PLAN, "packed tensor " + op->t->name + " used with a split antisymmetric pair");
        }
    }

    auto mu = make_units(t.mvars, mpairs, t.A, vars);
    auto nu = make_units(t.nvars, npairs, t.B, vars);
    auto ku = make_units(t.kvars, kpairs, t.A, vars);
    if (!unit_ok(mu, vars) || !unit_ok(nu, vars) || !unit_ok(ku, vars)) return;

    GemmStep g;
    g.tA = hA;
    g.tB = hB;
    g.tC = dest_x ? kScratch : hC;
    int64_t M = 1, N = 1, K = 1;
    for (auto& u : mu) M *= u.size;
    for (auto& u : nu) N *= u.size;
    for (auto& u : ku) K *= u.size;
    if (M > INT32_MAX || N > INT32_MAX || K > INT32_MAX) fail(CCSD_ERR_PLAN, "GEMM dimension exceeds 2^31");
    g.M = (int)M;
    g.N = (int)N;
    g.K = (int)K;
    g.alpha = t.coef * factor;

    {
        auto key_of = [&](const std::vector<int>& vl, const std::vector<std::pair<int, int>>& prs) {
            std::string s;
            for (int v : vl)
                s += std::to_string(v) + ':' + std::to_string(vars[v].space) + std::to_string(vars[v].spin) + ':' +
                     std::to_string(vars[v].irrep) + ',';
            for (auto& pr : prs) s += 'p' + std::to_string(pr.first) + '-' + std::to_string(pr.second) + ',';
            return s;
        };
        g.mkey = std::to_string(hA) + '|' + std::to_string(g.tC) + '|' + key_of(t.mvars, mpairs);
        g.nkey = std::to_string(hB) + '|' + key_of(t.nvars, npairs);
        g.kkey = key_of(t.kvars, kpairs);
    }
    std::vector<int> all_m = t.mvars, all_n = t.nvars, all_k = t.kvars;
    const Block& bA = *t.A.blk;
    const Block& bB = *t.B.blk;
    const Block& bC = *t.bC;
    fill_table(g.hAm, mu, vars, bA.offset, [&](const std::vector<int64_t>& val) { return operand_offset(t.A, val, all_m); });
    fill_table(g.hAk, ku, vars, 0, [&](const std::vector<int64_t>& val) { return operand_offset(t.A, val, all_k); });
    fill_table(g.hBk, ku, vars, 0, [&](const std::vector<int64_t>& val) { return operand_offset(t.B, val, all_k); });
    fill_table(g.hBn, nu, vars, bB.offset, [&](const std::vector<int64_t>& val) { return operand_offset(t.B, val, all_n); });
    if (dest_x) {
        // plain column-major scratch product: no variants
        g.nvm = g.nvn = 1;
        std::vector<char> um(vars.size(), 0), un(vars.size(), 0);
        for (int v : all_m) um[v] = 1;
        for (int v : all_n) un[v] = 1;
        fill_table(g.hCm[0], mu, vars, 0, [&](const std::vector<int64_t>& val) {
            int64_t off = 0;
            for (size_t p = 0; p < t.cvar.size(); p++)
                if (um[t.cvar[p]]) off += dest_x->stride[p] * val[t.cvar[p]];
            return off;
        });
        fill_table(g.hCn[0], nu, vars, 0, [&](const std::vector<int64_t>& val) {
            int64_t off = 0;
            for (size_t p = 0; p < t.cvar.size(); p++)
                if (un[t.cvar[p]]) off += dest_x->stride[p] * val[t.cvar[p]];
            return off;
        });
    } else {
        // C destinations (C unpacked): variants swap the values (and irreps) of restricted pairs;
        // a swapped pair with unequal irreps lands in the C block with those irreps exchanged.
        const Tensor& Ct = *ctx.tensors.at(hC);
        g.nvm = mpairs.empty() ? 1 : 2;
        g.nvn = npairs.empty() ? 1 : 2;
        if (mpairs.size() > 1 || npairs.size() > 1) fail(CCSD_ERR_PLAN, "more than one restricted output pair per factor");
        const Block* dest[2][2];
        for (int a = 0; a < g.nvm; a++)
            for (int b = 0; b < g.nvn; b++) {
                std::vector<int> irr = bC.irrep;
                if (a) std::swap(irr[mpairs[0].first], irr[mpairs[0].second]);
                if (b) std::swap(irr[npairs[0].first], irr[npairs[0].second]);
                dest[a][b] = find_block(Ct, cc, irr);
                if (!dest[a][b]) fail(CCSD_ERR_PLAN, "missing destination block for a restricted pair");
                touched.insert({cc, (int)Ct.cases[cc].block_of.at(irr)});
            }
        if (g.nvm == 2 && g.nvn == 2 && dest[1][1]->offset - dest[1][0]->offset != dest[0][1]->offset - dest[0][0]->offset)
            fail(CCSD_ERR_PLAN, "restricted pairs in both dimensions across irrep blocks");
        auto c_off = [&](const std::vector<int64_t>& val, const std::vector<int>& vl, int swapmask,
                         const std::vector<std::pair<int, int>>& prs, const Block& blk) {
            // variable whose value each variable takes (a restricted pair swapped in variant 1)
            int src[kMaxVars];
            char use[kMaxVars] = {0};
            for (size_t v = 0; v < vars.size(); v++) src[v] = (int)v;
            if (swapmask)
                for (auto& pr : prs) std::swap(src[pr.first], src[pr.second]);
            for (int v : vl) use[v] = 1;
            int64_t off = 0;
            for (size_t p = 0; p < t.cvar.size(); p++)
                if (use[t.cvar[p]]) off += blk.stride[p] * val[src[t.cvar[p]]];
            return off;
        };
        for (int v = 0; v < g.nvm; v++) {
            const Block& blk = *dest[v][0];
            fill_table(g.hCm[v], mu, vars, blk.offset,
                       [&](const std::vector<int64_t>& val) { return c_off(val, all_m, v, mpairs, blk); });
        }
        for (int v = 0; v < g.nvn; v++) {
            const Block& blk = *dest[0][v];
            const int64_t shift = dest[0][v]->offset - dest[0][0]->offset;
            fill_table(g.hCn[v], nu, vars, shift,
                       [&](const std::vector<int64_t>& val) { return c_off(val, all_n, v, npairs, blk); });
        }
        for (int a = 0; a < g.nvm; a++)
            for (int b = 0; b < g.nvn; b++) g.vsign[a * g.nvn + b] = ((a + b) % 2) ? -1.0 : 1.0;
    }
    // contiguity hints
    auto contig = [](const std::vector<int64_t>& t) {
        if (t.size() < 2) return true;
        size_t bad = 0;
        for (size_t i = 1; i < t.size(); i++) bad += (t[i] - t[i - 1] != 1);
        return bad * 8 < t.size();
    };
    g.a_kcontig = contig(g.hAk);
    g.a_mcontig = contig(g.hAm);
    g.b_kcontig = contig(g.hBk);
    g.b_ncontig = contig(g.hBn);
    plan.steps.push_back({Step::GEMM, (int)plan.gemms.size()});
    plan.gemms.push_back(std::move(g));
}

std::string idx_of(const std::string& s) { return s; }

}  // namespace

// ---------------------------------------------------------------------------
// mult
// ---------------------------------------------------------------------------

Plan plan_contract(Context& ctx, double alpha, int hA, const std::string& idxA, int hB, const std::string& idxB,
                   double beta, int hC, const std::string& idxC) {
    Tensor& A = ctx.tensor(hA);
    Tensor& B = ctx.tensor(hB);
    Tensor& C = ctx.tensor(hC);
    if (hA == hC || hB == hC) fail(CCSD_ERR_ARG, "output tensor aliases an input");
    if (C.packed()) fail(CCSD_ERR_PLAN, "packed output tensors are not supported");
    // plain (spatial, no antisymmetry) statements are plain einsums: no antisymmetriser,
    // no spin cases beyond all-alpha, no pair restrictions
    const bool plain = C.plain();
    if (A.plain() != plain || B.plain() != plain)
        fail(CCSD_ERR_PLAN, "plain and spin-orbital tensors mixed in one statement");
    Letters L;
    std::map<char, int> sp;
    index_check(A, idxA, "A", L.inA, sp);
    index_check(B, idxB, "B", L.inB, sp);
    index_check(C, idxC, "C", L.inC, sp);
    std::vector<char> internal;
    for (auto& kv : L.inA) {
        char c = kv.first;
        bool b = L.inB.count(c), cc = L.inC.count(c);
        if (b && cc) fail(CCSD_ERR_PLAN, std::string("index '") + c + "' appears in A, B and C");
        if (!b && !cc) fail(CCSD_ERR_PLAN, std::string("index '") + c + "' of A is summed without a partner");
        if (b) internal.push_back(c);
    }
    for (auto& kv : L.inB) {
        char c = kv.first;
        if (!L.inA.count(c) && !L.inC.count(c))
            fail(CCSD_ERR_PLAN, std::string("index '") + c + "' of B is summed without a partner");
    }
    for (auto& kv : L.inC)
        if (!L.inA.count(kv.first) && !L.inB.count(kv.first))
            fail(CCSD_ERR_PLAN, std::string("index '") + kv.first + "' of C appears in neither factor");

    // antisymmetrisers per C group
    std::vector<std::vector<int>> grp_pos;
    std::vector<std::vector<Shuffle>> grp_sh;
    for (int g = 0; g < 4 && !plain; g++) {
        std::vector<int> pos, sub;
        for (int p = 0; p < C.ndim; p++)
            if (C.group[p] == g) {
                pos.push_back(p);
                char c = idxC[p];
                sub.push_back(L.inA.count(c) ? 0 : (L.inB.count(c) ? 1 : 2));
            }
        if (pos.empty()) continue;
        grp_pos.push_back(pos);
        grp_sh.push_back(group_shuffles(pos, sub));
    }
    std::vector<std::pair<std::map<char, int>, int>> shuffles;
    if (grp_pos.empty())
        shuffles.push_back({{}, 1});
    else
        combine_shuffles(grp_pos, grp_sh, idxC, shuffles);

    const int nint = (int)internal.size();
    const int nirr = ctx.spaces.nirrep;
    Plan plan;
    std::set<std::pair<int, int>> touched;   // (case, block) of C that received a term
    std::vector<Plan> parts;
    // products X of the multi-image groups; those that fit in kBatchX together get disjoint
    // regions of the plan scratch, so that all products of the statement can run before
    // all image sums (and be grouped into few launches)
    struct XGroup {
        Plan part;          // [zero X] [GEMMs into X] [sums X -> C], X at offset 0
        int64_t nX = 0;
        bool batched = false;
        size_t slot = 0;    // position among the statement's parts
    };
    std::vector<XGroup> xgroups;
    constexpr int64_t kBatchX = 64ll << 20;   // doubles
    int64_t batched_total = 0;

    // Internal pairs antisymmetric in both factors (same group of A and same group of B,
    // nothing else internal in those groups): the spin assignments (a,b) and (b,a) give
    // equal contributions, so only alpha-before-beta is kept, with weight 2 -- the merge
    // of equal terms done by the reference's spin integration (spinorbital_tensor.cxx:676-694).
    std::vector<std::pair<int, int>> sym_int;
    if (!plain) {
        auto group_internal_count = [&](const Tensor& T, const std::map<char, int>& pos, int g) {
            int n = 0;
            for (char c : internal)
                if (T.group[pos.at(c)] == g) n++;
            return n;
        };
        for (int i = 0; i < nint; i++)
            for (int j = i + 1; j < nint; j++) {
                int gA = A.group[L.inA[internal[i]]], gB = B.group[L.inB[internal[i]]];
                if (A.group[L.inA[internal[j]]] != gA || B.group[L.inB[internal[j]]] != gB) continue;
                if (group_internal_count(A, L.inA, gA) != 2 || group_internal_count(B, L.inB, gB) != 2) continue;
                sym_int.push_back({i, j});
            }
    }

    // external letters in C order
    std::vector<char> ext(idxC.begin(), idxC.end());

    for (size_t cc = 0; cc < C.cases.size(); cc++) {
        const SpinCase& scC = C.cases[cc];
        for (size_t bi = 0; bi < scC.blocks.size(); bi++) {
            const Block& bC = scC.blocks[bi];
            if (bC.size == 0) continue;
            // Antisymmetriser terms that only exchange C positions of equal spin and irrep
            // compute the same product; group them by the (spin, irrep) each external letter
            // receives, compute the product once and write it to every image.
            struct Group {
                std::vector<std::pair<size_t, int>> images;   // (shuffle index, sign)
                std::vector<Term> terms;                      // built with the first shuffle
            };
            std::map<std::vector<int>, Group> groups;
            std::vector<std::vector<int>> group_order;
            for (size_t si = 0; si < shuffles.size(); si++) {
                auto& sh = shuffles[si];
                std::vector<int> key;
                for (char c : ext) {
                    int p = sh.first.count(c) ? sh.first.at(c) : L.inC[c];
                    key.push_back(scC.spin[p]);
                    key.push_back(bC.irrep[p]);
                }
                auto it = groups.find(key);
                if (it != groups.end()) {
                    it->second.images.push_back({si, sh.second});
                    continue;
                }
                Group& G = groups[key];
                group_order.push_back(key);
                G.images.push_back({si, sh.second});
                for_each_assignment(nint, 2, [&](const std::vector<int>& ispin) {
                    double wspin = 1.0;
                    for (auto& pr : sym_int) {
                        if (ispin[pr.first] > ispin[pr.second]) return;
                        if (ispin[pr.first] < ispin[pr.second]) wspin *= 2.0;
                    }
                    // variables: 0..C.ndim-1 = C positions, then internal letters
                    std::vector<Var> vars(C.ndim + nint);
                    std::map<char, int> var_of;
                    for (int p = 0; p < C.ndim; p++) {
                        vars[p].space = group_space(C.group[p]);
                        vars[p].spin = scC.spin[p];
                        vars[p].irrep = bC.irrep[p];
                        vars[p].len = ctx.spaces.n[vars[p].space][vars[p].spin][vars[p].irrep];
                    }
                    // external letters sit at their own C position unless the shuffle moves them
                    for (char c : ext) var_of[c] = L.inC[c];
                    for (auto& kv : sh.first) var_of[kv.first] = kv.second;
                    for (int i = 0; i < nint; i++) {
                        var_of[internal[i]] = C.ndim + i;
                        vars[C.ndim + i].space = sp[internal[i]];
                        vars[C.ndim + i].spin = ispin[i];
                    }
                    // canonical forms of A and B
                    std::vector<int> spinA(A.ndim), spinB(B.ndim);
                    for (int p = 0; p < A.ndim; p++) spinA[p] = vars[var_of[idxA[p]]].spin;
                    for (int p = 0; p < B.ndim; p++) spinB[p] = vars[var_of[idxB[p]]].spin;
                    std::vector<int> ordA, ordB;
                    int sgA, sgB, csA, csB;
                    if (!canonical(A, spinA, ordA, sgA, csA)) return;
                    if (!canonical(B, spinB, ordB, sgB, csB)) return;
                    for_each_assignment(nint, nirr, [&](const std::vector<int>& iirr) {
                        std::vector<Var> vv = vars;
                        for (int i = 0; i < nint; i++) {
                            vv[C.ndim + i].irrep = iirr[i];
                            vv[C.ndim + i].len = ctx.spaces.n[vv[C.ndim + i].space][vv[C.ndim + i].spin][iirr[i]];
                        }
                        Term t;
                        t.vars = vv;
                        t.cvar.resize(C.ndim);
                        for (int p = 0; p < C.ndim; p++) t.cvar[p] = p;
                        t.A.t = &A;
                        t.A.cs = csA;
                        t.B.t = &B;
                        t.B.cs = csB;
                        std::vector<int> irrA(A.ndim), irrB(B.ndim);
                        t.A.var.resize(A.ndim);
                        t.B.var.resize(B.ndim);
                        for (int q = 0; q < A.ndim; q++) {
                            t.A.var[q] = var_of[idxA[ordA[q]]];
                            irrA[q] = vv[t.A.var[q]].irrep;
                        }
                        for (int q = 0; q < B.ndim; q++) {
                            t.B.var[q] = var_of[idxB[ordB[q]]];
                            irrB[q] = vv[t.B.var[q]].irrep;
                        }
                        t.A.blk = find_block(A, csA, irrA);
                        t.B.blk = find_block(B, csB, irrB);
                        // beta applies to every C block for which both factor blocks exist
                        // (totally symmetric irrep tuples), even when they are empty
                        // (symblocked_tensor.cxx:1033-1062).  Packed factors store only the
                        // irrep-ordered half of their pair blocks; the other half is reached
                        // through the pair restriction, so existence is decided by symmetry.
                        int xa = 0, xb = 0;
                        for (int h : irrA) xa ^= h;
                        for (int h : irrB) xb ^= h;
                        if (xa == 0 && xb == 0) touched.insert({(int)cc, (int)bi});
                        if (!t.A.blk || !t.B.blk) return;
                        if (t.A.blk->size == 0 || t.B.blk->size == 0) return;
                        t.bC = &bC;
                        t.coef = alpha * wspin * sgA * sgB;   // shuffle sign applied per image
                        // m: C positions whose variable appears in A; n: in B
                        for (int q = 0; q < A.ndim; q++)
                            if (t.A.var[q] < C.ndim) t.mvars.push_back(t.A.var[q]);
                        for (int q = 0; q < B.ndim; q++)
                            if (t.B.var[q] < C.ndim) t.nvars.push_back(t.B.var[q]);
                        for (int i = 0; i < nint; i++) t.kvars.push_back(C.ndim + i);
                        G.terms.push_back(std::move(t));
                    });
                });
            }
            for (auto& key : group_order) {
                Group& G = groups[key];
                if (G.terms.empty()) continue;
                if (G.images.size() == 1) {
                    // a single image: contract straight into C
                    for (auto& t : G.terms) {
                        t.coef *= G.images[0].second;
                        Plan part;
                        lower_gemm(ctx, t, hA, hB, hC, (int)cc, touched, part);
                        if (!part.gemms.empty()) parts.push_back(std::move(part));
                    }
                    continue;
                }
                // several images: X[letters] = product (first shuffle), then C += sign * X per image
                const auto& sh0 = shuffles[G.images[0].first].first;
                const int ne = (int)ext.size();
                std::vector<int64_t> lenX(ne), strideX(ne);
                int64_t nX = 1;
                for (int k = 0; k < ne; k++) {
                    lenX[k] = ctx.spaces.n[group_space(C.group[L.inC[ext[k]]])][key[2 * k]][key[2 * k + 1]];
                    strideX[k] = nX;
                    nX *= lenX[k];
                }
                Dest dx;
                dx.scratch = true;
                dx.stride.assign(C.ndim, 0);
                for (int k = 0; k < ne; k++) {
                    int p0 = sh0.count(ext[k]) ? sh0.at(ext[k]) : L.inC[ext[k]];
                    dx.stride[p0] = strideX[k];
                }
                Plan part;
                part.scratch_elems = nX;
                {
                    ScaleStep z;
                    z.tC = kScratch;
                    z.off = 0;
                    z.n = nX;
                    z.beta = 0.0;
                    part.steps.push_back({Step::SCALE, (int)part.scales.size()});
                    part.scales.push_back(z);
                }
                for (auto& t : G.terms) lower_gemm(ctx, t, hA, hB, hC, (int)cc, touched, part, &dx);
                for (auto& im : G.images) {
                    const auto& shm = shuffles[im.first].first;
                    SumStep s;
                    s.tA = kScratch;
                    s.tC = hC;
                    s.ndim = ne;
                    s.offA = 0;
                    s.offC = bC.offset;
                    s.alpha = im.second;
                    for (int k = 0; k < ne; k++) {
                        int p = shm.count(ext[k]) ? shm.at(ext[k]) : L.inC[ext[k]];
                        s.len[k] = lenX[k];
                        s.sA[k] = strideX[k];
                        s.sC[k] = bC.stride[p];
                    }
                    part.steps.push_back({Step::SUM, (int)part.sums.size()});
                    part.sums.push_back(s);
                }
                XGroup xg;
                xg.nX = nX;
                xg.batched = batched_total + nX <= kBatchX;
                if (xg.batched) batched_total += nX;
                xg.part = std::move(part);
                // the group's products keep their place among the direct products
                xg.slot = parts.size();
                parts.push_back(Plan());
                xgroups.push_back(std::move(xg));
            }
        }
    }
    // beta once per touched block, before any contribution (no contribution reads C)
    if (beta != 1.0) {
        for (auto& cb : touched) {
            const Block& b = C.cases[cb.first].blocks[cb.second];
            ScaleStep s;
            s.tC = hC;
            s.off = b.offset;
            s.n = b.size;
            s.beta = beta;
            plan.steps.push_back({Step::SCALE, (int)plan.scales.size()});
            plan.scales.push_back(s);
        }
    }
    // Batched groups: one zero-fill of their regions, their products in group order among
    // the direct products, then all their image sums; the other groups (X too large to
    // keep apart) follow one by one, each reusing the start of the scratch.
    Plan sums;
    int64_t off = 0, classic_max = 0;
    std::vector<Plan> classic;
    if (batched_total > 0) {
        ScaleStep z;
        z.tC = kScratch;
        z.off = 0;
        z.n = batched_total;
        z.beta = 0.0;
        plan.steps.push_back({Step::SCALE, (int)plan.scales.size()});
        plan.scales.push_back(z);
    }
    for (auto& xg : xgroups) {
        const size_t slot = xg.slot;
        if (!xg.batched) {
            classic_max = std::max(classic_max, xg.nX);
            classic.push_back(std::move(xg.part));
            continue;
        }
        Plan g;
        for (auto& st : xg.part.steps) {
            if (st.kind == Step::GEMM) {
                GemmStep gs = std::move(xg.part.gemms[st.idx]);
                for (auto& v : gs.hCm[0]) v += off;
                g.steps.push_back({Step::GEMM, (int)g.gemms.size()});
                g.gemms.push_back(std::move(gs));
            } else if (st.kind == Step::SUM) {
                SumStep s = xg.part.sums[st.idx];
                s.offA += off;
                sums.steps.push_back({Step::SUM, (int)sums.sums.size()});
                sums.sums.push_back(s);
            }
        }
        parts[slot] = std::move(g);
        off += xg.nX;
    }
    for (auto& p : parts) plan.append(std::move(p));
    plan.append(std::move(sums));
    for (auto& p : classic) plan.append(std::move(p));
    plan.scratch_elems = std::max(plan.scratch_elems, std::max(batched_total, classic_max));
    return plan;
}

// ---------------------------------------------------------------------------
// sum
// ---------------------------------------------------------------------------

Plan plan_sum(Context& ctx, double alpha, int hA, const std::string& idxA, double beta, int hC,
              const std::string& idxC) {
    Tensor& A = ctx.tensor(hA);
    Tensor& C = ctx.tensor(hC);
    if (hA == hC) fail(CCSD_ERR_ARG, "sum with aliased input and output");
    if (C.packed() || A.packed()) fail(CCSD_ERR_PLAN, "sum over packed tensors is not supported");
    if (A.plain() != C.plain()) fail(CCSD_ERR_PLAN, "plain and spin-orbital tensors mixed in one sum");
    Letters L;
    std::map<char, int> sp;
    index_check(A, idxA, "A", L.inA, sp);
    index_check(C, idxC, "B", L.inC, sp);
    for (auto& kv : L.inA)
        if (!L.inC.count(kv.first)) fail(CCSD_ERR_PLAN, "traces in sum are not supported");
    for (auto& kv : L.inC)
        if (!L.inA.count(kv.first)) fail(CCSD_ERR_PLAN, "broadcast in sum is not supported");
    // every letter of C is in A, so no antisymmetriser applies (spinorbital_tensor.cxx:922)
    Plan plan;
    std::set<std::pair<int, int>> touched;
    std::vector<SumStep> parts;
    for (size_t cc = 0; cc < C.cases.size(); cc++) {
        const SpinCase& scC = C.cases[cc];
        std::vector<int> spinA(A.ndim);
        for (int p = 0; p < A.ndim; p++) spinA[p] = scC.spin[L.inC[idxA[p]]];
        std::vector<int> ordA;
        int sgA, csA;
        if (!canonical(A, spinA, ordA, sgA, csA)) continue;
        for (size_t bi = 0; bi < scC.blocks.size(); bi++) {
            const Block& bC = scC.blocks[bi];
            if (bC.size == 0) continue;
            std::vector<int> irrA(A.ndim);
            for (int q = 0; q < A.ndim; q++) irrA[q] = bC.irrep[L.inC[idxA[ordA[q]]]];
            const Block* bA = find_block(A, csA, irrA);
            if (!bA || bA->size == 0) continue;
            SumStep s;
            s.tA = hA;
            s.tC = hC;
            s.ndim = C.ndim;
            s.offA = bA->offset;
            s.offC = bC.offset;
            s.alpha = alpha * sgA;
            for (int p = 0; p < C.ndim; p++) {
                s.len[p] = bC.len[p];
                s.sC[p] = bC.stride[p];
                // canonical A position holding C position p
                int q = -1;
                for (int qq = 0; qq < A.ndim; qq++)
                    if (L.inC[idxA[ordA[qq]]] == p) q = qq;
                s.sA[p] = bA->stride[q];
            }
            touched.insert({(int)cc, (int)bi});
            parts.push_back(s);
        }
    }
    if (beta != 1.0) {
        for (auto& cb : touched) {
            const Block& b = C.cases[cb.first].blocks[cb.second];
            ScaleStep s;
            s.tC = hC;
            s.off = b.offset;
            s.n = b.size;
            s.beta = beta;
            plan.steps.push_back({Step::SCALE, (int)plan.scales.size()});
            plan.scales.push_back(s);
        }
    }
    for (auto& s : parts) {
        plan.steps.push_back({Step::SUM, (int)plan.sums.size()});
        plan.sums.push_back(s);
    }
    return plan;
}

// ---------------------------------------------------------------------------
// dot (full spin-orbital contraction to a scalar)
// ---------------------------------------------------------------------------

Plan plan_dot(Context& ctx, int hA, const std::string& idxA, int hB, const std::string& idxB) {
    Tensor& A = ctx.tensor(hA);
    Tensor& B = ctx.tensor(hB);
    if (A.packed() || B.packed()) fail(CCSD_ERR_PLAN, "dot over packed tensors is not supported");
    if (A.plain() != B.plain()) fail(CCSD_ERR_PLAN, "plain and spin-orbital tensors mixed in one dot");
    Letters L;
    std::map<char, int> sp;
    index_check(A, idxA, "A", L.inA, sp);
    index_check(B, idxB, "B", L.inB, sp);
    for (auto& kv : L.inA)
        if (!L.inB.count(kv.first)) fail(CCSD_ERR_PLAN, "dot needs every index in both factors");
    for (auto& kv : L.inB)
        if (!L.inA.count(kv.first)) fail(CCSD_ERR_PLAN, "dot needs every index in both factors");
    const int n = A.ndim;
    std::vector<char> letters(idxA.begin(), idxA.end());
    Plan plan;
    const int nirr = ctx.spaces.nirrep;
    for_each_assignment(n, 2, [&](const std::vector<int>& spin) {
        std::map<char, int> s_of;
        for (int i = 0; i < n; i++) s_of[letters[i]] = spin[i];
        std::vector<int> spinA(n), spinB(n);
        for (int p = 0; p < n; p++) spinA[p] = s_of[idxA[p]];
        for (int p = 0; p < n; p++) spinB[p] = s_of[idxB[p]];
        std::vector<int> ordA, ordB;
        int sgA, sgB, csA, csB;
        if (!canonical(A, spinA, ordA, sgA, csA)) return;
        if (!canonical(B, spinB, ordB, sgB, csB)) return;
        for_each_assignment(n, nirr, [&](const std::vector<int>& irr) {
            std::map<char, int> h_of;
            for (int i = 0; i < n; i++) h_of[letters[i]] = irr[i];
            std::vector<int> irrA(n), irrB(n);
            for (int q = 0; q < n; q++) irrA[q] = h_of[idxA[ordA[q]]];
            for (int q = 0; q < n; q++) irrB[q] = h_of[idxB[ordB[q]]];
            const Block* bA = find_block(A, csA, irrA);
            const Block* bB = find_block(B, csB, irrB);
            if (!bA || !bB || bA->size == 0) return;
            DotStep d;
            d.tA = hA;
            d.tB = hB;
            d.ndim = n;
            d.offA = bA->offset;
            d.offB = bB->offset;
            d.alpha = sgA * sgB;
            for (int q = 0; q < n; q++) {
                char c = idxA[ordA[q]];
                d.len[q] = bA->len[q];
                d.sA[q] = bA->stride[q];
                int qb = -1;
                for (int r = 0; r < n; r++)
                    if (idxB[ordB[r]] == c) qb = r;
                d.sB[q] = bB->stride[qb];
            }
            plan.steps.push_back({Step::DOT, (int)plan.dots.size()});
            plan.dots.push_back(d);
        });
    });
    return plan;
}

}  // namespace ccsd
