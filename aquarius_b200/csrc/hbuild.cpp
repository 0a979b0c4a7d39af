// Device-side assembly of the 13 spin-orbital blocks of H from a three-index factor.
//
// Role of the reference's H producers (src/operator/aomoints.cxx:1357-1387 assembly,
// src/operator/fakemoints.cxx:15-52 for synthetic sizes): every two-electron block is
// the antisymmetrised physicist-notation integral
//     <pq||rs> = (pr|qs) d(sp,sr) d(sq,ss) - (ps|qr) d(sp,ss) d(sq,sr),
// with the index order [upper..., lower...] of TwoElectronOperator
// (src/operator/2eoperator.cxx:13-21), and either (pq|rs) = sum_P B[P,p,q] B[P,r,s]
// or a dense (pq|rs) array (integrals read from an FCIDUMP, src/operator/fcidump.cxx).
// With the factor, each Coulomb / exchange piece of a block is one FP64 gather-GEMM
// over P whose epilogue scatters straight into the block; with the dense array it is
// one gather launch.  Blocks stored with packed pairs (V_abcd) go through a chunked
// temporary and a pack kernel.
#include <algorithm>
#include <cstring>

#include "engine.hpp"
#include "hbuild.hpp"

namespace ccsd {

namespace {

// device copies of host index tables, freed together (staged and freed in stream order:
// no host synchronisation per block product)
struct Tables {
    Context& ctx;
    std::vector<std::pair<void*, size_t>> held;
    template <class T>
    T* up(const std::vector<T>& h) {
        T* d = (T*)ctx.dmalloc(std::max<size_t>(h.size(), 1) * sizeof(T));
        ctx.stage_h2d(d, h.data(), h.size() * sizeof(T));
        held.push_back({d, std::max<size_t>(h.size(), 1) * sizeof(T)});
        return d;
    }
    ~Tables() {
        for (auto& p : held) ctx.dfree(p.first, p.second);
    }
};

struct Builder {
    Context& ctx;
    int n, naux, o;
    double* dB = nullptr;
    std::vector<int> aux_irrep;   // per P
    bool aux_known = false;
    const double* dEri = nullptr;  // dense (pq|rs) on the device instead of the factor

    // global spatial index of (space, irrep, x)
    int gidx(int space, int irrep, int x) const {
        const Spaces& S = ctx.spaces;
        int base = space == OCC ? 0 : o;
        return base + S.off[space][ALPHA][irrep] + x;
    }

    std::vector<int64_t> aux_list(int irrep) const {
        std::vector<int64_t> k;
        for (int P = 0; P < naux; P++)
            if (!aux_known || aux_irrep[P] == irrep) k.push_back((int64_t)P * n * n);
        return k;
    }

    // dense path: C[off + sum stride*x] += sign * (g_pa g_pb | g_pc g_pd), position 0
    // shifted by a0 (one gather launch; no arithmetic beyond the sign)
    void gather(double* C, int64_t off, const int* space, const int* irrep, const int* len, const int64_t* stride,
                int pa, int pb, int pc, int pd, double sign, int a0 = 0) {
        for (int p = 0; p < 4; p++)
            if (len[p] == 0) return;
        kern::EriGatherArgs g;
        Tables tb{ctx, {}};
        for (int p = 0; p < 4; p++) {
            std::vector<int> idx(len[p]);
            for (int x = 0; x < len[p]; x++) idx[x] = gidx(space[p], irrep[p], (p == 0 ? a0 : 0) + x);
            g.g[p] = tb.up(idx);
            g.len[p] = len[p];
            g.st[p] = stride[p];
        }
        g.C = C;
        g.off = off;
        g.pos[0] = pa;
        g.pos[1] = pb;
        g.pos[2] = pc;
        g.pos[3] = pd;
        g.n = n;
        g.sign = sign;
        kern::eri_gather(g, dEri, ctx.stream);
    }

    // Symmetry-blocked H: thousands of small block products.  With `batch` set the Coulomb
    // pieces are collected per level (a block's J piece in level 0, its K piece in level 1,
    // so that every launch writes disjoint blocks) and flush() runs each level as one
    // grouped FP64 launch with its tables uploaded in one copy, instead of one launch and
    // five table uploads per piece: in the serving mix, where every launch of a small solve
    // waits for a free SM behind the tiles of the large ones, this is the build's cost.
    struct Piece {
        double* C;
        double sign;
        int M, N, K;
        std::vector<int64_t> Am, Ak, Bn, Cm, Cn;
    };
    bool batch = false;
    std::vector<Piece> level[2];

    void flush() {
        for (auto& lv : level) {
            if (lv.empty()) continue;
            std::vector<int64_t> all;
            std::vector<size_t> at;
            for (auto& pc : lv)
                for (auto* t : {&pc.Am, &pc.Ak, &pc.Bn, &pc.Cm, &pc.Cn}) {
                    at.push_back(all.size());
                    all.insert(all.end(), t->begin(), t->end());
                }
            Tables tb{ctx, {}};
            const int64_t* d = tb.up(all);
            std::vector<kern::GemmArgs> probs;
            std::vector<int> tstart;
            int tiles = 0;
            size_t q = 0;
            for (auto& pc : lv) {
                kern::GemmArgs a;
                a.A = dB;
                a.B = dB;
                a.C = pc.C;
                a.M = pc.M;
                a.N = pc.N;
                a.K = pc.K;
                a.alpha = pc.sign;
                a.Am = d + at[q++];
                a.Ak = d + at[q++];
                a.Bk = a.Ak;
                a.Bn = d + at[q++];
                a.Cm[0] = d + at[q++];
                a.Cn[0] = d + at[q++];
                probs.push_back(a);
                tstart.push_back(tiles);
                tiles += kern::fp64_tiles(pc.M, pc.N);
            }
            kern::GemmArgs* dp = (kern::GemmArgs*)ctx.dmalloc(probs.size() * sizeof(kern::GemmArgs));
            int* dt = (int*)ctx.dmalloc(tstart.size() * sizeof(int));
            ctx.stage_h2d(dp, probs.data(), probs.size() * sizeof(kern::GemmArgs));
            ctx.stage_h2d(dt, tstart.data(), tstart.size() * sizeof(int));
            kern::gemm_fp64_grouped(dp, dt, (int)probs.size(), tiles, false, false, ctx.stream);
            ctx.dfree(dp, probs.size() * sizeof(kern::GemmArgs));
            ctx.dfree(dt, tstart.size() * sizeof(int));
            lv.clear();
        }
    }

    // (x0 x1 | x2 x3) pieces over positions (pa, pb | pc, pd) of a block, scattered into
    // C with sign: C[off + sum stride*x] += sign * sum_P B[P,a,b] B[P,c,d]
    void coulomb(double* C, int64_t off, const int* space, const int* irrep, const int* len,
                 const int64_t* stride, int pa, int pb, int pc, int pd, double sign, int lvl = 0) {
        if (dEri) {
            gather(C, off, space, irrep, len, stride, pa, pb, pc, pd, sign);
            return;
        }
        int64_t M = (int64_t)len[pa] * len[pb], N = (int64_t)len[pc] * len[pd];
        if (M == 0 || N == 0) return;
        std::vector<int64_t> k = aux_list(irrep[pa] ^ irrep[pb]);
        if (k.empty()) return;
        kern::GemmArgs a;
        std::vector<int64_t> Am(M), Bn(N), Cm(M), Cn(N);
        for (int y = 0; y < len[pb]; y++)
            for (int x = 0; x < len[pa]; x++) {
                int64_t m = x + (int64_t)len[pa] * y;
                Am[m] = (int64_t)gidx(space[pa], irrep[pa], x) * n + gidx(space[pb], irrep[pb], y);
                Cm[m] = off + stride[pa] * x + stride[pb] * y;
            }
        for (int y = 0; y < len[pd]; y++)
            for (int x = 0; x < len[pc]; x++) {
                int64_t m = x + (int64_t)len[pc] * y;
                Bn[m] = (int64_t)gidx(space[pc], irrep[pc], x) * n + gidx(space[pd], irrep[pd], y);
                Cn[m] = stride[pc] * x + stride[pd] * y;
            }
        if (batch) {
            level[lvl].push_back({C, sign, (int)M, (int)N, (int)k.size(), std::move(Am), std::move(k), std::move(Bn),
                                  std::move(Cm), std::move(Cn)});
            return;
        }
        Tables tb{ctx, {}};
        int64_t *dAm = tb.up(Am), *dK = tb.up(k), *dBn = tb.up(Bn), *dCm = tb.up(Cm), *dCn = tb.up(Cn);
        a.A = dB;
        a.B = dB;
        a.C = C;
        a.M = (int)M;
        a.N = (int)N;
        a.K = (int)k.size();
        a.alpha = sign;
        a.Am = dAm;
        a.Ak = dK;
        a.Bk = dK;
        a.Bn = dBn;
        a.Cm[0] = dCm;
        a.Cn[0] = dCn;
        a.a_kcontig = false;
        a.b_kcontig = false;
        kern::gemm_fp64(a, ctx.stream);
    }

    void one_electron(int h, const double* eps) {
        Tensor& T = ctx.tensor(h);
        for (auto& sc : T.cases)
            for (auto& b : sc.blocks) {
                if (b.size == 0) continue;
                int sp0 = group_space(T.group[0]), sp1 = group_space(T.group[1]);
                if (sp0 != sp1 || b.irrep[0] != b.irrep[1] || sc.spin[0] != sc.spin[1]) continue;
                std::vector<double> host(b.size, 0.0);
                for (int x = 0; x < b.len[0]; x++) host[x + (int64_t)x * b.len[0]] = eps[gidx(sp0, b.irrep[0], x)];
                ctx.stage_h2d(T.data + b.offset, host.data(), b.size * sizeof(double));
            }
    }

    // every same-spin block of a one-electron operator from a full spatial matrix
    // f[p*n + q] (row = upper index); alpha and beta share it
    void one_electron_full(int h, const double* f) {
        Tensor& T = ctx.tensor(h);
        for (auto& sc : T.cases)
            for (auto& b : sc.blocks) {
                if (b.size == 0) continue;
                if (sc.spin[0] != sc.spin[1] || b.irrep[0] != b.irrep[1]) continue;
                const int sp0 = group_space(T.group[0]), sp1 = group_space(T.group[1]);
                std::vector<double> host(b.size, 0.0);
                for (int y = 0; y < b.len[1]; y++)
                    for (int x = 0; x < b.len[0]; x++)
                        host[b.stride[0] * x + b.stride[1] * y] =
                            f[(int64_t)gidx(sp0, b.irrep[0], x) * n + gidx(sp1, b.irrep[1], y)];
                ctx.stage_h2d(T.data + b.offset, host.data(), b.size * sizeof(double));
            }
    }

    void two_electron(int h) {
        Tensor& T = ctx.tensor(h);
        for (auto& sc : T.cases)
            for (auto& b : sc.blocks) {
                if (b.size == 0) continue;
                int space[4], irr[4], len[4];
                for (int p = 0; p < 4; p++) {
                    space[p] = group_space(T.group[p]);
                    irr[p] = b.irrep[p];
                    len[p] = b.len[p];
                }
                const std::vector<int>& s = sc.spin;
                bool J = s[0] == s[2] && s[1] == s[3];
                bool K = s[0] == s[3] && s[1] == s[2];
                if (b.pairs.empty()) {
                    if (J) coulomb(T.data, b.offset, space, irr, len, b.stride.data(), 0, 2, 1, 3, 1.0, 0);
                    if (K) coulomb(T.data, b.offset, space, irr, len, b.stride.data(), 0, 3, 1, 2, -1.0, 1);
                } else {
                    const bool was = batch;   // a packed block's pieces feed the pack kernel at once
                    batch = false;
                    packed_block(T, sc, b, space, irr, len, J, K);
                    batch = was;
                }
            }
        flush();
    }

    // every block of a plain (spatial) two-electron tensor as one Coulomb piece
    // (x_pa x_pb | x_pc x_pd): the non-antisymmetrised <pq|rs> of the RHF integrals
    void coulomb_plain(int h, int pa, int pb, int pc, int pd) {
        Tensor& T = ctx.tensor(h);
        for (auto& sc : T.cases)
            for (auto& b : sc.blocks) {
                if (b.size == 0) continue;
                int space[4], irr[4], len[4];
                for (int p = 0; p < 4; p++) {
                    space[p] = group_space(T.group[p]);
                    irr[p] = b.irrep[p];
                    len[p] = b.len[p];
                }
                coulomb(T.data, b.offset, space, irr, len, b.stride.data(), pa, pb, pc, pd, 1.0);
            }
        flush();
    }

    // packed V_abcd-type block: chunk over the first index, build (ac|bd) and (ad|bc)
    // unpacked for the chunk, then pack <ab||cd> for canonical pairs
    void packed_block(Tensor& T, const SpinCase& sc, const Block& b, const int* space, const int* irr,
                      const int* len, bool J, bool K) {
        (void)sc;
        if (b.pairs.size() != 2 || b.pairs[0].p != 0 || b.pairs[1].p != 2)
            throw Error(CCSD_ERR_UNSUPPORTED, "packed build supports <ab||cd> pair layouts only");
        const int64_t per_a = (int64_t)len[1] * len[2] * len[3];
        int64_t chunk = std::max<int64_t>(1, (int64_t)(256ll << 20) / std::max<int64_t>(per_a, 1));
        chunk = std::min<int64_t>(chunk, len[0]);
        double* tJ = (double*)ctx.dmalloc(std::max<int64_t>(chunk * per_a, 1) * sizeof(double));
        double* tK = (double*)ctx.dmalloc(std::max<int64_t>(chunk * per_a, 1) * sizeof(double));
        for (int a0 = 0; a0 < len[0]; a0 += (int)chunk) {
            int a1 = std::min<int>(len[0], a0 + (int)chunk);
            int ca = a1 - a0;
            CCSD_CUDA(cudaMemsetAsync(tJ, 0, (size_t)ca * per_a * sizeof(double), ctx.stream));
            CCSD_CUDA(cudaMemsetAsync(tK, 0, (size_t)ca * per_a * sizeof(double), ctx.stream));
            // tJ[a', c, b, d] = (a c | b d) ; tK[a', d, b, c] = (a d | b c)   (a' = a - a0)
            int lenc[4] = {ca, len[2], len[1], len[3]};
            int spc[4] = {space[0], space[2], space[1], space[3]};
            int irc[4] = {irr[0], irr[2], irr[1], irr[3]};
            int64_t st[4] = {1, ca, (int64_t)ca * len[2], (int64_t)ca * len[2] * len[1]};
            if (J) coulomb_shift(tJ, spc, irc, lenc, st, a0, 1.0);
            int lenk[4] = {ca, len[3], len[1], len[2]};
            int spk[4] = {space[0], space[3], space[1], space[2]};
            int irk[4] = {irr[0], irr[3], irr[1], irr[2]};
            int64_t sk[4] = {1, ca, (int64_t)ca * len[3], (int64_t)ca * len[3] * len[1]};
            if (K) coulomb_shift(tK, spk, irk, lenk, sk, a0, 1.0);
            kern::pack_vvvv(T.data + b.offset, b.pairs[0].kind, b.pairs[1].kind, len[0], len[1], len[2], len[3],
                            b.pairs[1].stride, tJ, tK, a0, a1, J, K, ctx.stream);
        }
        ctx.dfree(tJ, chunk * per_a * sizeof(double));   // stream-ordered
        ctx.dfree(tK, chunk * per_a * sizeof(double));
    }

    // like coulomb() over positions (0,1 | 2,3) of a temporary whose position 0 starts at a0
    void coulomb_shift(double* C, const int* space, const int* irrep, const int* len, const int64_t* stride, int a0,
                       double sign) {
        if (dEri) {
            gather(C, 0, space, irrep, len, stride, 0, 1, 2, 3, sign, a0);
            return;
        }
        int64_t M = (int64_t)len[0] * len[1], N = (int64_t)len[2] * len[3];
        if (M == 0 || N == 0) return;
        std::vector<int64_t> k = aux_list(irrep[0] ^ irrep[1]);
        if (k.empty()) return;
        std::vector<int64_t> Am(M), Bn(N), Cm(M), Cn(N);
        for (int y = 0; y < len[1]; y++)
            for (int x = 0; x < len[0]; x++) {
                int64_t m = x + (int64_t)len[0] * y;
                Am[m] = (int64_t)gidx(space[0], irrep[0], a0 + x) * n + gidx(space[1], irrep[1], y);
                Cm[m] = stride[0] * x + stride[1] * y;
            }
        for (int y = 0; y < len[3]; y++)
            for (int x = 0; x < len[2]; x++) {
                int64_t m = x + (int64_t)len[2] * y;
                Bn[m] = (int64_t)gidx(space[2], irrep[2], x) * n + gidx(space[3], irrep[3], y);
                Cn[m] = stride[2] * x + stride[3] * y;
            }
        Tables tb{ctx, {}};
        int64_t *dAm = tb.up(Am), *dK = tb.up(k), *dBn = tb.up(Bn), *dCm = tb.up(Cm), *dCn = tb.up(Cn);
        kern::GemmArgs a;
        a.A = dB;
        a.B = dB;
        a.C = C;
        a.M = (int)M;
        a.N = (int)N;
        a.K = (int)k.size();
        a.alpha = sign;
        a.Am = dAm;
        a.Ak = dK;
        a.Bk = dK;
        a.Bn = dBn;
        a.Cm[0] = dCm;
        a.Cn[0] = dCn;
        kern::gemm_fp64(a, ctx.stream);
    }
};

int mk(Context& c, const char* name, int o0, int o1, int i0, int i1, int flags = 0) {
    int nout[2] = {o0, o1}, nin[2] = {i0, i1};
    return c.create_tensor(name, nout, nin, flags);
}

}  // namespace

void create_hamiltonian_tensors(Context& ctx, bool pack_vvvv, ccsd_hamiltonian* H) {
    H->fAI = mk(ctx, "f(ai)", 1, 0, 0, 1);
    H->fME = mk(ctx, "f(ia)", 0, 1, 1, 0);
    H->fAE = mk(ctx, "f(ab)", 1, 0, 1, 0);
    H->fMI = mk(ctx, "f(ij)", 0, 1, 0, 1);
    H->VMNIJ = mk(ctx, "<ij||kl>", 0, 2, 0, 2);
    H->VAMIJ = mk(ctx, "<ai||jk>", 1, 1, 0, 2);
    H->VMNEF = mk(ctx, "<ij||ab>", 0, 2, 2, 0);
    H->VAMEI = mk(ctx, "<ai||bj>", 1, 1, 1, 1);
    H->VAMEF = mk(ctx, "<ai||bc>", 1, 1, 2, 0);
    H->VABEF = mk(ctx, "<ab||cd>", 2, 0, 2, 0, pack_vvvv ? CCSD_TENSOR_PACKED : 0);
    // blocks equal by Hermiticity (aomoints.cxx:1375-1387) are views with permuted
    // strides instead of copies: <ij||ak> = <ak||ij>, <ab||ij> = <ij||ab>, <ab||ci> = <ci||ab>
    const int perm[4] = {2, 3, 0, 1};
    {
        int no[2] = {0, 2}, ni[2] = {1, 1};
        H->VMNEJ = ctx.create_view("<ij||ak>", H->VAMIJ, no, ni, perm);
    }
    {
        int no[2] = {2, 0}, ni[2] = {0, 2};
        H->VABIJ = ctx.create_view("<ab||ij>", H->VMNEF, no, ni, perm);
    }
    {
        int no[2] = {2, 0}, ni[2] = {1, 1};
        H->VABEJ = ctx.create_view("<ab||ci>", H->VAMEF, no, ni, perm);
    }
}

void create_rhf_hamiltonian_tensors(Context& ctx, ccsd_rhf_hamiltonian* H) {
    const int P = CCSD_TENSOR_PLAIN;
    H->fAI = mk(ctx, "fAI", 1, 0, 0, 1, P);
    H->fAB = mk(ctx, "fAB", 1, 0, 1, 0, P);
    H->fIJ = mk(ctx, "fIJ", 0, 1, 0, 1, P);
    H->VABCD = mk(ctx, "<Ab|Cd>", 2, 0, 2, 0, P);
    H->VABCI = mk(ctx, "<Ab|Ci>", 2, 0, 1, 1, P);
    H->VABIJ = mk(ctx, "<Ab|Ij>", 2, 0, 0, 2, P);
    H->VAIBJ = mk(ctx, "<Ai|Bj>", 1, 1, 1, 1, P);
    H->VAIJB = mk(ctx, "<Ai|Jb>", 1, 1, 1, 1, P);
    H->VAIJK = mk(ctx, "<Ai|Jk>", 1, 1, 0, 2, P);
    H->VIJKL = mk(ctx, "<Ij|Kl>", 0, 2, 0, 2, P);
}

namespace {

// <pq|rs> = (pr|qs): positions (0,2 | 1,3) of every block, except VAIJB whose element
// <ai|jb> = (aj|ib) is stored at [a, i, b, j] (positions 0,3 | 1,2); the block list of
// the reference's RHF integrals (rhfaomoints.cxx:59-66)
void fill_rhf_two_electron(Builder& bld, const ccsd_rhf_hamiltonian* H) {
    for (int h : {H->VABCD, H->VABCI, H->VABIJ, H->VAIBJ, H->VAIJK, H->VIJKL}) bld.coulomb_plain(h, 0, 2, 1, 3);
    bld.coulomb_plain(H->VAIJB, 0, 3, 1, 2);
}

void require_closed_shell(const Spaces& S, const char* who) {
    for (int h = 0; h < S.nirrep; h++)
        for (int sp = 0; sp < 2; sp++)
            if (S.n[sp][ALPHA][h] != S.n[sp][BETA][h])
                throw Error(CCSD_ERR_ARG, std::string(who) + " needs a closed-shell (alpha = beta) space");
}

}  // namespace

void build_rhf_hamiltonian(Context& ctx, int naux, const double* B, const double* eps, const int* aux_per_irrep,
                           ccsd_rhf_hamiltonian* H) {
    const Spaces& S = ctx.spaces;
    require_closed_shell(S, "the RHF builder");
    Builder bld{ctx, S.total(VRT, ALPHA) + S.total(OCC, ALPHA), naux, S.total(OCC, ALPHA)};
    if (aux_per_irrep) {
        bld.aux_known = true;
        for (int h = 0; h < S.nirrep; h++)
            for (int k = 0; k < aux_per_irrep[h]; k++) bld.aux_irrep.push_back(h);
        if ((int)bld.aux_irrep.size() != naux) throw Error(CCSD_ERR_ARG, "aux_per_irrep does not sum to naux");
    }
    const int64_t nB = (int64_t)naux * bld.n * bld.n;
    bld.dB = (double*)ctx.dmalloc(nB * sizeof(double));
    CCSD_CUDA(cudaMemcpyAsync(bld.dB, B, nB * sizeof(double), cudaMemcpyHostToDevice, ctx.stream));
    create_rhf_hamiltonian_tensors(ctx, H);
    bld.batch = S.nirrep > 1;
    bld.one_electron(H->fAB, eps);
    bld.one_electron(H->fIJ, eps);
    fill_rhf_two_electron(bld, H);
    CCSD_CUDA(cudaStreamSynchronize(ctx.stream));
    ctx.dfree(bld.dB, nB * sizeof(double));
}

void build_rhf_hamiltonian_device(Context& ctx, int n, const double* fock, const double* d_eri,
                                  ccsd_rhf_hamiltonian* H) {
    const Spaces& S = ctx.spaces;
    require_closed_shell(S, "the RHF builder");
    if (n != S.total(VRT, ALPHA) + S.total(OCC, ALPHA))
        throw Error(CCSD_ERR_ARG, "orbital count differs from the context's spaces");
    Builder bld{ctx, n, 0, S.total(OCC, ALPHA)};
    bld.dEri = d_eri;
    create_rhf_hamiltonian_tensors(ctx, H);
    for (int h : {H->fAI, H->fAB, H->fIJ}) bld.one_electron_full(h, fock);
    fill_rhf_two_electron(bld, H);
    CCSD_CUDA(cudaStreamSynchronize(ctx.stream));
}

namespace {
// a dense (pq|rs) copied to the device for the lifetime of a build
struct DeviceEri {
    Context& c;
    double* p = nullptr;
    int64_t bytes = 0;
    DeviceEri(Context& ctx, int n, const double* eri) : c(ctx) {
        const int64_t ne = (int64_t)n * n * n * n;
        bytes = ne * (int64_t)sizeof(double);
        p = (double*)c.dmalloc(bytes);
        CCSD_CUDA(cudaMemcpyAsync(p, eri, bytes, cudaMemcpyHostToDevice, c.stream));
    }
    ~DeviceEri() {
        cudaStreamSynchronize(c.stream);
        c.dfree(p, bytes);
    }
};
}  // namespace

void build_rhf_hamiltonian_dense(Context& ctx, int n, const double* fock, const double* eri, ccsd_rhf_hamiltonian* H) {
    if (n != ctx.spaces.total(VRT, ALPHA) + ctx.spaces.total(OCC, ALPHA))
        throw Error(CCSD_ERR_ARG, "orbital count differs from the context's spaces");
    DeviceEri d(ctx, n, eri);
    build_rhf_hamiltonian_device(ctx, n, fock, d.p, H);
}

void build_hamiltonian(Context& ctx, int naux, const double* B, const double* eps, const int* aux_per_irrep,
                       bool pack_vvvv, ccsd_hamiltonian* H) {
    const Spaces& S = ctx.spaces;
    for (int h = 0; h < S.nirrep; h++)
        for (int sp = 0; sp < 2; sp++)
            if (S.n[sp][ALPHA][h] != S.n[sp][BETA][h])
                throw Error(CCSD_ERR_ARG, "the factor builder needs a closed-shell (alpha = beta) space");
    Builder bld{ctx, S.total(VRT, ALPHA) + S.total(OCC, ALPHA), naux, S.total(OCC, ALPHA)};
    if (aux_per_irrep) {
        bld.aux_known = true;
        for (int h = 0; h < S.nirrep; h++)
            for (int k = 0; k < aux_per_irrep[h]; k++) bld.aux_irrep.push_back(h);
        if ((int)bld.aux_irrep.size() != naux) throw Error(CCSD_ERR_ARG, "aux_per_irrep does not sum to naux");
    }
    const int64_t nB = (int64_t)naux * bld.n * bld.n;
    bld.dB = (double*)ctx.dmalloc(nB * sizeof(double));
    CCSD_CUDA(cudaMemcpyAsync(bld.dB, B, nB * sizeof(double), cudaMemcpyHostToDevice, ctx.stream));

    create_hamiltonian_tensors(ctx, pack_vvvv, H);
    bld.batch = S.nirrep > 1;

    bld.one_electron(H->fAE, eps);
    bld.one_electron(H->fMI, eps);
    for (int h : {H->VMNIJ, H->VAMIJ, H->VMNEF, H->VAMEI, H->VAMEF, H->VABEF}) bld.two_electron(h);
    CCSD_CUDA(cudaStreamSynchronize(ctx.stream));
    ctx.dfree(bld.dB, nB * sizeof(double));
}

void build_hamiltonian_device(Context& ctx, int n, const double* fock, const double* d_eri, bool pack_vvvv,
                              ccsd_hamiltonian* H) {
    const Spaces& S = ctx.spaces;
    for (int h = 0; h < S.nirrep; h++)
        for (int sp = 0; sp < 2; sp++)
            if (S.n[sp][ALPHA][h] != S.n[sp][BETA][h])
                throw Error(CCSD_ERR_ARG, "the dense-integral builder needs a closed-shell (alpha = beta) space");
    if (n != S.total(VRT, ALPHA) + S.total(OCC, ALPHA))
        throw Error(CCSD_ERR_ARG, "orbital count differs from the context's spaces");
    Builder bld{ctx, n, 0, S.total(OCC, ALPHA)};
    bld.dEri = d_eri;
    create_hamiltonian_tensors(ctx, pack_vvvv, H);
    for (int h : {H->fAI, H->fME, H->fAE, H->fMI}) bld.one_electron_full(h, fock);
    for (int h : {H->VMNIJ, H->VAMIJ, H->VMNEF, H->VAMEI, H->VAMEF, H->VABEF}) bld.two_electron(h);
    CCSD_CUDA(cudaStreamSynchronize(ctx.stream));
}

void build_hamiltonian_dense(Context& ctx, int n, const double* fock, const double* eri, bool pack_vvvv,
                             ccsd_hamiltonian* H) {
    if (n != ctx.spaces.total(VRT, ALPHA) + ctx.spaces.total(OCC, ALPHA))
        throw Error(CCSD_ERR_ARG, "orbital count differs from the context's spaces");
    DeviceEri d(ctx, n, eri);
    build_hamiltonian_device(ctx, n, fock, d.p, pack_vvvv, H);
}

}  // namespace ccsd
