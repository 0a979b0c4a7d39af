"""Row slabs of one CCSD iteration: the bounded CPU sample of the benchmark workload.

TEST INFRASTRUCTURE ONLY (the checker side; see ccsd_oracle.py).  Only the CPU tests and
the CPU legs of bench.py use it; it loads nothing of the engine's library.

Why a sample.  ccsd_oracle.CCSD (the numpy restatement of src/cc/ccsd.cxx:123-192 over
full spin-orbital arrays) needs, at o=32 v=256, the full <am||ef> and <ab||ej> arrays
(69 GB each) and (pq|rs) (55 GB): more than a 196 GB host holds, and about 20 minutes of
16 cores per iteration.  The CPU baseline therefore times the same statements at the same
sizes on a slab of rows of every output:

* outputs whose first index is virtual (FAE, WAMIJ, WAMEI, Z1, Z2) for a in Sv, a few
  spin-orbital virtuals;
* outputs whose first index is occupied (FME, FMI, WMNIJ, WMNEJ) for m in So;
* the elementwise tail (Tau, the Jacobi weight and update, energy, convergence, the DIIS
  dots and linear combination) on the same rows of Z1, Z2.

Every statement is a sum of contractions over its other indices, so producing a fraction
f of its rows costs f of its full work: the full iteration is estimated as sum over the
statements of t_slab / f.  A term under P(ab) needs X[Sv, :] and X[:, Sv] of its product X
(2 f of the work of X); its f is counted that way.  Operands that a statement reads whole
are laid out once, before timing, so that each slab contraction is one GEMM on
contiguous memory and the timed work is the contraction itself (the full oracle
transposes some operands on every call: the sample leaves that cost out, in the CPU's
favour).

tests/test_ccsd_slab.py checks on small problems that every slab equals the rows of the
oracle's own statement, and that the slabs over all rows reproduce ccsd_oracle's residual.
"""
from __future__ import annotations

import time

import numpy as np

from .ccsd_oracle import es, weight


def eri_sub(B, p, q, r, s):
    """(pq|rs) for index lists: sum_P B[P,p,q] B[P,r,s] -> [p, q, r, s]."""
    naux = B.shape[0]
    X = B[:, p][:, :, q].reshape(naux, -1)
    Y = B[:, r][:, :, s].reshape(naux, -1)
    return (X.T @ Y).reshape(len(p), len(q), len(r), len(s))


def so_block(B, idx, rows=None):
    """Spin-orbital <pq||rs> for spatial index lists idx = (p, q, r, s), as ccsd_oracle's
    _so_block; `rows`: spin-orbital indices of the first position to keep (all if None)."""
    p, q, r, s = (np.asarray(x) for x in idx)
    np_full = len(p)
    if rows is not None:
        rows = np.asarray(rows)
        sp_rows = np.unique(rows % np_full)
        p = p[sp_rows]
    J = eri_sub(B, p, r, q, s).transpose(0, 2, 1, 3)   # (pr|qs) as [p,q,r,s]
    K = eri_sub(B, p, s, q, r).transpose(0, 2, 3, 1)   # (ps|qr) as [p,q,r,s]
    n0, n1, n2, n3 = len(p), len(q), len(r), len(s)
    out = np.zeros((2 * n0, 2 * n1, 2 * n2, 2 * n3))
    for sp in (0, 1):
        for sq in (0, 1):
            for sr in (0, 1):
                for ss in (0, 1):
                    val = None
                    if sp == sr and sq == ss:
                        val = J.copy()
                    if sp == ss and sq == sr:
                        val = -K if val is None else val - K
                    if val is not None:
                        out[sp * n0:(sp + 1) * n0, sq * n1:(sq + 1) * n1,
                            sr * n2:(sr + 1) * n2, ss * n3:(ss + 1) * n3] = val
    if rows is None:
        return out
    # spin-orbital row x = spin * np_full + spatial  ->  row of `out`
    pos = {a: k for k, a in enumerate(sp_rows)}
    sel = [(x // np_full) * n0 + pos[x % np_full] for x in rows]
    return out[sel]


class SlabIteration:
    """The statements of ccsd_oracle.CCSD.residual and iterate on row slabs.

    B, eps: the synthetic factor and orbital energies (closed shell, occupied first);
    o: spatial occupied count; sv, so: spin-orbital row subsets (virtual, occupied).
    """

    def __init__(self, B, eps, o, sv, so, diis_order=8):
        n = len(eps)
        v = n - o
        self.o, self.v, self.n = o, v, n
        self.sv = np.asarray(sorted(sv))
        self.so = np.asarray(sorted(so))
        self.fv = len(self.sv) / (2 * v)
        self.fo = len(self.so) / (2 * o)
        self.order = diis_order
        O, V = np.arange(o), np.arange(o, n)
        sv_, so_ = self.sv, self.so
        f = np.diag(eps)

        def f_so(rows, cols):
            fr = f[np.ix_(rows, cols)]
            out = np.zeros((2 * len(rows), 2 * len(cols)))
            out[:len(rows), :len(cols)] = fr
            out[len(rows):, len(cols):] = fr
            return out
        self.fAI, self.fME, self.fAE, self.fMI = f_so(V, O), f_so(O, V), f_so(V, V), f_so(O, O)
        self.dv = -np.concatenate([eps[o:], eps[o:]])
        self.do = np.concatenate([eps[:o], eps[:o]])
        # blocks read whole
        VMNEF = so_block(B, (O, O, V, V))
        self.VMNEF_S = np.ascontiguousarray(VMNEF[so_])
        self.VMNEJ = so_block(B, (O, O, V, O))
        self.VMNIJ_S = so_block(B, (O, O, O, O), rows=so_)
        self.VAMIJ_S = so_block(B, (V, O, O, O), rows=sv_)
        # row slabs of the large blocks
        self.VAMEF_S = so_block(B, (V, O, V, V), rows=sv_)
        self.VAMEI_S = so_block(B, (V, O, V, O), rows=sv_)
        self.VABEJ_S = so_block(B, (V, V, V, O), rows=sv_)
        self.VABIJ_S = so_block(B, (V, V, O, O), rows=sv_)
        # ladder: (ae|bf) for the spatial rows a of Sv, as [a, b, e, f]
        self.sp_rows = np.unique(sv_ % v)
        self.vvvv_rows = np.ascontiguousarray(eri_sub(B, V[self.sp_rows], V, V, V).transpose(0, 2, 1, 3))
        # whole-read operands laid out for one GEMM per slab contraction
        oo, vv = 2 * o, 2 * v
        self.VMNEF_e_mnf = np.ascontiguousarray(VMNEF.transpose(2, 0, 1, 3)).reshape(vv, -1)
        self.VMNEF_me_nf = np.ascontiguousarray(VMNEF.transpose(0, 2, 1, 3)).reshape(oo * vv, oo * vv)
        del VMNEF

    # -- operands that change every iteration, laid out once per sample -------------------
    def prepare(self, T1, T2, Tau, I):
        """Full-size inputs of the slab statements: the amplitudes, Tau and the whole-read
        intermediates I (FME, FMI, FAE, WMNIJ, WMNEJ, WAMIJ, WAMEI)."""
        o2, v2, v = 2 * self.o, 2 * self.v, self.v
        self.T1, self.T2, self.Tau, self.I = T1, T2, Tau, I
        self.T2_nef_i = np.ascontiguousarray(T2.transpose(3, 0, 1, 2)).reshape(o2 * v2 * v2, o2)
        self.T2_me_bj = self.T2_nef_i.reshape(o2 * v2, v2 * o2)       # the same [n, e, f, i] array
        self.Tau_mef_i = np.ascontiguousarray(Tau.transpose(3, 0, 1, 2)).reshape(o2 * v2 * v2, o2)
        self.Tau_spins = np.ascontiguousarray(
            Tau.reshape(2, v, 2, v, o2 * o2).transpose(0, 2, 1, 3, 4)).reshape(2, 2, v * v, o2 * o2)
        W = I["WAMEI"]
        self.WAMEI_bi_me = np.ascontiguousarray(W.transpose(0, 3, 1, 2)).reshape(v2 * o2, o2 * v2)
        self.WAMIJ_m_bij = np.ascontiguousarray(I["WAMIJ"].transpose(1, 0, 2, 3)).reshape(o2, -1)

    # -- the statements ----------------------------------------------------------------
    def _ladder(self):
        """Z2[a in Sv, b, i, j] += sum_ef (ae|bf) d(sa,se) d(sb,sf) Tau[e,f,i,j]."""
        v, o2 = self.v, 2 * self.o
        out = np.empty((len(self.sv), 2, v, o2 * o2))
        pos = {a: k for k, a in enumerate(self.sp_rows)}
        for k, a in enumerate(self.sv):
            sa, r = a // v, pos[a % v]
            G = self.vvvv_rows[r].reshape(v, v * v)            # [b, (e, f)]
            for sb in (0, 1):
                out[k, sb] = G @ self.Tau_spins[sa, sb]
        return out.reshape(len(self.sv), 2 * v, o2, o2)

    def statements(self):
        """(name, fraction of the statement's full work, callable) in ccsd.cxx order.
        Each callable stores its slab in self.out."""
        sv, so = self.sv, self.so
        T1, T2, Tau, I = self.T1, self.T2, self.Tau, self.I
        o2, v2 = 2 * self.o, 2 * self.v
        out = self.out = {}
        fv, fo = self.fv, self.fo

        def fme():
            out["FME"] = self.fME[so] + es('mnef,fn->me', self.VMNEF_S, T1)

        def fmi():
            x = self.fMI[so].copy()
            x += 0.5 * (self.VMNEF_S.reshape(len(so), -1) @ self.T2_nef_i)
            x += es('me,ei->mi', I["FME"][so], T1)
            x += es('nmfi,fn->mi', self.VMNEJ[:, so], T1)
            out["FMI"] = x

        def fae():
            x = self.fAE[sv].copy()
            T2S = np.ascontiguousarray(T2[sv].transpose(0, 2, 3, 1)).reshape(len(sv), -1)   # [a, (m n f)]
            x -= 0.5 * (T2S @ self.VMNEF_e_mnf.T)
            x -= es('me,am->ae', I["FME"], T1[sv])
            x += es('amef,fm->ae', self.VAMEF_S, T1)
            out["FAE"] = x

        def wmnij():
            x = self.VMNIJ_S.copy()
            x += 0.5 * es('mnef,efij->mnij', self.VMNEF_S, Tau)
            y = es('mnej,ei->mnij', self.VMNEJ[so], T1)
            x += y - y.transpose(0, 1, 3, 2)
            out["WMNIJ"] = x

        def wmnej():
            out["WMNEJ"] = self.VMNEJ[so] + es('mnef,fj->mnej', self.VMNEF_S, T1)

        def wamij():
            x = self.VAMIJ_S.copy()
            x += 0.5 * es('amef,efij->amij', self.VAMEF_S, Tau)
            y = es('amej,ei->amij', self.VAMEI_S, T1)
            x += y - y.transpose(0, 1, 3, 2)
            out["WAMIJ"] = x

        def wamei():
            x = self.VAMEI_S.copy()
            T2S = np.ascontiguousarray(T2[sv].transpose(2, 1, 0, 3)).reshape(o2 * v2, -1)   # [(n f), (a i)]
            y = (self.VMNEF_me_nf @ T2S).reshape(o2, v2, len(sv), o2)                        # [m, e, a, i]
            x += 0.5 * y.transpose(2, 0, 1, 3)
            x += es('amef,fi->amei', self.VAMEF_S, T1)
            x -= es('nmei,an->amei', I["WMNEJ"], T1[sv])
            out["WAMEI"] = x

        def z1():
            x = self.fAI[sv].copy()
            x += es('ae,ei->ai', self.fAE[sv], T1)
            x -= es('mi,am->ai', I["FMI"], T1[sv])
            x -= es('amei,em->ai', self.VAMEI_S, T1)
            x += es('me,aeim->ai', I["FME"], T2[sv])
            x += 0.5 * (self.VAMEF_S.reshape(len(sv), -1) @ self.Tau_mef_i)
            x -= 0.5 * es('mnei,eamn->ai', I["WMNEJ"], T2[:, sv])
            out["Z1"] = x

        def z2_local():
            x = self.VABIJ_S.copy()
            y = es('abej,ei->abij', self.VABEJ_S, T1)
            x += y - y.transpose(0, 1, 3, 2)
            y = es('mi,abmj->abij', I["FMI"], T2[sv])
            x -= y - y.transpose(0, 1, 3, 2)
            x += 0.5 * es('mnij,abmn->abij', I["WMNIJ"], Tau[sv])
            out["Z2"] = x

        def z2_wamij():
            # -P(ab) W(am,ij) t(b,m): rows a in Sv need X[Sv, :] and X[:, Sv]
            xa = es('amij,bm->abij', I["WAMIJ"][sv], T1)
            xb = (T1[sv] @ self.WAMIJ_m_bij).reshape(len(sv), v2, o2, o2)                   # X[b, a] as [a, b]
            out["Z2"] -= xa - xb

        def z2_fae():
            xa = es('ae,ebij->abij', I["FAE"][sv], T2)
            xb = es('be,eaij->abij', I["FAE"], T2[:, sv])                                      # X[b, a] as [a, b]
            out["Z2"] += xa - xb

        def z2_ladder():
            out["Z2"] += self._ladder()

        def z2_ring():
            # P(ab) P(ij) sum_em W[a,m,e,i] T2[e,b,j,m]
            WS = np.ascontiguousarray(I["WAMEI"][sv].transpose(0, 3, 1, 2)).reshape(len(sv) * o2, o2 * v2)
            xa = (WS @ self.T2_me_bj).reshape(len(sv), o2, v2, o2).transpose(0, 2, 1, 3)     # [a, b, i, j]
            T2S = np.ascontiguousarray(T2[:, sv].transpose(3, 0, 1, 2)).reshape(o2 * v2, -1)  # [(m e), (a j)]
            xb = (self.WAMEI_bi_me @ T2S).reshape(v2, o2, len(sv), o2).transpose(2, 0, 1, 3)  # X[b,a,i,j] as [a,b,i,j]
            x = xa - xb
            out["Z2"] += x - x.transpose(0, 1, 3, 2)

        return [("FME", fo, fme), ("FMI", fo, fmi), ("FAE", fv, fae), ("WMNIJ", fo, wmnij), ("WMNEJ", fo, wmnej),
                ("WAMIJ", fv, wamij), ("WAMEI", fv, wamei), ("Z1", fv, z1), ("Z2 local terms", fv, z2_local),
                ("Z2 P(ab) W(am,ij) T1", 2 * fv, z2_wamij), ("Z2 P(ab) F(ae) T2", 2 * fv, z2_fae),
                ("Z2 particle ladder", fv, z2_ladder), ("Z2 ring", 2 * fv, z2_ring)]

    def tail(self, ring):
        """ccsd.cxx:182-192 on the rows a in Sv: weight, T += Z, Tau, energy, max-norm, DIIS
        (inner products with the stored rows of `ring` and the linear combination)."""
        sv = self.sv
        D1 = self.dv[sv][:, None] + self.do[None, :]
        D2 = (self.dv[sv][:, None, None, None] + self.dv[None, :, None, None]
              + self.do[None, None, :, None] + self.do[None, None, None, :])
        Z1 = weight(self.out["Z1"], D1)
        Z2 = weight(self.out["Z2"], D2)
        T1 = self.T1[sv] + Z1
        T2 = self.T2[sv] + Z2
        tau = T2 + np.einsum('ai,bj->abij', T1, self.T1) - np.einsum('aj,bi->abij', T1, self.T1)
        e = float(np.vdot(self.fAI[sv], T1) + 0.25 * np.vdot(self.VABIJ_S, tau))
        conv = float(max(np.abs(Z1).max(initial=0.0), np.abs(Z2).max(initial=0.0)))
        # DIIS: store (x, dx), inner products with the ring, x <- sum c_i x_i, dx <- sum c_i dx_i
        stored = (T1.copy(), T2.copy(), Z1.copy(), Z2.copy())
        dots = [float(np.vdot(Z1, d1) + 0.25 * np.vdot(Z2, d2)) for _, _, d1, d2 in ring]
        c = np.full(len(ring), 1.0 / max(len(ring), 1))
        acc = [np.zeros_like(a) for a in stored]
        for ci, entry in zip(c, ring):
            for a, x in zip(acc, entry):
                a += ci * x
        return e, conv, dots

    def run(self, ring=None):
        """One sampled iteration: {statement: (seconds, fraction)} and the estimated seconds
        of the full iteration (sum of seconds / fraction)."""
        times = {}
        for name, frac, fn in self.statements():
            t0 = time.perf_counter()
            fn()
            times[name] = (time.perf_counter() - t0, frac)
        if ring is not None:
            t0 = time.perf_counter()
            self.tail(ring)
            times["update, energy, DIIS"] = (time.perf_counter() - t0, self.fv)
        est = sum(t / f for t, f in times.values())
        return times, est


def timing_inputs(s: SlabIteration, seed=0, diis_order=8):
    """Seeded full-size amplitudes and intermediates of the right shapes for timing (the
    values of the workload's own iterations do not change the cost of these dense
    contractions), and a DIIS ring of `diis_order` stored rows of the slab."""
    rng = np.random.default_rng(seed)
    o2, v2 = 2 * s.o, 2 * s.v
    T1 = 1e-3 * rng.standard_normal((v2, o2))
    T2 = 1e-3 * rng.standard_normal((v2, v2, o2, o2))
    Tau = T2 + np.einsum('ai,bj->abij', T1, T1)
    I = dict(FME=1e-3 * rng.standard_normal((o2, v2)), FMI=1e-3 * rng.standard_normal((o2, o2)),
             FAE=1e-3 * rng.standard_normal((v2, v2)), WMNIJ=1e-3 * rng.standard_normal((o2, o2, o2, o2)),
             WMNEJ=1e-3 * rng.standard_normal((o2, o2, v2, o2)), WAMIJ=1e-3 * rng.standard_normal((v2, o2, o2, o2)),
             WAMEI=1e-3 * rng.standard_normal((v2, o2, v2, o2)))
    s.prepare(T1, T2, Tau, I)
    k = len(s.sv)
    ring = [(1e-3 * rng.standard_normal((k, o2)), 1e-3 * rng.standard_normal((k, v2, o2, o2)),
             1e-3 * rng.standard_normal((k, o2)), 1e-3 * rng.standard_normal((k, v2, o2, o2)))
            for _ in range(diis_order)]
    return ring
