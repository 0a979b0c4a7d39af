"""CPU FP64 oracle for the CCSD amplitude iteration.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only the tests, the
smoke entry point and the CPU-baseline leg of bench.py may import it.  The
product path (aquarius_b200) never calls it.

It restates, in plain numpy over FULL spin-orbital arrays (every index runs
over alpha and beta spin-orbitals; blocks forbidden by spin are stored as
zeros), the reference's algorithm:

* one iteration, statement for statement:          src/cc/ccsd.cxx:123-192
* initial guess and MP2 energy:                    src/cc/ccsd.cxx:50-62
* implicit antisymmetrisation P(A-lines|B-lines)
  of external lines split across the two factors,
  per orbital space, separately for upper/lower:   src/tensor/spinorbital_tensor.cxx:637-669
* Jacobi weight with the |den| < 1e-4 -> 0 rule:   src/tensor/ctf_tensor.cxx:480-514
* denominators  d_a = -f_aa, d_i = +f_ii:           src/operator/denominator.hpp:50-73
* DIIS ring, bordered system, dsysv + eps retry:   src/convergence/diis.hpp:70-227
  (inner product weights 1, 1, 1/4 for T0,T1,T2: src/operator/excitationoperator.hpp:77-87)
* convergence = max-abs of the weighted update:    src/operator/excitationoperator.hpp:92-102,
                                                   src/util/iterative.hpp:126-188
* integral blocks <pq||rs> with [out..., in...]
  index order (13 blocks of H):                     src/operator/2eoperator.cxx:10-21,
                                                   src/operator/aomoints.cxx:1357-1387

Spin-orbital index convention used here: occupied p in [0,2o): spatial p % o,
spin p // o (0 = alpha); virtual likewise with v.

The particle ladder 1/2 sum_ef <ab||ef> tau_efij is evaluated through the
identity  1/2 sum_ef <ab||ef> tau_efij = sum_ef (ae|bf) d(sa,se) d(sb,sf) tau_efij
(tau is antisymmetric in ef), which avoids materialising the (2v)^4 array;
`ladder_literal=True` uses the literal <ab||ef> array instead (tiny sizes).

The DIIS linear system is solved with LAPACK dsysv (Bunch-Kaufman), the same
routine the reference reaches through lawrap's hesv for real data.
"""
from __future__ import annotations

import numpy as np
from scipy.linalg import lapack

# ----------------------------------------------------------------------------
# integrals
# ----------------------------------------------------------------------------


def eri_from_factor(B: np.ndarray) -> np.ndarray:
    """(pq|rs) = sum_P B[P,p,q] B[P,r,s]  (spatial, chemist's notation)."""
    naux, n, _ = B.shape
    Bm = B.reshape(naux, n * n)
    return (Bm.T @ Bm).reshape(n, n, n, n)


def _so_block(eri, idx, nspat):
    """Full spin-orbital <pq||rs> block for spatial index lists idx=(p,q,r,s).

    <pq||rs> = (pr|qs) d(sp,sr) d(sq,ss) - (ps|qr) d(sp,ss) d(sq,sr)
    """
    p, q, r, s = idx
    J = eri[np.ix_(p, r, q, s)].transpose(0, 2, 1, 3)   # (pr|qs) as [p,q,r,s]
    K = eri[np.ix_(p, s, q, r)].transpose(0, 2, 3, 1)   # (ps|qr) as [p,q,r,s]
    n0, n1, n2, n3 = nspat
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
    return out


class Hamiltonian:
    """Spin-orbital blocks of H for a closed-shell reference (f diagonal or not).

    fock: (n,n) spatial Fock matrix in the MO basis (occupied first).
    eri:  (n,n,n,n) spatial (pq|rs).
    """

    def __init__(self, fock: np.ndarray, eri: np.ndarray, o: int, ladder_literal: bool = False):
        n = fock.shape[0]
        v = n - o
        self.o, self.v, self.n = o, v, n
        O = np.arange(o)
        V = np.arange(o, n)

        def f_so(rows, cols):
            fr = fock[np.ix_(rows, cols)]
            nr, nc = len(rows), len(cols)
            out = np.zeros((2 * nr, 2 * nc))
            out[:nr, :nc] = fr
            out[nr:, nc:] = fr
            return out

        self.fAI = f_so(V, O)
        self.fME = f_so(O, V)
        self.fAE = f_so(V, V)
        self.fMI = f_so(O, O)
        self.VMNIJ = _so_block(eri, (O, O, O, O), (o, o, o, o))
        self.VAMIJ = _so_block(eri, (V, O, O, O), (v, o, o, o))
        self.VMNEJ = _so_block(eri, (O, O, V, O), (o, o, v, o))
        self.VABIJ = _so_block(eri, (V, V, O, O), (v, v, o, o))
        self.VMNEF = _so_block(eri, (O, O, V, V), (o, o, v, v))
        self.VAMEI = _so_block(eri, (V, O, V, O), (v, o, v, o))
        self.VAMEF = _so_block(eri, (V, O, V, V), (v, o, v, v))
        self.VABEJ = _so_block(eri, (V, V, V, O), (v, v, v, o))
        # spatial (ae|bf) for the ladder identity
        self.eri_vvvv = np.ascontiguousarray(eri[np.ix_(V, V, V, V)])
        self.VABEF = _so_block(eri, (V, V, V, V), (v, v, v, v)) if ladder_literal else None
        # denominators (reference: d_A = -f_AA, d_I = +f_II), per spin-orbital
        self.dv = -np.concatenate([np.diag(fock)[o:], np.diag(fock)[o:]])
        self.do = np.concatenate([np.diag(fock)[:o], np.diag(fock)[:o]])


# ----------------------------------------------------------------------------
# helpers
# ----------------------------------------------------------------------------

def P01(x):
    """P(ab) on the first two axes: X_ab.. - X_ba.."""
    return x - x.transpose(1, 0, 2, 3)


def P23(x):
    """P(ij) on the last two axes."""
    return x - x.transpose(0, 1, 3, 2)


def es(spec, *ops):
    """einsum of the statements.  A two-factor contraction without batch (Hadamard) indices
    goes through one tensordot (a BLAS GEMM after transposes); numpy's einsum path search
    left some of the iteration's terms (e.g. 'amef,efim->ai') off BLAS, 10x slower."""
    if len(ops) == 2:
        ins, out = spec.split('->')
        ia, ib = ins.split(',')
        con = [c for c in ia if c in ib and c not in out]
        plain = (len(set(ia)) == len(ia) and len(set(ib)) == len(ib)
                 and all((c in out) != (c in con) for c in ia + ib))
        if plain:
            fa = [c for c in ia if c not in con]
            fb = [c for c in ib if c not in con]
            r = np.tensordot(ops[0], ops[1], axes=([ia.index(c) for c in con], [ib.index(c) for c in con]))
            cur = fa + fb
            return r.transpose([cur.index(c) for c in out])
    return np.einsum(spec, *ops, optimize=True)


def weight(x, dens):
    """CTFTensor::weight: x /= sum of denominators, 0 where |den| < 1e-4."""
    den = dens
    out = np.where(np.abs(den) < 1e-4, 0.0, x / np.where(np.abs(den) < 1e-4, 1.0, den))
    return out


class Amplitudes:
    def __init__(self, T1, T2):
        self.T1 = T1
        self.T2 = T2

    def copy(self):
        return Amplitudes(self.T1.copy(), self.T2.copy())


def inner(x: Amplitudes, y: Amplitudes) -> float:
    """ExcitationOperator::dot: <T0,T0'> + <T1,T1'> + 1/4 <T2,T2'> over full ranges (T0 = 0)."""
    return float(np.vdot(x.T1, y.T1) + 0.25 * np.vdot(x.T2, y.T2))


class DIIS:
    """src/convergence/diis.hpp:36-228 for one x and one dx."""

    def __init__(self, order=5, start=1, damping=0.0):
        self.nextrap = order
        self.start = start
        self.damping = damping
        self.e = np.zeros((order + 1, order + 1))
        self.c = np.zeros(order + 1)
        self.old_x = [None] * order
        self.old_dx = [None] * order
        self.last_info = 0

    def extrapolate(self, x: Amplitudes, dx: Amplitudes):
        n = self.nextrap
        if n <= 1:
            return
        # rotate so that data of iteration n-k sits in slot k
        self.old_x = [self.old_x[-1]] + self.old_x[:-1]
        self.old_dx = [self.old_dx[-1]] + self.old_dx[:-1]
        self.e = np.roll(np.roll(self.e, 1, axis=0), 1, axis=1)
        self.c = np.roll(self.c, 1)
        self.old_x[0] = x.copy()
        self.old_dx[0] = dx.copy()
        self.e[0, 0] = inner(dx, dx)
        nreal = 1
        for i in range(1, n):
            if self.old_dx[i] is None:
                break
            self.e[i, 0] = inner(dx, self.old_dx[i])
            self.e[0, i] = self.e[i, 0]
            nreal += 1
        for i in range(nreal):
            self.e[i, nreal] = -1.0
            self.e[nreal, i] = -1.0
            self.c[i] = 0.0
        self.e[nreal, nreal] = 0.0
        self.c[nreal] = -1.0
        if nreal == 1:
            return
        self.start -= 1
        if self.start > 1:
            if self.damping > 0.0:
                for arr0, arr1 in ((self.old_x[0].T1, self.old_x[1].T1), (self.old_x[0].T2, self.old_x[1].T2)):
                    arr0 *= (self.damping - 1)
                    arr0 += self.damping * arr1
            return
        m = nreal + 1
        a = self.e[:m, :m].copy()
        b = self.c[:m].copy()
        _, _, sol, info = lapack.dsysv(a, b, lower=0)
        if info > 0:
            eps = self.e[nreal - 1, nreal - 1] * np.finfo(float).eps
            a = self.e[:m, :m].copy()
            a[np.arange(nreal), np.arange(nreal)] += eps
            _, _, sol, info = lapack.dsysv(a, b, lower=0)
        self.last_info = info
        if info != 0:
            raise RuntimeError("DIIS: Info in hesv: %d" % info)
        self.c[:m] = sol
        c = self.c
        dx.T1[...] = self.old_dx[0].T1 * c[0]
        dx.T2[...] = self.old_dx[0].T2 * c[0]
        x.T1[...] = self.old_x[0].T1 * c[0]
        x.T2[...] = self.old_x[0].T2 * c[0]
        for i in range(1, nreal):
            dx.T1 += self.old_dx[i].T1 * c[i]
            dx.T2 += self.old_dx[i].T2 * c[i]
            x.T1 += self.old_x[i].T1 * c[i]
            x.T2 += self.old_x[i].T2 * c[i]


# ----------------------------------------------------------------------------
# CCSD
# ----------------------------------------------------------------------------

class CCSD:
    def __init__(self, H: Hamiltonian, diis_order=5, diis_start=1, diis_damping=0.0):
        self.H = H
        v2, o2 = H.fAI.shape
        self.D1 = H.dv[:, None] + H.do[None, :]
        self.D2 = (H.dv[:, None, None, None] + H.dv[None, :, None, None]
                   + H.do[None, None, :, None] + H.do[None, None, None, :])
        # ccsd.cxx:50-62 -- T(1) = fAI, T(2) = VABIJ, weighted
        self.T = Amplitudes(weight(H.fAI.copy(), self.D1), weight(H.VABIJ.copy(), self.D2))
        self.Z = Amplitudes(np.zeros((v2, o2)), np.zeros((v2, v2, o2, o2)))
        self.Tau = self.make_tau(self.T)
        self.mp2 = float(np.vdot(H.fAI, self.T.T1) + 0.25 * np.vdot(H.VABIJ, self.Tau))
        self.diis = DIIS(diis_order, diis_start, diis_damping)
        self.energy = self.mp2
        self.conv = np.finfo(float).max
        self.iter = 0
        self.keep_intermediates = False   # residual() keeps its intermediates (CPU tests)
        self.intermediates = None

    @staticmethod
    def make_tau(T):
        # Tau = T2 + 1/2 P(ab) P(ij) t_ai t_bj
        tt = np.einsum('ai,bj->abij', T.T1, T.T1)
        return T.T2 + 0.5 * P23(P01(tt))

    def ladder(self, Tau):
        H = self.H
        if H.VABEF is not None:
            return 0.5 * es('abef,efij->abij', H.VABEF, Tau)
        v, o2 = H.v, 2 * H.o
        if getattr(H, "_vvvv_ab_ef", None) is None:
            # (ae|bf) as a [ab, ef] matrix, formed once: each spin case is then one GEMM
            H._vvvv_ab_ef = np.ascontiguousarray(H.eri_vvvv.transpose(0, 2, 1, 3)).reshape(v * v, v * v)
        tr = Tau.reshape(2, v, 2, v, o2 * o2)
        # the four (sa, sb) spin cases side by side: [ef, (sa, sb, ij)]
        rhs = np.ascontiguousarray(tr.transpose(1, 3, 0, 2, 4)).reshape(v * v, 4 * o2 * o2)
        out = (H._vvvv_ab_ef @ rhs).reshape(v, v, 2, 2, o2, o2)
        return np.ascontiguousarray(out.transpose(2, 0, 3, 1, 4, 5)).reshape(2 * v, 2 * v, o2, o2)

    def residual(self, T: Amplitudes):
        """ccsd.cxx:123-180: intermediates and the unweighted Z(1), Z(2)."""
        H = self.H
        T1, T2 = T.T1, T.T2
        Tau = self.make_tau(T)

        FME = H.fME + es('mnef,fn->me', H.VMNEF, T1)

        FMI = H.fMI.copy()
        FMI += 0.5 * es('mnef,efin->mi', H.VMNEF, T2)
        FMI += es('me,ei->mi', FME, T1)
        FMI += es('nmfi,fn->mi', H.VMNEJ, T1)

        FAE = H.fAE.copy()
        FAE -= 0.5 * es('mnef,afmn->ae', H.VMNEF, T2)
        FAE -= es('me,am->ae', FME, T1)
        FAE += es('amef,fm->ae', H.VAMEF, T1)

        WMNIJ = H.VMNIJ.copy()
        WMNIJ += 0.5 * es('mnef,efij->mnij', H.VMNEF, Tau)
        WMNIJ += P23(es('mnej,ei->mnij', H.VMNEJ, T1))

        WMNEJ = H.VMNEJ + es('mnef,fj->mnej', H.VMNEF, T1)

        WAMIJ = H.VAMIJ.copy()
        WAMIJ += 0.5 * es('amef,efij->amij', H.VAMEF, Tau)
        WAMIJ += P23(es('amej,ei->amij', H.VAMEI, T1))

        WAMEI = H.VAMEI.copy()
        WAMEI += 0.5 * es('mnef,afni->amei', H.VMNEF, T2)
        WAMEI += es('amef,fi->amei', H.VAMEF, T1)
        WAMEI -= es('nmei,an->amei', WMNEJ, T1)

        Z1 = H.fAI.copy()
        Z1 += es('ae,ei->ai', H.fAE, T1)
        Z1 -= es('mi,am->ai', FMI, T1)
        Z1 -= es('amei,em->ai', H.VAMEI, T1)
        Z1 += es('me,aeim->ai', FME, T2)
        Z1 += 0.5 * es('amef,efim->ai', H.VAMEF, Tau)
        Z1 -= 0.5 * es('mnei,eamn->ai', WMNEJ, T2)

        Z2 = H.VABIJ.copy()
        Z2 += P23(es('abej,ei->abij', H.VABEJ, T1))
        Z2 -= P01(es('amij,bm->abij', WAMIJ, T1))
        Z2 += P01(es('ae,ebij->abij', FAE, T2))
        Z2 -= P23(es('mi,abmj->abij', FMI, T2))
        Z2 += self.ladder(Tau)
        Z2 += 0.5 * es('mnij,abmn->abij', WMNIJ, Tau)
        Z2 += P23(P01(es('amei,ebjm->abij', WAMEI, T2)))
        if self.keep_intermediates:
            self.intermediates = dict(Tau=Tau, FME=FME, FMI=FMI, FAE=FAE, WMNIJ=WMNIJ, WMNEJ=WMNEJ, WAMIJ=WAMIJ,
                                      WAMEI=WAMEI, Z1=Z1, Z2=Z2)
        return Z1, Z2

    def energy_of(self, T: Amplitudes):
        Tau = self.make_tau(T)
        return float(np.vdot(self.H.fAI, T.T1) + 0.25 * np.vdot(self.H.VABIJ, Tau))

    def iterate(self):
        """One CCSD::iterate (ccsd.cxx:91-193)."""
        Z1, Z2 = self.residual(self.T)
        self.Z.T1[...] = weight(Z1, self.D1)
        self.Z.T2[...] = weight(Z2, self.D2)
        self.T.T1 += self.Z.T1
        self.T.T2 += self.Z.T2
        self.energy = self.energy_of(self.T)
        self.conv = float(max(np.abs(self.Z.T1).max(initial=0.0), np.abs(self.Z.T2).max(initial=0.0)))
        self.diis.extrapolate(self.T, self.Z)
        self.iter += 1
        return self.energy, self.conv

    def run(self, conv_tol=1e-9, max_iter=50, callback=None):
        """Iterative::run (iterative.hpp:126-166)."""
        it = 1
        while it <= max_iter and not (self.conv < conv_tol):
            e, c = self.iterate()
            if callback is not None:
                callback(it, e, c, self)
            it += 1
        return self.energy


# ----------------------------------------------------------------------------
# conveniences for the synthetic closed-shell problem
# ----------------------------------------------------------------------------

def hamiltonian_from_factor(B, eps, o, ladder_literal=False):
    eri = eri_from_factor(B)
    return Hamiltonian(np.diag(eps), eri, o, ladder_literal=ladder_literal)


def spin_block(x, spins, dims):
    """Extract one spin block from a full spin-orbital array.

    spins: tuple of 0/1 per axis, dims: spatial extent per axis.
    """
    sl = tuple(slice(s * d, (s + 1) * d) for s, d in zip(spins, dims))
    return x[sl]
