"""Second, independent CPU oracle: closed-shell spin-adapted CCSD.

TEST INFRASTRUCTURE ONLY (see ccsd_oracle.py).  Restates RHFCCSD::iterate
(src/cc/rhfccsd.cxx:193-327) and its setup (src/cc/rhfccsd.cxx:44-110) over
spatial orbitals.  Its integrals are the non-antisymmetrised physicist-notation
blocks  V_pqrs = <pq|rs> = (pr|qs):
  VABIJ <ab|ij>, VAIBJ <ai|bj>, VAIJB <ai|jb>, VABCI <ab|ci>, VAIJK <ai|jk>,
  VIJKL <ij|kl>, VABCD <ab|cd>.
It is used only to cross-check the converged spin-orbital energy: the two
formulations share no code and must agree to the convergence threshold.
"""
from __future__ import annotations

import numpy as np
from scipy.linalg import lapack


def es(spec, *ops):
    return np.einsum(spec, *ops, optimize=True)


def weight(x, den):
    small = np.abs(den) < 1e-4
    return np.where(small, 0.0, x / np.where(small, 1.0, den))


class RHFCCSD:
    def __init__(self, fock, eri, o, diis_order=5):
        n = fock.shape[0]
        v = n - o
        Ox, Vx = slice(0, o), slice(o, n)
        phys = eri.transpose(0, 2, 1, 3)            # <pq|rs> = (pr|qs)
        self.fAI = fock[Vx, Ox].copy()
        self.fAB = fock[Vx, Vx].copy()
        self.fIJ = fock[Ox, Ox].copy()
        self.VABIJ = phys[Vx, Vx, Ox, Ox].copy()
        self.VAIBJ = phys[Vx, Ox, Vx, Ox].copy()
        self.VAIJB = phys[Vx, Ox, Ox, Vx].copy()
        self.VABCI = phys[Vx, Vx, Vx, Ox].copy()
        self.VAIJK = phys[Vx, Ox, Ox, Ox].copy()
        self.VIJKL = phys[Ox, Ox, Ox, Ox].copy()
        self.VABCD = phys[Vx, Vx, Vx, Vx].copy()
        dA = -np.diag(fock)[o:]
        dI = np.diag(fock)[:o]
        self.D1 = dA[:, None] + dI[None, :]
        self.D2 = dA[:, None, None, None] + dA[None, :, None, None] + dI[None, None, :, None] + dI[None, None, None, :]
        self.T1 = weight(self.fAI.copy(), self.D1)
        self.T2 = weight(self.VABIJ.copy(), self.D2)
        self.VABIJSA = 2 * self.VABIJ - self.VABIJ.transpose(0, 1, 3, 2)
        self.VAIJBSA = 2 * self.VAIJB - self.VAIBJ.transpose(0, 1, 3, 2)
        Tau = self.T2 + es('ai,bj->abij', self.T1, self.T1)
        self.mp2 = 2 * float(np.vdot(self.fAI, self.T1)) + float(np.vdot(self.VABIJSA, Tau))
        self.order = diis_order
        self.xs, self.dxs = [], []
        self.energy = self.mp2
        self.conv = np.finfo(float).max

    def iterate(self):
        Z1, Z2 = self.residual(self.T1, self.T2)
        fAI, VABIJSA = self.fAI, self.VABIJSA
        Z1 = weight(Z1, self.D1)
        Z2 = weight(Z2, self.D2)
        T1 = self.T1 + Z1
        T2 = self.T2 + Z2
        Tau = T2 + es('ai,bj->abij', T1, T1)
        self.energy = 2 * float(np.vdot(fAI, T1)) + float(np.vdot(VABIJSA, Tau))
        self.conv = max(np.abs(Z1).max(), np.abs(Z2).max())
        self.T1, self.T2 = self._diis(T1, T2, Z1, Z2)
        return self.energy, self.conv

    def residual(self, T1, T2):
        """The intermediates and the unweighted residual (rhfccsd.cxx:237-316)."""
        fAI, fAB, fIJ = self.fAI, self.fAB, self.fIJ
        VABIJ, VAIBJ, VAIJB, VABCI = self.VABIJ, self.VAIBJ, self.VAIJB, self.VABCI
        VAIJK, VIJKL, VABCD = self.VAIJK, self.VIJKL, self.VABCD
        VABIJSA, VAIJBSA = self.VABIJSA, self.VAIJBSA

        Tau = T2 + es('ai,bj->abij', T1, T1)
        TauSA = 2 * Tau - Tau.transpose(0, 1, 3, 2)
        T2SA = 2 * T2 - T2.transpose(0, 1, 3, 2)

        FME = fAI.T + es('efmn,fn->me', VABIJSA, T1)
        FMI = fIJ + es('efmn,efin->mi', VABIJSA, T2) + es('me,ei->mi', FME, T1) \
            + 2 * es('finm,fn->mi', VAIJK, T1) - es('fimn,fn->mi', VAIJK, T1)
        FAE = fAB - es('efmn,afmn->ae', VABIJSA, T2) - es('me,am->ae', FME, T1) \
            + 2 * es('efam,fm->ae', VABCI, T1) - es('feam,fm->ae', VABCI, T1)

        WMNIJ = 0.5 * VIJKL + 0.5 * es('efmn,efij->mnij', VABIJ, Tau) + es('ejmn,ei->mnij', VAIJK, T1)
        WMNIJ = WMNIJ + WMNIJ.transpose(1, 0, 3, 2)

        WMNEJ = VAIJK.transpose(2, 3, 0, 1) + es('efmn,fj->mnej', VABIJ, T1)

        WAMIJ = VAIJK + es('efam,efij->amij', VABCI, Tau) + es('amej,ei->amij', VAIBJ, T1) \
            + es('amie,ej->amij', VAIJB, T1)

        WAMIE = VAIJBSA + 0.5 * es('efmn,afin->amie', VABIJSA, T2SA) + 2 * es('feam,fi->amie', VABCI, T1) \
            - es('efam,fi->amie', VABCI, T1) - 2 * es('mnei,an->amie', WMNEJ, T1) + es('nmei,an->amie', WMNEJ, T1)

        WAMEI = VAIBJ - 0.5 * es('efnm,afni->amei', VABIJ, T2) + es('efam,fi->amei', VABCI, T1) \
            - es('nmei,an->amei', WMNEJ, T1)

        Z1 = fAI + es('ae,ei->ai', fAB, T1) - es('mi,am->ai', FMI, T1) + es('amie,em->ai', VAIJBSA, T1) \
            + es('me,aeim->ai', FME, T2SA) + es('efam,efim->ai', VABCI, TauSA) - es('mnei,eamn->ai', WMNEJ, T2SA)

        Z2 = 0.5 * VABIJ + es('abej,ei->abij', VABCI, T1) - es('amij,bm->abij', WAMIJ, T1) \
            + es('ae,ebij->abij', FAE, T2) - es('mi,abmj->abij', FMI, T2) + 0.5 * es('abef,efij->abij', VABCD, Tau) \
            + 0.5 * es('mnij,abmn->abij', WMNIJ, Tau) + 0.5 * es('amie,ebmj->abij', WAMIE, T2SA) \
            - 0.5 * es('amei,ebjm->abij', WAMEI, T2) - es('amej,ebim->abij', WAMEI, T2)
        Z2 = Z2 + Z2.transpose(1, 0, 3, 2)
        return Z1, Z2

    def _diis(self, T1, T2, Z1, Z2):
        # diis.hpp:70-227 with two x and two dx; inner product sum_j <dx_j, dx'_j>
        self.xs.insert(0, (T1.copy(), T2.copy()))
        self.dxs.insert(0, (Z1.copy(), Z2.copy()))
        del self.xs[self.order:], self.dxs[self.order:]
        k = len(self.dxs)
        if k == 1:
            return T1, T2
        e = np.zeros((k + 1, k + 1))
        for i in range(k):
            for j in range(k):
                e[i, j] = float(np.vdot(self.dxs[i][0], self.dxs[j][0]) + np.vdot(self.dxs[i][1], self.dxs[j][1]))
        e[:k, k] = e[k, :k] = -1.0
        c = np.zeros(k + 1)
        c[k] = -1.0
        _, _, sol, info = lapack.dsysv(e, c, lower=0)
        if info != 0:
            raise RuntimeError("DIIS: Info in hesv: %d" % info)
        T1 = sum(sol[i] * self.xs[i][0] for i in range(k))
        T2 = sum(sol[i] * self.xs[i][1] for i in range(k))
        return T1, T2

    def hbar(self):
        """"Form Hbar" of RHFCCSD<U>::run (rhfccsd.cxx:110-186) from the current T1, T2, in
        the reference's index orders (W(Am,Ie) as [a, m, i, e])."""
        T1, T2 = self.T1, self.T2
        fAI, fAB, fIJ = self.fAI, self.fAB, self.fIJ
        VABIJ, VAIBJ, VAIJB, VABCI = self.VABIJ, self.VAIBJ, self.VAIJB, self.VABCI
        VAIJK, VIJKL, VABCD = self.VAIJK, self.VIJKL, self.VABCD
        VABIJSA, VAIJBSA = self.VABIJSA, self.VAIJBSA
        Tau = T2 + es('ai,bj->abij', T1, T1)
        T2SA = 2 * T2 - T2.transpose(0, 1, 3, 2)
        FME = fAI.T + es('efmn,fn->me', VABIJSA, T1)
        FMI = fIJ + es('efmn,efin->mi', VABIJSA, T2) + es('me,ei->mi', FME, T1) \
            + 2 * es('finm,fn->mi', VAIJK, T1) - es('fimn,fn->mi', VAIJK, T1)
        FAE = fAB - es('efmn,afmn->ae', VABIJSA, T2) - es('me,am->ae', FME, T1) \
            + 2 * es('efam,fm->ae', VABCI, T1) - es('feam,fm->ae', VABCI, T1)
        WMNIJ = 0.5 * VIJKL + 0.5 * es('efmn,efij->mnij', VABIJ, Tau) + es('ejmn,ei->mnij', VAIJK, T1)
        WMNIJ = WMNIJ + WMNIJ.transpose(1, 0, 3, 2)
        WMNEJ = VAIJK.transpose(2, 3, 0, 1) + es('efmn,fj->mnej', VABIJ, T1)
        WAMIJ = VAIJK + es('efam,efij->amij', VABCI, Tau) + es('amej,ei->amij', VAIBJ, T1) \
            + es('amie,ej->amij', VAIJB, T1) - es('nmij,an->amij', WMNIJ, T1) \
            + es('nmej,aein->amij', WMNEJ, T2SA) - es('mnej,aein->amij', WMNEJ, T2) \
            - es('mnei,aenj->amij', WMNEJ, T2) + es('me,aeij->amij', FME, T2)
        WAMIE = VAIJBSA + es('efmn,afin->amie', VABIJSA, T2SA) + 2 * es('feam,fi->amie', VABCI, T1) \
            - es('efam,fi->amie', VABCI, T1)
        WAMEI = VAIBJ - es('efnm,afni->amei', VABIJ, T2) + es('efam,fi->amei', VABCI, T1)
        WABEJ = VABCI + es('mnej,abmn->abej', WMNEJ, Tau) - 0.5 * es('bmje,am->abej', WAMIE, T1) \
            - 0.5 * es('bmej,am->abej', WAMEI, T1) - es('amej,bm->abej', WAMEI, T1) \
            + es('abef,fj->abej', VABCD, T1) + es('efam,fbmj->abej', VABCI, T2SA) \
            - es('feam,fbmj->abej', VABCI, T2) - es('febm,afmj->abej', VABCI, T2) - es('me,abmj->abej', FME, T2)
        WAMIE = WAMIE - 2 * es('mnei,an->amie', WMNEJ, T1) + es('nmei,an->amie', WMNEJ, T1)
        WAMEI = WAMEI - es('nmei,an->amei', WMNEJ, T1)
        return {"FME": FME, "FMI": FMI, "FAE": FAE, "WMNIJ": WMNIJ, "WMNEJ": WMNEJ, "WAMIJ": WAMIJ,
                "WAMIE": WAMIE, "WAMEI": WAMEI, "WABEJ": WABEJ}

    def run(self, conv_tol=1e-9, max_iter=50):
        it = 1
        while it <= max_iter and not (self.conv < conv_tol):
            self.iterate()
            it += 1
        return self.energy
