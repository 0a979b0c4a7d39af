"""CPU FP64 oracle for the steps after the CCSD iteration: the similarity-transformed
Hamiltonian (Hbar) and the Lambda-CCSD iteration, over full spin-orbital arrays.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only the tests and the smoke
entry point may import it.  The product path (aquarius_b200) never calls it.

It restates, statement for statement and in the reference's order:

* Hbar = (H e^T)_c up to two-electron terms, the form CCSD hands to Lambda
  (isHbar = true, T truncated at doubles):        src/operator/st2eoperator.hpp:59-130,
                                                  built by src/cc/ccsd.cxx:83-86
* the Lambda-CCSD initial guess, intermediates,
  residual, weight, update, energy, convergence
  and DIIS:                                       src/cc/lambdaccsd.cxx:27-133
* weight and norm of a de-excitation operator
  (dot weights 1, 1/4 as the excitation
  operator):                                      src/operator/deexcitationoperator.hpp:63-102
* denominators from the diagonals of Hbar's
  F_ae and F_mi (Denominator of H = Hbar):        src/cc/lambdaccsd.cxx:40,
                                                  src/operator/denominator.hpp:22-73

Every statement is an einsum over the full index ranges with the written factor, followed
by the implicit antisymmetrisation of output lines that come from both factors, separately
for upper/lower and occupied/virtual (src/tensor/spinorbital_tensor.cxx:637-669) -- the
same semantics as ccsd_oracle, here applied by one general helper instead of explicit
P(ab)/P(ij) calls.

Array conventions follow ccsd_oracle: a tensor's axes are its upper indices then its lower
indices, virtual before occupied within each; Lambda amplitudes are L1[i, a] and
L2[i, j, a, b] (upper occupied, lower virtual), as DeexcitationOperator stores them.
"""
from __future__ import annotations

from itertools import combinations

import numpy as np

from . import ccsd_oracle as O

# (upper vrt, upper occ, lower vrt, lower occ) line counts of every block used here
SHAPES = {
    "ia": (0, 1, 1, 0), "ai": (1, 0, 0, 1), "ij": (0, 1, 0, 1), "ab": (1, 0, 1, 0),
    "ijkl": (0, 2, 0, 2), "aijk": (1, 1, 0, 2), "ijak": (0, 2, 1, 1), "abij": (2, 0, 0, 2),
    "ijab": (0, 2, 2, 0), "aibj": (1, 1, 1, 1), "aibc": (1, 1, 2, 0), "abci": (2, 0, 1, 1),
    "abcd": (2, 0, 2, 0),
}


def _shuffle_sum(x, axes, from_a):
    """Sum over the ways of placing the A-lines and the B-lines of one output group on its
    positions, keeping each set's own order, with the sign of the permutation."""
    g = len(axes)
    na = sum(from_a)
    if na in (0, g):
        return x
    a_lines = [k for k in range(g) if from_a[k]]
    b_lines = [k for k in range(g) if not from_a[k]]
    out = np.zeros_like(x)
    for pos_a in combinations(range(g), na):
        pos_b = [p for p in range(g) if p not in pos_a]
        # source line placed at each position of the group
        src = [None] * g
        for p, k in zip(pos_a, a_lines):
            src[p] = k
        for p, k in zip(pos_b, b_lines):
            src[p] = k
        inv = sum(1 for p in range(g) for q in range(p + 1, g) if src[p] > src[q])
        perm = list(range(x.ndim))
        for p in range(g):
            perm[axes[p]] = axes[src[p]]
        out += (-1.0) ** inv * x.transpose(perm)
    return out


def contract(alpha, A, ia, B, ib, ic, shape_c):
    """alpha * A[ia] * B[ib] -> C[ic] with implicit antisymmetrisation of C's groups."""
    x = alpha * np.einsum(f"{ia},{ib}->{ic}", A, B, optimize=True)
    pos = 0
    for g in shape_c:
        letters = ic[pos:pos + g]
        x = _shuffle_sum(x, list(range(pos, pos + g)), [c in ia for c in letters])
        pos += g
    return x


def _vabef(H):
    if getattr(H, "VABEF", None) is not None:
        return H.VABEF
    v = H.v
    r = np.arange(v)
    return O._so_block(H.eri_vvvv, (r, r, r, r), (v, v, v, v))


def hbar(H, T1, T2):
    """STTwoElectronOperator(H, T, isHbar=true) for T = T1 + T2 (st2eoperator.hpp:59-130).

    Returns the 13 blocks keyed by the reference's block names (ia, ij, ab, ai, ijkl, aijk,
    ijak, abij, ijab, aibj, aibc, abci, abcd).  Note that the first statement assigns the
    occupied-virtual block, so the bare f_me does not survive (zero for an SCF reference).
    """
    X = {"ia": H.fME.copy(), "ij": H.fMI.copy(), "ab": H.fAE.copy(), "ai": H.fAI.copy(),
         "ijkl": H.VMNIJ.copy(), "aijk": H.VAMIJ.copy(), "ijak": H.VMNEJ.copy(), "abij": H.VABIJ.copy(),
         "ijab": H.VMNEF.copy(), "aibj": H.VAMEI.copy(), "aibc": H.VAMEF.copy(), "abci": H.VABEJ.copy(),
         "abcd": _vabef(H).copy()}
    Tau = T2 + contract(0.5, T1, "ai", T1, "bj", "abij", SHAPES["abij"])

    def c(alpha, A, ia, B, ib, blk, ic):
        return contract(alpha, A, ia, B, ib, ic, SHAPES[blk])

    X["ia"] = c(1.0, X["ijab"], "mnef", T1, "fn", "ia", "me")

    X["ij"] += c(0.5, X["ijab"], "nmef", T2, "efni", "ij", "mi")
    X["ij"] += c(1.0, X["ia"], "me", T1, "ei", "ij", "mi")
    X["ij"] += c(1.0, X["ijak"], "nmfi", T1, "fn", "ij", "mi")

    X["ijkl"] += c(0.5, X["ijab"], "mnef", Tau, "efij", "ijkl", "mnij")
    X["ijkl"] += c(1.0, X["ijak"], "nmei", T1, "ej", "ijkl", "mnij")

    X["ijak"] += c(1.0, X["ijab"], "mnef", T1, "fj", "ijak", "mnej")

    X["ai"][...] = 0.0

    X["ab"] -= c(0.5, X["ijab"], "mnfe", T2, "famn", "ab", "ae")
    X["ab"] -= c(1.0, X["ia"], "me", T1, "am", "ab", "ae")
    X["ab"] += c(1.0, X["aibc"], "anef", T1, "fn", "ab", "ae")

    X["aijk"] += c(0.5, X["aibc"], "amef", Tau, "efij", "aijk", "amij")
    X["aijk"] += c(1.0, X["aibj"], "amej", T1, "ei", "aijk", "amij")

    X["aibj"] -= c(0.5, X["ijab"], "mnef", T2, "afin", "aibj", "amei")
    X["aibj"] -= c(1.0, X["aibc"], "amfe", T1, "fi", "aibj", "amei")
    X["aibj"] -= c(1.0, X["ijak"], "nmei", T1, "an", "aibj", "amei")

    X["abij"][...] = 0.0

    X["aijk"] += c(1.0, X["ijak"], "nmej", T2, "aein", "aijk", "amij")
    X["aijk"] -= c(1.0, X["ijkl"], "nmij", T1, "an", "aijk", "amij")
    X["aijk"] += c(1.0, X["ia"], "me", T2, "aeij", "aijk", "amij")

    X["aibj"] -= c(0.5, X["ijab"], "mnef", T2, "afin", "aibj", "amei")
    X["aibj"] += c(0.5, X["ijak"], "nmei", T1, "an", "aibj", "amei")

    X["abci"] += c(0.5, X["ijak"], "mnej", T2, "abmn", "abci", "abej")
    X["abci"] -= c(1.0, X["aibj"], "amej", T1, "bm", "abci", "abej")
    X["abci"] += c(1.0, X["aibc"], "amef", T2, "fbmj", "abci", "abej")
    X["abci"] += c(1.0, X["abcd"], "abef", T1, "fj", "abci", "abej")
    X["abci"] -= c(1.0, X["ia"], "me", T2, "abmj", "abci", "abej")

    X["aibj"] -= c(0.5, X["ijak"], "nmei", T1, "an", "aibj", "amei")

    X["abcd"] += c(0.5, X["ijab"], "mnef", Tau, "abmn", "abcd", "abef")
    X["abcd"] -= c(1.0, X["aibc"], "amef", T1, "bm", "abcd", "abef")

    X["aibc"] -= c(1.0, X["ijab"], "nmef", T1, "an", "aibc", "amef")
    return X


class LambdaCCSD:
    """LambdaCCSD::run / iterate (lambdaccsd.cxx:27-133) on an Hbar from hbar()."""

    def __init__(self, Hb, T1, T2, diis_order=5, diis_start=1):
        self.Hb, self.T1, self.T2 = Hb, T1, T2
        dv = -np.diag(Hb["ab"]).copy()
        do = np.diag(Hb["ij"]).copy()
        self.D1 = do[:, None] + dv[None, :]                                      # [i, a]
        self.D2 = (do[:, None, None, None] + do[None, :, None, None]
                   + dv[None, None, :, None] + dv[None, None, None, :])         # [i, j, a, b]
        # L(0) = 1, L(1)[ia] = T(1)[ai], L(2)[ijab] = T(2)[abij]
        self.L = O.Amplitudes(T1.T.copy(), T2.transpose(2, 3, 0, 1).copy())
        self.Z = O.Amplitudes(np.zeros_like(self.L.T1), np.zeros_like(self.L.T2))
        self.diis = O.DIIS(diis_order, diis_start)
        self.energy = 0.0
        self.conv = np.finfo(float).max
        self.iter = 0

    def residual(self, L1, L2):
        H, T2 = self.Hb, self.T2
        sh = {"ij": SHAPES["ij"], "ab": SHAPES["ab"], "Z1": SHAPES["ia"], "Z2": SHAPES["ijab"]}

        def c(alpha, A, ia, B, ib, out, ic):
            return contract(alpha, A, ia, B, ib, ic, sh[out])

        GIM = c(0.5, T2, "efno", L2, "moef", "ij", "mn")
        GEA = c(-0.5, T2, "egmn", L2, "mnfg", "ab", "ef")

        Z1 = H["ia"].copy()
        Z1 += c(1.0, H["ab"], "ea", L1, "ie", "Z1", "ia")
        Z1 -= c(1.0, H["ij"], "im", L1, "ma", "Z1", "ia")
        Z1 -= c(1.0, H["aibj"], "eiam", L1, "me", "Z1", "ia")
        Z1 += c(0.5, H["abci"], "efam", L2, "imef", "Z1", "ia")
        Z1 -= c(0.5, H["aijk"], "eimn", L2, "mnea", "Z1", "ia")
        Z1 -= c(1.0, H["ijak"], "inam", GIM, "mn", "Z1", "ia")
        Z1 -= c(1.0, H["aibc"], "fiea", GEA, "ef", "Z1", "ia")

        Z2 = H["ijab"].copy()
        Z2 += c(1.0, H["ia"], "ia", L1, "jb", "Z2", "ijab")
        Z2 += c(1.0, H["aibc"], "ejab", L1, "ie", "Z2", "ijab")
        Z2 -= c(1.0, H["ijak"], "ijam", L1, "mb", "Z2", "ijab")
        Z2 += c(1.0, H["ab"], "ea", L2, "ijeb", "Z2", "ijab")
        Z2 -= c(1.0, H["ij"], "im", L2, "mjab", "Z2", "ijab")
        Z2 += c(0.5, H["abcd"], "efab", L2, "ijef", "Z2", "ijab")
        Z2 += c(0.5, H["ijkl"], "ijmn", L2, "mnab", "Z2", "ijab")
        Z2 += c(1.0, H["aibj"], "eiam", L2, "mjbe", "Z2", "ijab")
        Z2 -= c(1.0, H["ijab"], "mjab", GIM, "im", "Z2", "ijab")
        Z2 += c(1.0, H["ijab"], "ijeb", GEA, "ea", "Z2", "ijab")
        return Z1, Z2

    def iterate(self):
        Z1, Z2 = self.residual(self.L.T1, self.L.T2)
        self.Z.T1[...] = O.weight(Z1, self.D1)
        self.Z.T2[...] = O.weight(Z2, self.D2)
        self.L.T1 += self.Z.T1
        self.L.T2 += self.Z.T2
        self.energy = 0.25 * float(np.vdot(self.Hb["ijab"], self.L.T2))
        self.conv = float(max(np.abs(self.Z.T1).max(initial=0.0), np.abs(self.Z.T2).max(initial=0.0)))
        self.diis.extrapolate(self.L, self.Z)
        self.iter += 1
        return self.energy, self.conv

    def run(self, conv_tol=1e-9, max_iter=50):
        """Iterative::run (iterative.hpp:126-166)."""
        it = 1
        while it <= max_iter and not (self.conv < conv_tol):
            self.iterate()
            it += 1
        return self.energy


def lambda_from_ccsd(cc, diis_order=5):
    """Hbar of a converged ccsd_oracle.CCSD and a Lambda solver on it."""
    Hb = hbar(cc.H, cc.T.T1, cc.T.T2)
    return Hb, LambdaCCSD(Hb, cc.T.T1, cc.T.T2, diis_order=diis_order)
