"""Molecules, Gaussian basis sets, RHF/UHF and the MO-basis CCSD Hamiltonian.

TEST INFRASTRUCTURE ONLY (part of the oracle): it turns the reference's end-to-end test
inputs (test/input.aq: molecule, basis set, SCF) into the spin-orbital Hamiltonian
that the CCSD oracle and the device engine both consume, so that both can be checked
against the reference's known SCF / MP2 / CCSD energies.

What it restates, in its own code:
* basis-set file format (EMSL block: shell count, l values, contraction and primitive
  counts, exponents, coefficient matrix):             src/input/basis.cxx (BasisSet reader)
* spherical (pure) shells, the input default:           src/input/molecule.cxx:1241-1273
* SCF: the reference's "localaoscf" task is a UHF
  (src/scf/aouhf.cxx:291, src/scf/uhf.cxx) with DIIS
  on the orbital gradient FDS - SDF (uhf.cxx:362-402); closed shells give the RHF result
* AO -> MO transformation, no frozen core:             src/operator/aomoints.cxx

The SCF / CCSD energies are invariant to any non-singular transformation of the AO
basis inside its span, so contracted functions need not be normalised the way the
reference normalises them; only the span (pure vs Cartesian d) matters.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import native

ELEMENTS = {"H": 1, "HE": 2, "LI": 3, "BE": 4, "B": 5, "C": 6, "N": 7, "O": 8, "F": 9, "NE": 10}


# ----------------------------------------------------------------------------
# basis sets
# ----------------------------------------------------------------------------

def parse_basis(text: str, element: str):
    """Contracted shells of one element from an EMSL-format basis file.

    Returns a list of (l, exps, coefs) with one entry per contracted function group
    column (zero coefficients dropped); coefficients refer to normalised primitives.
    """
    lines = text.splitlines()
    tag = element.upper() + ":"
    start = None
    for i, ln in enumerate(lines):
        if ln.strip().upper().startswith(tag):
            start = i
            break
    if start is None:
        raise KeyError(element)
    toks = []
    for ln in lines[start + 2:]:
        s = ln.strip()
        if ":" in s:
            break
        toks.extend(s.split())
    pos = 0

    def take(k):
        nonlocal pos
        out = toks[pos:pos + k]
        pos += k
        return out

    ngroup = int(take(1)[0])
    ls = [int(x) for x in take(ngroup)]
    ncon = [int(x) for x in take(ngroup)]
    nprim = [int(x) for x in take(ngroup)]
    shells = []
    for g in range(ngroup):
        exps = np.array([float(x) for x in take(nprim[g])])
        coef = np.array([float(x) for x in take(nprim[g] * ncon[g])]).reshape(nprim[g], ncon[g])
        for c in range(ncon[g]):
            keep = coef[:, c] != 0.0
            shells.append((ls[g], exps[keep].copy(), coef[keep, c].copy()))
    return shells


def _prim_norm(a, l):
    """Norm of x^l exp(-a r^2)."""
    dfact = 1.0
    for k in range(2 * l - 1, 0, -2):
        dfact *= k
    return (2 * a / math.pi) ** 0.75 * (4 * a) ** (l / 2) / math.sqrt(dfact)


def _cart_to_pure(l):
    """Columns: pure components as combinations of the Cartesian components, in the
    order x^l, x^(l-1)y, x^(l-1)z, ... (i descending, then j descending)."""
    if l == 0:
        return np.eye(1)
    if l == 1:
        return np.eye(3)
    if l == 2:
        # cartesian order: xx, xy, xz, yy, yz, zz
        T = np.zeros((6, 5))
        T[1, 0] = 1.0                      # xy
        T[4, 1] = 1.0                      # yz
        T[0, 2], T[3, 2], T[5, 2] = -1.0, -1.0, 2.0  # 2zz - xx - yy
        T[2, 3] = 1.0                      # xz
        T[0, 4], T[3, 4] = 1.0, -1.0       # xx - yy
        return T
    raise NotImplementedError("pure shells above d are not needed for these tests")


@dataclass
class Molecule:
    symbols: list
    coords: np.ndarray               # bohr, (natom, 3)
    charge: int = 0
    multiplicity: int = 1
    charges: np.ndarray = field(init=False)

    def __post_init__(self):
        self.coords = np.asarray(self.coords, dtype=np.float64).reshape(-1, 3)
        self.charges = np.array([ELEMENTS[s.upper()] for s in self.symbols], dtype=np.float64)

    @property
    def nelec(self):
        return int(self.charges.sum()) - self.charge

    @property
    def nalpha_nbeta(self):
        n, s2 = self.nelec, self.multiplicity - 1
        return (n + s2) // 2, (n - s2) // 2

    def nuclear_repulsion(self):
        e = 0.0
        for i in range(len(self.symbols)):
            for j in range(i):
                e += self.charges[i] * self.charges[j] / np.linalg.norm(self.coords[i] - self.coords[j])
        return e


def ao_integrals(mol: Molecule, basis: dict, spherical=True):
    """S, Hcore, (mu nu|la si) over the molecule's AO basis.

    basis: element -> list of (l, exps, coefs) (from parse_basis).
    """
    shells, trans = [], []
    for sym, xyz in zip(mol.symbols, mol.coords):
        for l, exps, coefs in basis[sym.upper()]:
            c = np.array([cf * _prim_norm(a, l) for a, cf in zip(exps, coefs)])
            shells.append((l, xyz, exps, c))
            trans.append(_cart_to_pure(l) if spherical else np.eye((l + 1) * (l + 2) // 2))
    S, T, V, eri = native.cartesian_integrals(shells, mol.charges, mol.coords)
    nc = sum(t.shape[0] for t in trans)
    ns = sum(t.shape[1] for t in trans)
    X = np.zeros((nc, ns))
    r = c = 0
    for t in trans:
        X[r:r + t.shape[0], c:c + t.shape[1]] = t
        r += t.shape[0]
        c += t.shape[1]
    S = X.T @ S @ X
    H = X.T @ (T + V) @ X
    eri = np.einsum("pqrs,pa,qb,rc,sd->abcd", eri, X, X, X, X, optimize=True)
    # renormalise the pure functions (cosmetic: energies do not depend on it)
    d = 1.0 / np.sqrt(np.diag(S))
    S = S * d[:, None] * d[None, :]
    H = H * d[:, None] * d[None, :]
    eri = eri * d[:, None, None, None] * d[None, :, None, None] * d[None, None, :, None] * d[None, None, None, :]
    return S, H, eri


# ----------------------------------------------------------------------------
# SCF
# ----------------------------------------------------------------------------

@dataclass
class SCFResult:
    energy: float
    enuc: float
    Ca: np.ndarray
    Cb: np.ndarray
    ea: np.ndarray
    eb: np.ndarray
    na: int
    nb: int
    iterations: int


def _diis_extrap(focks, errs):
    m = len(focks)
    B = -np.ones((m + 1, m + 1))
    B[m, m] = 0.0
    for i in range(m):
        for j in range(m):
            B[i, j] = sum(float(np.vdot(ei, ej)) for ei, ej in zip(errs[i], errs[j]))
    rhs = np.zeros(m + 1)
    rhs[m] = -1.0
    c = np.linalg.solve(B, rhs)[:m]
    return [sum(c[i] * focks[i][k] for i in range(m)) for k in range(len(focks[0]))]


def scf(mol: Molecule, S, H, eri, conv=1e-12, max_iter=200, diis_start=2, diis_order=8, unrestricted=None):
    """RHF (closed shell) or UHF; core-Hamiltonian guess, DIIS on FDS - SDF."""
    na, nb = mol.nalpha_nbeta
    if unrestricted is None:
        unrestricted = na != nb
    enuc = mol.nuclear_repulsion()
    w, U = np.linalg.eigh(S)
    X = U @ np.diag(w ** -0.5) @ U.T

    def diag(F):
        e, Cp = np.linalg.eigh(X.T @ F @ X)
        return e, X @ Cp

    ea, Ca = diag(H)
    eb, Cb = ea.copy(), Ca.copy()
    focks, errs = [], []
    E_old = 0.0
    for it in range(1, max_iter + 1):
        Da = Ca[:, :na] @ Ca[:, :na].T
        Db = Cb[:, :nb] @ Cb[:, :nb].T
        J = np.einsum("pqrs,rs->pq", eri, Da + Db)
        Fa = H + J - np.einsum("prqs,rs->pq", eri, Da)
        Fb = H + J - np.einsum("prqs,rs->pq", eri, Db)
        E = enuc + 0.5 * (np.vdot(Da, H + Fa) + np.vdot(Db, H + Fb))
        ra = Fa @ Da @ S - S @ Da @ Fa
        rb = Fb @ Db @ S - S @ Db @ Fb
        err = max(np.abs(ra).max(), np.abs(rb).max())
        if abs(E - E_old) < conv and err < 1e-9:
            return SCFResult(float(E), enuc, Ca, Cb, ea, eb, na, nb, it)
        E_old = E
        focks.append((Fa, Fb))
        errs.append((ra, rb))
        if len(focks) > diis_order:
            focks.pop(0)
            errs.pop(0)
        if it >= diis_start and len(focks) >= 2:
            Fa, Fb = _diis_extrap(focks, errs)
        if unrestricted:
            ea, Ca = diag(Fa)
            eb, Cb = diag(Fb)
        else:
            ea, Ca = diag(0.5 * (Fa + Fb))
            eb, Cb = ea, Ca
    raise RuntimeError("SCF did not converge")


# ----------------------------------------------------------------------------
# spin-orbital MO Hamiltonian
# ----------------------------------------------------------------------------

class SpinOrbitalHamiltonian:
    """The 13 H blocks over spin-orbitals ordered, in each of occ and vrt, alpha first.

    Spin-orbital counts: occ = na + nb, vrt = (n - na) + (n - nb).  Built with the literal
    <ab||ef> block (the ladder identity of the closed-shell oracle Hamiltonian needs
    shared spatial orbitals).  Attributes match ccsd_oracle.Hamiltonian.
    """

    def __init__(self, res: SCFResult, H, eri):
        n = H.shape[0]
        na, nb = res.na, res.nb
        Ca, Cb = res.Ca, res.Cb
        # spin-orbital coefficient lists: (C column, spin)
        cols = ([(Ca[:, i], 0) for i in range(na)] + [(Cb[:, i], 1) for i in range(nb)]
                + [(Ca[:, i], 0) for i in range(na, n)] + [(Cb[:, i], 1) for i in range(nb, n)])
        C = np.array([c for c, _ in cols]).T               # AO x SO
        spin = np.array([s for _, s in cols])
        no = na + nb
        nso = 2 * n
        Da = Ca[:, :na] @ Ca[:, :na].T
        Db = Cb[:, :nb] @ Cb[:, :nb].T
        J = np.einsum("pqrs,rs->pq", eri, Da + Db)
        Fa = H + J - np.einsum("prqs,rs->pq", eri, Da)
        Fb = H + J - np.einsum("prqs,rs->pq", eri, Db)
        F = np.zeros((nso, nso))
        same = spin[:, None] == spin[None, :]
        Fa_mo = C.T @ Fa @ C
        Fb_mo = C.T @ Fb @ C
        F[:] = np.where(spin[:, None] == 0, Fa_mo, Fb_mo) * same
        mo = np.einsum("pqrs,pa,qb,rc,sd->abcd", eri, C, C, C, C, optimize=True)   # (ab|cd) spatial parts
        # make the 8-fold permutational symmetry exact (the transformation's rounding
        # differs between images): the blocks then are exactly antisymmetric / Hermitian
        mo = 0.5 * (mo + mo.transpose(1, 0, 2, 3))
        mo = 0.5 * (mo + mo.transpose(0, 1, 3, 2))
        mo = 0.5 * (mo + mo.transpose(2, 3, 0, 1))
        # <pq|rs> = (pr|qs) d(sp,sr) d(sq,ss)
        phys = mo.transpose(0, 2, 1, 3) * (same[:, None, :, None] * same[None, :, None, :])
        G = phys - phys.transpose(0, 1, 3, 2)
        O = np.arange(no)
        V = np.arange(no, nso)
        blk = lambda a, b, c, d: np.ascontiguousarray(G[np.ix_(a, b, c, d)])
        self.nocc = (na, nb)
        self.nvrt = (n - na, n - nb)
        self.fAI = np.ascontiguousarray(F[np.ix_(V, O)])
        self.fME = np.ascontiguousarray(F[np.ix_(O, V)])
        self.fAE = np.ascontiguousarray(F[np.ix_(V, V)])
        self.fMI = np.ascontiguousarray(F[np.ix_(O, O)])
        self.VMNIJ = blk(O, O, O, O)
        self.VAMIJ = blk(V, O, O, O)
        self.VMNEJ = blk(O, O, V, O)
        self.VABIJ = blk(V, V, O, O)
        self.VMNEF = blk(O, O, V, V)
        self.VAMEI = blk(V, O, V, O)
        self.VAMEF = blk(V, O, V, V)
        self.VABEJ = blk(V, V, V, O)
        self.VABEF = blk(V, V, V, V)
        self.dv = -np.diag(self.fAE).copy()
        self.do = np.diag(self.fMI).copy()


# ----------------------------------------------------------------------------
# fixtures
# ----------------------------------------------------------------------------

def from_fixture(fixture: dict, name: str):
    """(Molecule, basis) for one entry of a molecules fixture (geometry in bohr)."""
    m = fixture["molecules"][name]
    mol = Molecule([a[0] for a in m["atoms"]], [a[1:] for a in m["atoms"]], multiplicity=m["multiplicity"])
    table = fixture["basis"][m["basis_set"]]
    basis = {el: [(l, np.array(e), np.array(c)) for l, e, c in shells] for el, shells in table.items()}
    return mol, basis


def solve_scf(fixture: dict, name: str):
    """AO integrals + SCF for a fixture entry: (SCFResult, Hcore, eri)."""
    mol, basis = from_fixture(fixture, name)
    S, H, eri = ao_integrals(mol, basis)
    return scf(mol, S, H, eri), H, eri


def mo_integrals(res: SCFResult, H, eri):
    """Spatial MO integrals of a closed-shell result: (h, (pq|rs)) over the alpha
    orbitals, with the 8-fold symmetry made exact."""
    C = res.Ca
    h = C.T @ H @ C
    h = 0.5 * (h + h.T)
    mo = np.einsum("pqrs,pa,qb,rc,sd->abcd", eri, C, C, C, C, optimize=True)
    mo = 0.5 * (mo + mo.transpose(1, 0, 2, 3))
    mo = 0.5 * (mo + mo.transpose(0, 1, 3, 2))
    mo = 0.5 * (mo + mo.transpose(2, 3, 0, 1))
    return h, mo
