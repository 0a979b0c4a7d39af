"""The CPU oracle (test infrastructure) against independent restatements and closed forms."""
import numpy as np
import pytest

import aquarius_b200 as A
from oracle import ccsd_oracle as O
from oracle import rhf_ccsd as R


def _problem(seed, o, v, fock_noise=0.0):
    eps, B, *_ = A.synth_problem(seed, o, v)
    eri = O.eri_from_factor(B)
    F = np.diag(eps)
    if fock_noise:
        rng = np.random.default_rng(seed)
        X = rng.standard_normal(F.shape)
        F = F + fock_noise * (X + X.T)
    return F, eri


@pytest.mark.parametrize("o,v,seed,noise", [(3, 7, 1, 0.0), (4, 9, 2, 0.01), (2, 11, 5, 0.02)])
def test_spin_orbital_and_spin_adapted_oracles_agree(built_lib, o, v, seed, noise):
    F, eri = _problem(seed, o, v, noise)
    so = O.CCSD(O.Hamiltonian(F, eri, o), diis_order=8)
    e_so = so.run(1e-11, 100)
    rhf = R.RHFCCSD(F, eri, o, diis_order=8)
    e_rhf = rhf.run(1e-11, 100)
    assert abs(so.mp2 - rhf.mp2) < 1e-13
    assert abs(e_so - e_rhf) < 1e-10


def test_ladder_identity_matches_literal_vvvv(built_lib):
    F, eri = _problem(3, 3, 6)
    lit = O.CCSD(O.Hamiltonian(F, eri, 3, ladder_literal=True))
    idn = O.CCSD(O.Hamiltonian(F, eri, 3))
    a, b = lit.ladder(lit.Tau), idn.ladder(idn.Tau)
    assert np.abs(a - b).max() < 1e-15


def test_mp2_closed_form(built_lib):
    F, eri = _problem(4, 3, 8)
    c = O.CCSD(O.Hamiltonian(F, eri, 3))
    ref = 0.25 * np.sum(c.H.VABIJ ** 2 / c.D2)
    assert abs(c.mp2 - ref) < 1e-15


def test_amplitude_antisymmetry_preserved(built_lib):
    F, eri = _problem(5, 3, 7, 0.01)
    c = O.CCSD(O.Hamiltonian(F, eri, 3), diis_order=5)
    for _ in range(4):
        c.iterate()
    T2 = c.T.T2
    assert np.abs(T2 + T2.transpose(1, 0, 2, 3)).max() < 1e-15
    assert np.abs(T2 + T2.transpose(0, 1, 3, 2)).max() < 1e-15


def test_weight_zero_rule():
    x = np.array([1.0, 2.0, 3.0])
    d = np.array([1e-5, -2.0, 0.5])
    assert np.array_equal(O.weight(x, d), np.array([0.0, -1.0, 6.0]))


def test_diis_coefficients_sum_to_one(built_lib):
    F, eri = _problem(6, 3, 7)
    c = O.CCSD(O.Hamiltonian(F, eri, 3), diis_order=4)
    for _ in range(6):
        c.iterate()
        n = sum(x is not None for x in c.diis.old_dx)
        if n > 1:
            assert abs(c.diis.c[:n].sum() - 1.0) < 1e-10


def test_implicit_antisymmetrisation_helper():
    """The general helper of the Hbar/Lambda oracle gives the CCSD oracle's explicit
    P(ab)P(ij) forms: Tau and the ring term P(ab)P(ij) W_amei t_ebjm."""
    from oracle import lambda_ccsd as LC
    rng = np.random.default_rng(5)
    v, o = 6, 4
    T1 = rng.standard_normal((v, o))
    T2 = rng.standard_normal((v, v, o, o))
    T2 = T2 - T2.transpose(1, 0, 2, 3)
    T2 = T2 - T2.transpose(0, 1, 3, 2)
    W = rng.standard_normal((v, o, v, o))
    tau = O.CCSD.make_tau(O.Amplitudes(T1, T2))
    assert np.abs(T2 + LC.contract(0.5, T1, "ai", T1, "bj", "abij", LC.SHAPES["abij"]) - tau).max() < 1e-14
    ring = O.P23(O.P01(np.einsum("amei,ebjm->abij", W, T2)))
    assert np.abs(LC.contract(1.0, W, "amei", T2, "ebjm", "abij", LC.SHAPES["abij"]) - ring).max() < 1e-13


def test_hbar_without_amplitudes_is_the_bare_hamiltonian(built_lib):
    """With T = 0 every Hbar block is the bare block, except those the isHbar form
    assigns: the occupied-virtual Fock block and <ab||ij> and f_ai set to zero."""
    from oracle import lambda_ccsd as LC
    F, eri = _problem(4, 3, 5)
    H = O.Hamiltonian(F, eri, 3, ladder_literal=True)
    T1 = np.zeros_like(H.fAI)
    T2 = np.zeros_like(H.VABIJ)
    X = LC.hbar(H, T1, T2)
    bare = {"ij": H.fMI, "ab": H.fAE, "ijkl": H.VMNIJ, "aijk": H.VAMIJ, "ijak": H.VMNEJ, "ijab": H.VMNEF,
            "aibj": H.VAMEI, "aibc": H.VAMEF, "abci": H.VABEJ, "abcd": H.VABEF}
    for k, b in bare.items():
        assert np.array_equal(X[k], b), k
    for k in ("ia", "ai", "abij"):
        assert not X[k].any(), k


@pytest.mark.parametrize("o,v,seed", [(3, 7, 4), (4, 9, 6)])
def test_spin_orbital_hbar_matches_spin_adapted(built_lib, o, v, seed):
    """Two restatements that share no code: the spin-orbital Hbar (st2eoperator.hpp:59-130)
    of the converged spin-orbital T and the closed-shell "Form Hbar" (rhfccsd.cxx:110-186)
    of the converged spatial T give the same intermediates.  The spatial ones are spin blocks
    (A, I alpha; m, j beta): F = alpha-alpha blocks, W(Mn,Ij) = ijkl[AbAb]-type blocks, and
    W(Am,Ie) = -2 W[Am,eI]_(alpha beta beta alpha) - W[Am,Ei]_(alpha beta alpha beta)."""
    from oracle import lambda_ccsd as LC
    F, eri = _problem(seed, o, v)
    rhf = R.RHFCCSD(F, eri, o, diis_order=8)
    rhf.run(1e-12, 100)
    H = O.Hamiltonian(F, eri, o, ladder_literal=True)
    cc = O.CCSD(H, diis_order=8)
    cc.run(1e-12, 100)
    assert abs(rhf.energy - cc.energy) < 1e-12
    Hr = rhf.hbar()
    Hs = LC.hbar(H, cc.T.T1, cc.T.T2)

    def blk(x, spins, dims):
        return x[tuple(slice(s * d, (s + 1) * d) for s, d in zip(spins, dims))]

    pairs = {"FME": ("ia", (0, 0), (o, v)), "FMI": ("ij", (0, 0), (o, o)), "FAE": ("ab", (0, 0), (v, v)),
             "WMNIJ": ("ijkl", (0, 1, 0, 1), (o, o, o, o)), "WMNEJ": ("ijak", (0, 1, 0, 1), (o, o, v, o)),
             "WAMIJ": ("aijk", (0, 1, 0, 1), (v, o, o, o)), "WAMEI": ("aibj", (0, 1, 0, 1), (v, o, v, o)),
             "WABEJ": ("abci", (0, 1, 0, 1), (v, v, v, o))}
    for name, (key, spins, dims) in pairs.items():
        r = Hr[name]
        assert np.abs(r - blk(Hs[key], spins, dims)).max() < 1e-12 * max(1.0, np.abs(r).max()), name
    ring = -2 * blk(Hs["aibj"], (0, 1, 1, 0), (v, o, v, o)) - blk(Hs["aibj"], (0, 1, 0, 1), (v, o, v, o))
    assert np.abs(Hr["WAMIE"].transpose(0, 1, 3, 2) - ring).max() < 1e-12
