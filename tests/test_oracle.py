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
