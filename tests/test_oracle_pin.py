"""The CPU oracle against the reference's own end-to-end known answers.

test/input.aq:1-24 (H2O/cc-pVDZ, closed shell) and test/input.aq:47-71 (CH2/cc-pVDZ,
triplet, UHF) compare the SCF, MP2, CCSD and Lambda-CCSD energies to 1e-9 Eh.  The fixture
(tests/golden/molecules.json) holds the geometries, basis sets and those energies;
the integrals, the SCF and the CCSD iterations are the oracle's own.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import ccsd_oracle as O
from oracle import lambda_ccsd as LC
from oracle import scf

FIXTURE = json.loads((Path(__file__).parent / "golden" / "molecules.json").read_text())


@pytest.fixture(scope="module", params=["h2o-pvdz", "ch2-pvdz"])
def system(request):
    name = request.param
    res, H, eri = scf.solve_scf(FIXTURE, name)
    return name, res, scf.SpinOrbitalHamiltonian(res, H, eri)


def test_scf_energy(system):
    name, res, _ = system
    known = FIXTURE["molecules"][name]["known"]
    assert abs(res.energy - known["scf"]) < known["tolerance"], (res.energy, known["scf"])


def test_mp2_and_ccsd_energies(system):
    name, res, Hso = system
    known = FIXTURE["molecules"][name]["known"]
    cc = O.CCSD(Hso, diis_order=5)
    assert abs(cc.mp2 - known["mp2"]) < known["tolerance"], (cc.mp2, known["mp2"])
    e = cc.run(conv_tol=1e-11, max_iter=100)
    assert cc.conv < 1e-11
    assert abs(e - known["ccsd"]) < known["tolerance"], (e, known["ccsd"])


def test_lambda_energy(system):
    """Hbar of the converged T (st2eoperator.hpp, isHbar) and the Lambda iteration
    (lambdaccsd.cxx): 1/4 <mn||ef> l_mn^ef at convergence."""
    name, res, Hso = system
    known = FIXTURE["molecules"][name]["known"]
    cc = O.CCSD(Hso, diis_order=5)
    cc.run(conv_tol=1e-11, max_iter=100)
    Hb, lam = LC.lambda_from_ccsd(cc)
    e = lam.run(conv_tol=1e-11, max_iter=100)
    assert lam.conv < 1e-11
    assert abs(e - known["lambda"]) < known["tolerance"], (e, known["lambda"])
    # L2 keeps the antisymmetry of its upper and lower pairs
    L2 = lam.L.T2
    assert np.abs(L2 + L2.transpose(1, 0, 2, 3)).max() < 1e-13
    assert np.abs(L2 + L2.transpose(0, 1, 3, 2)).max() < 1e-13


def test_spin_orbital_hamiltonian_symmetries(system):
    _, res, Hso = system
    na, nb = Hso.nocc
    # Brillouin: the converged SCF has no occupied-virtual Fock coupling
    assert np.abs(Hso.fAI).max() < 1e-7
    # antisymmetry and Hermiticity of the stored blocks
    assert np.array_equal(Hso.VABEF, -Hso.VABEF.transpose(1, 0, 2, 3))
    assert np.array_equal(Hso.VABIJ, Hso.VMNEF.transpose(2, 3, 0, 1))
    assert np.array_equal(Hso.VMNEJ, Hso.VAMIJ.transpose(2, 3, 0, 1))
    # spin blocks forbidden by spin conservation are zero (alpha-beta Fock block)
    va = Hso.nvrt[0]
    assert np.abs(Hso.fAE[:va, va:]).max() == 0.0


def h2o_equilibrium():
    """H2O with O-H 0.9572 A and H-O-H 104.52 deg, O at the origin (C1), in bohr."""
    r = 0.9572 / 0.529177210903
    half = np.deg2rad(104.52) / 2
    return scf.Molecule(["O", "H", "H"], [[0, 0, 0], [r * np.sin(half), 0, r * np.cos(half)],
                                          [-r * np.sin(half), 0, r * np.cos(half)]])


def test_h2o_equilibrium_two_oracles_agree():
    """The CPU-runnable workload (H2O/cc-pVDZ at its equilibrium geometry, all electrons,
    residual 1e-10, DIIS 8): no reference energy exists for it, so the spin-orbital
    oracle is checked against the independent spin-adapted one."""
    from oracle import rhf_ccsd as R
    basis = {el: [(l, np.array(e), np.array(c)) for l, e, c in sh] for el, sh in FIXTURE["basis"]["cc-pVDZ"].items()}
    mol = h2o_equilibrium()
    S, H, eri = scf.ao_integrals(mol, basis)
    res = scf.scf(mol, S, H, eri)
    assert -76.1 < res.energy < -75.9
    h, mo = scf.mo_integrals(res, H, eri)
    fock = h + 2 * np.einsum("pqii->pq", mo[:, :, :5, :5]) - np.einsum("piiq->pq", mo[:, :5, :5, :])
    so = O.CCSD(O.Hamiltonian(fock, mo, 5), diis_order=8)
    e_so = so.run(conv_tol=1e-10, max_iter=100)
    rhf = R.RHFCCSD(fock, mo, 5, diis_order=8)
    e_rhf = rhf.run(1e-10, 100)
    assert abs(so.mp2 - rhf.mp2) < 1e-12
    assert abs(e_so - e_rhf) < 1e-9


def test_integrals_overlap_normalised():
    mol, basis = scf.from_fixture(FIXTURE, "h2o-pvdz")
    S, H, eri = scf.ao_integrals(mol, basis)
    assert S.shape == (24, 24)
    assert np.allclose(np.diag(S), 1.0, atol=1e-13)
    # 8-fold permutational symmetry of (mu nu|la si)
    assert np.allclose(eri, eri.transpose(1, 0, 2, 3), atol=1e-14)
    assert np.allclose(eri, eri.transpose(2, 3, 0, 1), atol=1e-14)
    # positive definite Coulomb metric
    w = np.linalg.eigvalsh(eri.reshape(24 * 24, 24 * 24))
    assert w.min() > -1e-12
