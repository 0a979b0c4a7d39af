"""The device engine against the reference's own end-to-end known answers.

test/input.aq:1-24 (H2O/cc-pVDZ, closed shell) and :47-71 (CH2/cc-pVDZ triplet, UHF):
SCF, MP2 and CCSD energies to 1e-9 Eh, the reference's tolerance.  The H2O integrals
reach the engine through its FCIDUMP reader (src/operator/fcidump.cxx); the UHF blocks
through ccsd_hamiltonian_create + block writes.  Integrals and SCF come from the oracle.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import aquarius_b200 as A
from oracle import ccsd_oracle as O
from oracle import scf
from tests.helpers import write_fcidump, write_full

pytestmark = pytest.mark.gpu

FIXTURE = json.loads((Path(__file__).parent / "golden" / "molecules.json").read_text())
BASE_BLOCKS = ["fAI", "fME", "fAE", "fMI", "VMNIJ", "VAMIJ", "VMNEF", "VAMEI", "VAMEF", "VABEF"]


@pytest.fixture(scope="module")
def h2o():
    res, H, eri = scf.solve_scf(FIXTURE, "h2o-pvdz")
    h, mo = scf.mo_integrals(res, H, eri)
    return res, h, mo, FIXTURE["molecules"]["h2o-pvdz"]["known"]


@pytest.fixture(scope="module")
def ch2():
    res, H, eri = scf.solve_scf(FIXTURE, "ch2-pvdz")
    return res, scf.SpinOrbitalHamiltonian(res, H, eri), FIXTURE["molecules"]["ch2-pvdz"]["known"]


def _rotation(rng, n):
    q, r = np.linalg.qr(rng.standard_normal((n, n)))
    return q * np.sign(np.diag(r))


@pytest.mark.parametrize("pack", [True, False], ids=["packed", "unpacked"])
def test_h2o_fcidump_known_answers(h2o, tmp_path, pack):
    res, h, mo, known = h2o
    path = tmp_path / "FCIDUMP"
    write_fcidump(path, h, mo, nelec=10, ecore=res.enuc)
    with A.Context(0) as ctx:
        H, escf = ctx.hamiltonian_from_fcidump(path, pack_vvvv=pack)
        assert abs(escf - known["scf"]) < known["tolerance"], escf
        s = ctx.solver(H, conv_tol=1e-11, max_iter=100, diis_order=5)
        assert abs(s.mp2 - known["mp2"]) < known["tolerance"], s.mp2
        e, conv, iters = s.run()
        assert conv < 1e-11
        assert abs(e - known["ccsd"]) < known["tolerance"], (e, iters)
        s.close()
        H.destroy()


def test_h2o_semicanonical_rotated_orbitals(h2o, tmp_path):
    """Rotations inside occ and inside vrt leave E(SCF) and E(CCSD) unchanged; the
    semicanonical option brings the Fock blocks back to diagonal form."""
    res, h, mo, known = h2o
    rng = np.random.default_rng(5)
    U = np.zeros((24, 24))
    U[:5, :5] = _rotation(rng, 5)
    U[5:, 5:] = _rotation(rng, 19)
    h2 = U.T @ h @ U
    mo2 = np.einsum("pqrs,pa,qb,rc,sd->abcd", mo, U, U, U, U, optimize=True)
    mo2 = 0.5 * (mo2 + mo2.transpose(1, 0, 2, 3))
    mo2 = 0.5 * (mo2 + mo2.transpose(0, 1, 3, 2))
    mo2 = 0.5 * (mo2 + mo2.transpose(2, 3, 0, 1))
    path = tmp_path / "FCIDUMP.rot"
    write_fcidump(path, 0.5 * (h2 + h2.T), mo2, nelec=10, ecore=res.enuc)
    with A.Context(0) as ctx:
        H, escf = ctx.hamiltonian_from_fcidump(path, semicanonical=True)
        assert abs(escf - known["scf"]) < known["tolerance"]
        fae = H["fAE"].to_full()
        assert np.abs(fae - np.diag(np.diag(fae))).max() < 1e-10
        s = ctx.solver(H, conv_tol=1e-11, max_iter=100)
        e, conv, _ = s.run()
        assert abs(e - known["ccsd"]) < known["tolerance"], e
        s.close()


def test_h2o_noncanonical_matches_oracle_every_iteration(h2o):
    """Non-diagonal Fock blocks (rotated orbitals, no semicanonicalisation): every
    off-diagonal Fock term of the iteration is exercised against the oracle."""
    res, h, mo, known = h2o
    rng = np.random.default_rng(9)
    U = np.zeros((24, 24))
    U[:5, :5] = _rotation(rng, 5)
    U[5:, 5:] = _rotation(rng, 19)
    mo2 = np.einsum("pqrs,pa,qb,rc,sd->abcd", mo, U, U, U, U, optimize=True)
    mo2 = 0.5 * (mo2 + mo2.transpose(1, 0, 2, 3))
    mo2 = 0.5 * (mo2 + mo2.transpose(0, 1, 3, 2))
    mo2 = 0.5 * (mo2 + mo2.transpose(2, 3, 0, 1))
    h2 = U.T @ h @ U
    h2 = 0.5 * (h2 + h2.T)
    fock = h2 + 2 * np.einsum("pqii->pq", mo2[:, :, :5, :5]) - np.einsum("piiq->pq", mo2[:, :5, :5, :])
    ref = O.CCSD(O.Hamiltonian(fock, mo2, 5, ladder_literal=True), diis_order=5)
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=[19], occ=[5])
        H = ctx.hamiltonian_from_integrals(fock, mo2)
        s = ctx.solver(H, diis_order=5)
        assert abs(s.mp2 - ref.mp2) < 1e-12
        for it in range(8):
            e_ref, c_ref = ref.iterate()
            e, c = s.iterate()
            assert abs(e - e_ref) < 1e-11, (it, e, e_ref)
            assert abs(c - c_ref) <= 1e-9 * max(1e-3, c_ref), (it, c, c_ref)
        assert np.abs(s.T2.to_full() - ref.T.T2).max() < 1e-11
        s.close()


@pytest.mark.parametrize("pack", [True, False], ids=["packed", "unpacked"])
def test_ch2_uhf_known_answers(ch2, pack):
    res, Hso, known = ch2
    (na, nb), (va, vb) = Hso.nocc, Hso.nvrt
    ref = O.CCSD(Hso, diis_order=5)
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=[va], occ=[na], vrt_beta=[vb], occ_beta=[nb])
        H = ctx.hamiltonian(pack_vvvv=pack)
        for name in BASE_BLOCKS:
            write_full(H[name], getattr(Hso, name))
        # the Hermitian views follow the blocks they alias
        assert np.array_equal(H["VABIJ"].to_full(), Hso.VABIJ)
        s = ctx.solver(H, conv_tol=1e-11, max_iter=100, diis_order=5)
        assert abs(s.mp2 - ref.mp2) < 1e-12
        assert abs(s.mp2 - known["mp2"]) < known["tolerance"], s.mp2
        for it in range(5):
            e_ref, _ = ref.iterate()
            e, _ = s.iterate()
            assert abs(e - e_ref) < 1e-11, (it, e, e_ref)
        e, conv, iters = s.run()
        assert conv < 1e-11
        assert abs(e - known["ccsd"]) < known["tolerance"], (e, iters)
        s.close()


def test_h2o_split_precision_known_answer(h2o, tmp_path):
    """Split-BF16 contractions (every product routed to the tensor-core kernel) with the
    FP64 refinement near convergence reach the reference's CCSD energy."""
    res, h, mo, known = h2o
    path = tmp_path / "FCIDUMP"
    write_fcidump(path, h, mo, nelec=10, ecore=res.enuc)
    with A.Context(0) as ctx:
        ctx.set_split_routing("all")
        H, _ = ctx.hamiltonian_from_fcidump(path)
        s = ctx.solver(H, conv_tol=1e-10, max_iter=100, precision="split", refine_tol=1e-7)
        e, conv, iters = s.run()
        assert ctx.split_launches() > 0
        assert conv < 1e-10
        assert abs(e - known["ccsd"]) < known["tolerance"], (e, iters)
        s.close()
