"""Spin-orbital Hbar and Lambda-CCSD on the device against the CPU oracle and the
reference's known answers.

Hbar is the product CCSD::run hands on (ccsd.cxx:83-86): STTwoElectronOperator(H, T,
isHbar) (st2eoperator.hpp:59-130).  Lambda-CCSD is LambdaCCSD<U>::run / iterate
(lambdaccsd.cxx:27-133).  The oracle (oracle/lambda_ccsd.py) restates both over full
spin-orbital arrays; its Lambda energies are pinned to test/input.aq:24 (H2O/cc-pVDZ) and
:71 (CH2/cc-pVDZ triplet, UHF) on the CPU.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import aquarius_b200 as A
from oracle import ccsd_oracle as O
from oracle import lambda_ccsd as LC
from oracle import scf
from tests.helpers import write_full

pytestmark = pytest.mark.gpu

FIXTURE = json.loads((Path(__file__).parent / "golden" / "molecules.json").read_text())
# engine block -> the reference's TwoElectronOperator block name (oracle keys)
HBAR_KEYS = {"fAI": "ai", "fME": "ia", "fAE": "ab", "fMI": "ij", "VMNIJ": "ijkl", "VAMIJ": "aijk",
             "VMNEJ": "ijak", "VABIJ": "abij", "VMNEF": "ijab", "VAMEI": "aibj", "VAMEF": "aibc",
             "VABEJ": "abci", "VABEF": "abcd"}
BASE_BLOCKS = ["fAI", "fME", "fAE", "fMI", "VMNIJ", "VAMIJ", "VMNEF", "VAMEI", "VAMEF", "VABEF"]


def _converged(ctx, o, v, seed, nirrep):
    eps, B, occ, vrt, aux = A.synth_problem(seed, o, v, nirrep=nirrep)
    ctx.set_spaces(vrt=vrt, occ=occ)
    H = ctx.hamiltonian_from_factor(B, eps, aux_per_irrep=aux if nirrep > 1 else None, pack_vvvv=False)
    s = ctx.solver(H, conv_tol=1e-11, max_iter=100, diis_order=8)
    _, c, _ = s.run()
    assert c < 1e-11
    return s, O.hamiltonian_from_factor(B, eps, o, ladder_literal=True)


@pytest.mark.parametrize("nirrep", [1, 4])
def test_hbar_blocks_match_oracle(nirrep):
    """All 13 blocks, from the engine's converged T, against the oracle's Hbar of that T."""
    o, v = (3, 8) if nirrep == 1 else (6, 16)
    with A.Context(0) as ctx:
        s, Href = _converged(ctx, o, v, 21, nirrep)
        want = LC.hbar(Href, s.T1.to_full(), s.T2.to_full())
        hb = s.hbar()
        for name, key in HBAR_KEYS.items():
            got, w = hb[name].to_full(), want[key]
            assert got.shape == w.shape, name
            assert np.abs(got - w).max() <= 1e-11 * max(1.0, np.abs(w).max()), (name, np.abs(got - w).max())
        # formed again from the same amplitudes: the same blocks
        again = s.hbar()
        assert np.array_equal(again["VABEF"].to_full(), hb["VABEF"].to_full())
        s.close()


@pytest.mark.parametrize("nirrep,graph", [(1, False), (1, True), (4, False)])
def test_lambda_matches_oracle_every_iteration(nirrep, graph):
    o, v = (3, 8) if nirrep == 1 else (6, 16)
    with A.Context(0) as ctx:
        s, Href = _converged(ctx, o, v, 22, nirrep)
        T1, T2 = s.T1.to_full(), s.T2.to_full()
        ref = LC.LambdaCCSD(LC.hbar(Href, T1, T2), T1, T2, diis_order=8)
        lam = s.lambda_solver(diis_order=8, use_graph=graph)
        # L(1)[ia] = T(1)[ai], L(2)[ijab] = T(2)[abij]
        assert np.array_equal(lam.L1.to_full(), T1.T)
        assert np.array_equal(lam.L2.to_full(), T2.transpose(2, 3, 0, 1))
        for it in range(10):
            e_ref, c_ref = ref.iterate()
            e, c = lam.iterate()
            assert abs(e - e_ref) < 1e-11, (it, e, e_ref)
            assert abs(c - c_ref) <= 1e-9 * max(1e-3, c_ref), (it, c, c_ref)
        assert np.abs(lam.L1.to_full() - ref.L.T1).max() < 1e-10
        assert np.abs(lam.L2.to_full() - ref.L.T2).max() < 1e-10
        lam.close()
        s.close()


def test_lambda_lifetime_and_packed_errors():
    with A.Context(0) as ctx:
        eps, B, occ, vrt, _ = A.synth_problem(5, 3, 8)
        ctx.set_spaces(vrt=vrt, occ=occ)
        Hp = ctx.hamiltonian_from_factor(B, eps, pack_vvvv=True)
        sp = ctx.solver(Hp)
        with pytest.raises(A.CcsdError) as e:
            sp.hbar()
        assert e.value.code == 9          # packed <ab||ef>: CCSD_ERR_UNSUPPORTED
        sp.close()
        Hp.destroy()
        H = ctx.hamiltonian_from_factor(B, eps, pack_vvvv=False)
        s = ctx.solver(H)
        s.iterate()
        lam = s.lambda_solver()
        with pytest.raises(A.CcsdError):
            s.close()                      # the Lambda solver still reads T and Hbar
        with pytest.raises(A.CcsdError):
            s.hbar()                       # Hbar is in use
        lam.iterate()
        lam.close()
        s.close()


def test_lambda_h2o_known_answer():
    """H2O/cc-pVDZ: CCSD, Hbar and Lambda on the device reach the reference's Lambda
    energy (test/input.aq:24) to its 1e-9 Eh tolerance."""
    res, Hao, eri = scf.solve_scf(FIXTURE, "h2o-pvdz")
    h, mo = scf.mo_integrals(res, Hao, eri)
    known = FIXTURE["molecules"]["h2o-pvdz"]["known"]
    no, n = 5, h.shape[0]
    fock = h + 2 * np.einsum("pqii->pq", mo[:, :, :no, :no]) - np.einsum("piiq->pq", mo[:, :no, :no, :])
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=[n - no], occ=[no])
        H = ctx.hamiltonian_from_integrals(fock, mo, pack_vvvv=False)
        s = ctx.solver(H, conv_tol=1e-11, max_iter=100, diis_order=5)
        e, c, _ = s.run()
        assert c < 1e-11 and abs(e - known["ccsd"]) < known["tolerance"]
        lam = s.lambda_solver(conv_tol=1e-11, max_iter=100, diis_order=5)
        el, cl, it = lam.run()
        assert cl < 1e-11
        assert abs(el - known["lambda"]) < known["tolerance"], (el, it)
        lam.close()
        s.close()


def test_lambda_ch2_uhf_known_answer():
    """CH2 triplet (UHF, alpha and beta spaces differ): the reference's Lambda energy
    (test/input.aq:71)."""
    res, Hao, eri = scf.solve_scf(FIXTURE, "ch2-pvdz")
    Hso = scf.SpinOrbitalHamiltonian(res, Hao, eri)
    known = FIXTURE["molecules"]["ch2-pvdz"]["known"]
    (na, nb), (va, vb) = Hso.nocc, Hso.nvrt
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=[va], occ=[na], vrt_beta=[vb], occ_beta=[nb])
        H = ctx.hamiltonian(pack_vvvv=False)
        for name in BASE_BLOCKS:
            write_full(H[name], getattr(Hso, name))
        s = ctx.solver(H, conv_tol=1e-11, max_iter=100, diis_order=5)
        e, c, _ = s.run()
        assert c < 1e-11 and abs(e - known["ccsd"]) < known["tolerance"]
        lam = s.lambda_solver(conv_tol=1e-11, max_iter=100, diis_order=5)
        el, cl, it = lam.run()
        assert cl < 1e-11
        assert abs(el - known["lambda"]) < known["tolerance"], (el, it)
        lam.close()
        s.close()
