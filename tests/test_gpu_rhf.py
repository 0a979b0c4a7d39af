"""Closed-shell spin-adapted CCSD (RHFCCSD, src/cc/rhfccsd.cxx) on the device.

The engine's plain-tensor path against the spatial-orbital oracle (oracle/rhf_ccsd.py)
iteration by iteration, against the spin-orbital engine on the same problem, and
against the reference's H2O/cc-pVDZ known answers (test/input.aq:1-24).
"""
import json
from pathlib import Path

import numpy as np
import pytest

import aquarius_b200 as A
from oracle import rhf_ccsd as R
from oracle import scf

pytestmark = pytest.mark.gpu

FIXTURE = json.loads((Path(__file__).parent / "golden" / "molecules.json").read_text())


def _factor_problem(seed, o, v, nirrep):
    eps, B, occ, vrt, aux = A.synth_problem(seed, o, v, nirrep=nirrep)
    eri = np.einsum("Ppq,Prs->pqrs", B, B, optimize=True)
    return eps, B, occ, vrt, aux, eri


def _run_pair(o, v, seed, nirrep=1, iters=10, diis_order=8, precision="fp64", use_graph=False):
    eps, B, occ, vrt, aux, eri = _factor_problem(seed, o, v, nirrep)
    ref = R.RHFCCSD(np.diag(eps), eri, o, diis_order=diis_order)
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=vrt, occ=occ)
        H = ctx.rhf_hamiltonian_from_factor(B, eps, aux_per_irrep=aux if nirrep > 1 else None)
        s = ctx.solver(H, diis_order=diis_order, precision=precision, use_graph=use_graph)
        assert abs(s.mp2 - ref.mp2) < 1e-12 * max(1.0, abs(ref.mp2)), (s.mp2, ref.mp2)
        worst_e = 0.0
        for it in range(iters):
            e_ref, c_ref = ref.iterate()
            e, c = s.iterate()
            worst_e = max(worst_e, abs(e - e_ref))
            assert abs(c - c_ref) <= 1e-9 * max(1e-3, c_ref), (it, c, c_ref)
        dT1 = np.abs(s.T1.to_full() - ref.T1).max()
        dT2 = np.abs(s.T2.to_full() - ref.T2).max()
        s.close()
        H.destroy()
    return worst_e, dT1, dT2


@pytest.mark.parametrize("o,v,seed", [(3, 7, 1), (4, 10, 2), (5, 12, 3)])
def test_rhf_fp64_matches_oracle_every_iteration(o, v, seed):
    de, dt1, dt2 = _run_pair(o, v, seed)
    assert de < 1e-11 and dt1 < 1e-11 and dt2 < 1e-11, (de, dt1, dt2)


@pytest.mark.parametrize("nirrep", [2, 4, 8])
def test_rhf_symmetry_blocked_matches_oracle(nirrep):
    de, dt1, dt2 = _run_pair(8, 20, 5, nirrep=nirrep, iters=8)
    assert de < 1e-11 and dt2 < 1e-11, (de, dt2)


def test_rhf_graph_replay_matches_oracle():
    de, dt1, dt2 = _run_pair(4, 10, 6, use_graph=True)
    assert de < 1e-11 and dt2 < 1e-11


def test_rhf_blocks_are_the_spatial_integrals():
    """<ab|cd> = (ac|bd) in every block; VAIJB keeps <ai|jb> at [a, i, b, j]."""
    o, v = 3, 6
    eps, B, occ, vrt, aux, eri = _factor_problem(11, o, v, 1)
    phys = eri.transpose(0, 2, 1, 3)
    Ox, Vx = slice(0, o), slice(o, o + v)
    want = {"VABCD": phys[Vx, Vx, Vx, Vx], "VABCI": phys[Vx, Vx, Vx, Ox], "VABIJ": phys[Vx, Vx, Ox, Ox],
            "VAIBJ": phys[Vx, Ox, Vx, Ox], "VAIJB": phys[Vx, Ox, Ox, Vx].transpose(0, 1, 3, 2),
            "VAIJK": phys[Vx, Ox, Ox, Ox], "VIJKL": phys[Ox, Ox, Ox, Ox],
            "fAB": np.diag(eps[o:]), "fIJ": np.diag(eps[:o]), "fAI": np.zeros((v, o))}
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=vrt, occ=occ)
        H = ctx.rhf_hamiltonian_from_factor(B, eps)
        for name, ref in want.items():
            got = H[name].to_full()
            assert got.shape == ref.shape, name
            assert np.abs(got - ref).max() < 1e-12, name
        H.destroy()


def test_rhf_energy_equals_spin_orbital_energy():
    """Both formulations converge to the same CCSD energy on one closed-shell problem."""
    o, v = 4, 12
    eps, B, occ, vrt, aux, eri = _factor_problem(9, o, v, 1)
    energies = {}
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=vrt, occ=occ)
        for kind in ("rhf", "spin-orbital"):
            H = ctx.rhf_hamiltonian_from_factor(B, eps) if kind == "rhf" else ctx.hamiltonian_from_factor(B, eps)
            s = ctx.solver(H, conv_tol=1e-11, max_iter=100, diis_order=8)
            e, c, it = s.run()
            assert c < 1e-11, (kind, c, it)
            energies[kind] = e
            s.close()
            H.destroy()
    assert abs(energies["rhf"] - energies["spin-orbital"]) < 1e-9, energies


def test_rhf_split_matches_fp64():
    """The split-BF16 contractions on the RHF statements (every product routed to the
    tcgen05 kernel) track the FP64 iteration to the split tolerance."""
    o, v = 8, 48
    eps, B, occ, vrt, aux, eri = _factor_problem(13, o, v, 1)
    res = {}
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=vrt, occ=occ)
        H = ctx.rhf_hamiltonian_from_factor(B, eps)
        for prec in ("fp64", "split"):
            if prec == "split":
                ctx.set_split_routing("all")
            n0 = ctx.split_launches()
            s = ctx.solver(H, diis_order=8, precision=prec)
            es = [s.iterate()[0] for _ in range(8)]
            res[prec] = (es, s.T2.to_full(), ctx.split_launches() - n0)
            s.close()
        H.destroy()
    assert res["fp64"][2] == 0 and res["split"][2] > 0
    de = max(abs(a - b) for a, b in zip(res["fp64"][0], res["split"][0]))
    dt2 = np.abs(res["fp64"][1] - res["split"][1]).max()
    assert de < 1e-8 * max(1.0, abs(res["fp64"][0][-1])), de
    assert dt2 < 1e-7, dt2


def test_rhf_h2o_known_answers():
    """H2O/cc-pVDZ through the dense-integral RHF builder: the reference's SCF, MP2 and
    CCSD energies (test/input.aq:1-24) to its 1e-9 Eh tolerance."""
    res, Hao, eri_ao = scf.solve_scf(FIXTURE, "h2o-pvdz")
    h, mo = scf.mo_integrals(res, Hao, eri_ao)
    known = FIXTURE["molecules"]["h2o-pvdz"]["known"]
    n, no = h.shape[0], 5
    J = np.einsum("pqii->pq", mo[:, :, :no, :no])
    K = np.einsum("piiq->pq", mo[:, :no, :no, :])
    fock = h + 2 * J - K
    escf = res.enuc + sum(h[i, i] + fock[i, i] for i in range(no))
    assert abs(escf - known["scf"]) < known["tolerance"]
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=[n - no], occ=[no])
        H = ctx.rhf_hamiltonian_from_integrals(fock, mo)
        s = ctx.solver(H, conv_tol=1e-11, max_iter=100, diis_order=5)
        assert abs(s.mp2 - known["mp2"]) < known["tolerance"], s.mp2
        e, conv, iters = s.run()
        assert conv < 1e-11
        assert abs(e - known["ccsd"]) < known["tolerance"], (e, iters)
        s.close()
        H.destroy()


@pytest.mark.parametrize("nirrep", [1, 4])
def test_rhf_hbar_matches_oracle(nirrep):
    """The closed-shell Hbar intermediates (rhfccsd.cxx:110-186) after a converged solve."""
    o, v = (4, 12) if nirrep == 1 else (8, 20)
    eps, B, occ, vrt, aux, eri = _factor_problem(17, o, v, nirrep)
    ref = R.RHFCCSD(np.diag(eps), eri, o, diis_order=8)
    ref.run(1e-11, 100)
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=vrt, occ=occ)
        H = ctx.rhf_hamiltonian_from_factor(B, eps, aux_per_irrep=aux if nirrep > 1 else None)
        s = ctx.solver(H, diis_order=8, conv_tol=1e-11, max_iter=100)
        e, c, it = s.run()
        assert c < 1e-11 and abs(e - ref.energy) < 1e-10
        got = s.hbar()
        want = ref.hbar()
        want["WAMIE"] = want["WAMIE"].transpose(0, 1, 3, 2)   # engine order [a, m, e, i]
        for name, w in want.items():
            g = got[name].to_full()
            assert g.shape == w.shape, name
            assert np.abs(g - w).max() < 1e-9 * max(1.0, np.abs(w).max()), (name, np.abs(g - w).max())
        s.close()
        H.destroy()
