"""CCSD iteration on the device versus the CPU oracle, iteration by iteration."""
import numpy as np
import pytest

import aquarius_b200 as A
from oracle import ccsd_oracle as O

pytestmark = pytest.mark.gpu


def _run_pair(o, v, seed, nirrep=1, iters=12, diis_order=8, precision="fp64", use_graph=False, pack=True):
    eps, B, occ, vrt, aux = A.synth_problem(seed, o, v, nirrep=nirrep)
    ref = O.CCSD(O.hamiltonian_from_factor(B, eps, o), diis_order=diis_order)
    ctx = A.Context(0)
    try:
        ctx.set_spaces(vrt=vrt, occ=occ)
        H = ctx.hamiltonian_from_factor(B, eps, aux_per_irrep=aux if nirrep > 1 else None, pack_vvvv=pack)
        s = ctx.solver(H, diis_order=diis_order, precision=precision, use_graph=use_graph)
        assert abs(s.mp2 - ref.mp2) < 1e-12
        worst_e = 0.0
        for it in range(iters):
            e_ref, c_ref = ref.iterate()
            e, c = s.iterate()
            worst_e = max(worst_e, abs(e - e_ref))
            assert abs(c - c_ref) <= 1e-9 * max(1e-3, c_ref), (it, c, c_ref)
        dT2 = np.abs(s.T2.to_full() - ref.T.T2).max()
        dT1 = np.abs(s.T1.to_full() - ref.T.T1).max()
        s.close()
        return worst_e, dT1, dT2
    finally:
        ctx.close()


@pytest.mark.parametrize("o,v,seed", [(3, 7, 1), (4, 10, 2), (5, 12, 3)])
def test_c1_fp64_matches_oracle_every_iteration(o, v, seed):
    de, dt1, dt2 = _run_pair(o, v, seed)
    assert de < 1e-11 and dt1 < 1e-11 and dt2 < 1e-11


def test_unpacked_vvvv_matches_oracle():
    de, dt1, dt2 = _run_pair(3, 8, 4, pack=False)
    assert de < 1e-11 and dt2 < 1e-11


@pytest.mark.parametrize("grouped", [True, False], ids=["grouped", "one-launch-per-block"])
@pytest.mark.parametrize("nirrep", [2, 4, 8])
def test_symmetry_blocked_matches_oracle(nirrep, grouped, monkeypatch):
    """Symmetry-blocked statements run their small block contractions as grouped
    launches by default; CCSD_GROUP_GEMMS=0 launches each block on its own."""
    monkeypatch.setenv("CCSD_GROUP_GEMMS", "1" if grouped else "0")
    de, dt1, dt2 = _run_pair(8, 20, 5, nirrep=nirrep, iters=8)
    assert de < 1e-11 and dt2 < 1e-11


def test_grouped_launches_cut_the_launch_count(monkeypatch):
    counts = {}
    for grouped in (True, False):
        monkeypatch.setenv("CCSD_GROUP_GEMMS", "1" if grouped else "0")
        eps, B, occ, vrt, aux = A.synth_problem(5, 8, 20, nirrep=8)
        with A.Context(0) as ctx:
            ctx.set_spaces(vrt=vrt, occ=occ)
            H = ctx.hamiltonian_from_factor(B, eps, aux_per_irrep=aux)
            s = ctx.solver(H, diis_order=8)
            s.iterate()
            n0 = ctx.launch_count()
            s.iterate()
            counts[grouped] = ctx.launch_count() - n0
            s.close()
    assert counts[True] * 5 < counts[False], counts


def test_graph_replay_matches_eager():
    de, dt1, dt2 = _run_pair(4, 10, 6, use_graph=True)
    assert de < 1e-11 and dt2 < 1e-11


def test_converges_like_oracle():
    eps, B, *_ = A.synth_problem(9, 4, 12)
    ref = O.CCSD(O.hamiltonian_from_factor(B, eps, 4), diis_order=8)
    e_ref = ref.run(1e-10, 60)
    ctx = A.Context(0)
    try:
        ctx.set_spaces(vrt=[12], occ=[4])
        H = ctx.hamiltonian_from_factor(B, eps)
        s = ctx.solver(H, diis_order=8, conv_tol=1e-10, max_iter=60)
        e, c, n = s.run()
        assert c < 1e-10 and n == ref.iter
        assert abs(e - e_ref) < 1e-12
        s.close()
    finally:
        ctx.close()
