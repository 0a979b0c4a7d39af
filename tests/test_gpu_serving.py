"""The serving loop (ccsd_server_*): continuous batching with admission by device bytes.

A request's result is the same alone and in a mix of concurrent solves (its kernels and
reductions do not depend on the others), the mix really overlaps on the device, the
admitted bytes never exceed the budget, and a request larger than the budget is refused.
"""
import numpy as np
import pytest

import aquarius_b200 as A

pytestmark = pytest.mark.gpu

MIX = [(4, 24, 1, 11), (5, 30, 2, 12), (6, 36, 1, 13), (4, 20, 4, 14), (4, 28, 1, 15), (8, 26, 8, 16)]


def _serve(reqs, **kw):
    with A.Server(0, conv_tol=1e-10, max_iter=100, **kw) as srv:
        ids = {srv.submit_synthetic(o, v, nirrep=h, seed=s): (o, v, h, s) for o, v, h, s in reqs}
        srv.wait(600)
        res = {ids[r["id"]]: r for r in srv.poll()}
        return res, srv.stats()


def test_result_alone_equals_result_in_mix():
    mixed, st = _serve(MIX, max_active=8)
    assert st["peak_active"] >= 2
    for key in MIX:
        alone, _ = _serve([key], max_active=1)
        a, m = alone[key], mixed[key]
        assert a["status"] == 0 and m["status"] == 0
        assert a["iterations"] == m["iterations"]
        assert abs(a["energy"] - m["energy"]) <= 1e-12, (key, a["energy"], m["energy"])
        assert a["conv"] < 1e-10


# large enough that natural routing puts the particle ladder and other big products on the
# tcgen05 split kernel (o=12 v=96: ladder blocks M = K = v^2, N = o^2)
MIX_SPLIT = [(12, 96, 1, 21), (4, 24, 1, 11), (10, 70, 1, 22), (8, 26, 8, 16), (6, 36, 1, 13)]


def test_split_graph_result_alone_equals_result_in_mix():
    """The precision the benchmark serves with: INT8 split slices with the 3 -> 4 slice
    refinement, every iteration replayed as a CUDA graph."""
    kw = dict(precision="split_i8", refine_tol=1e-5, use_graph=True)
    mixed, st = _serve(MIX_SPLIT, max_active=8, **kw)
    assert st["peak_active"] >= 2
    for key in MIX_SPLIT:
        alone, _ = _serve([key], max_active=1, **kw)
        a, m = alone[key], mixed[key]
        assert a["status"] == 0 and m["status"] == 0, (key, a["message"], m["message"])
        assert a["iterations"] == m["iterations"]
        assert abs(a["energy"] - m["energy"]) <= 1e-12, (key, a["energy"], m["energy"])
        assert a["conv"] < 1e-10


def test_served_solve_matches_direct_solver():
    o, v, h, s = MIX[1]
    res, _ = _serve([MIX[1]], max_active=1)
    eps, B, occ, vrt, aux = A.synth_problem(s, o, v, nirrep=h)
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=vrt, occ=occ)
        H = ctx.hamiltonian_from_factor(B, eps, aux_per_irrep=aux)
        sol = ctx.solver(H, conv_tol=1e-10, max_iter=100, diis_order=8)
        e, c, it = sol.run()
        assert res[MIX[1]]["iterations"] == it
        assert abs(res[MIX[1]]["energy"] - e) <= 1e-12
        assert abs(res[MIX[1]]["mp2"] - sol.mp2) <= 1e-12
        sol.close()


def test_admission_respects_the_memory_budget():
    need = []
    for o, v, h, s in MIX:
        occ, vrt, _ = A.synth_irreps(s, h, o, v)
        need.append(A.plan_query(vrt, occ, diis_order=8)[1])
    budget = int(max(need) * 1.5)
    res, st = _serve(MIX, max_active=8, memory_budget=budget)
    assert all(r["status"] == 0 for r in res.values())
    assert st["peak_bytes"] <= budget
    assert st["peak_bytes"] >= max(need)
    # a solve is never admitted before its predecessor in arrival order
    order = sorted(res.values(), key=lambda r: r["id"])
    assert all(a["t_admit"] <= b["t_admit"] for a, b in zip(order, order[1:]))


def test_request_larger_than_the_budget_is_refused():
    res, _ = _serve([(6, 36, 1, 13)], max_active=2, memory_budget=1 << 20)
    r = res[(6, 36, 1, 13)]
    assert r["status"] == 3   # CCSD_ERR_OOM
