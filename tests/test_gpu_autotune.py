"""The slice autotuner on the device (ccsd_options.autotune_de).

At o=12 v=96 (C1, natural routing: the particle ladder, the ring terms and W(am,ij) on the
tcgen05 split kernel) a 4-slice INT8 solve tunes its slice count per statement on its
second iteration.  The chosen statements' measured energy changes add up to at most the
budget, and the solve still matches the oracle (src/cc/ccsd.cxx:91-193) at every iteration:
|dE| <= 1e-8 Eh, max|dT2| <= 1e-7."""
import numpy as np
import pytest

import aquarius_b200 as A
from oracle import ccsd_oracle as O

pytestmark = pytest.mark.gpu

O_, V_, SEED = 12, 96, 41


def _solve(budget, iters, ref=None):
    eps, B, *_ = A.synth_problem(SEED, O_, V_)
    rows = []
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=[V_], occ=[O_])
        H = ctx.hamiltonian_from_factor(B, eps)
        s = ctx.solver(H, diis_order=8, precision="split_i8", slices=4, autotune_de=budget)
        for _ in range(iters):
            e, _ = s.iterate()
            if ref is not None:
                e_ref, _ = ref.iterate()
                rows.append((abs(e - e_ref), float(np.abs(s.T2.to_full() - ref.T.T2).max())))
        report = s.slice_report()
        s.close()
        H.destroy()
    return report, rows


def test_tuned_solve_matches_oracle_every_iteration():
    eps, B, *_ = A.synth_problem(SEED, O_, V_)
    ref = O.CCSD(O.hamiltonian_from_factor(B, eps, O_), diis_order=8)
    budget = 1e-9
    report, rows = _solve(budget, 8, ref)
    assert len(report) >= 3
    assert all(ns in (3, 4) for ns, _, _ in report)
    dropped = [abs(de) for ns, de, _ in report if ns == 3]
    assert sum(dropped) <= budget
    assert any(de != 0.0 for _, de, _ in report)          # the trials ran
    for it, (de, dt2) in enumerate(rows):
        assert de <= 1e-8 and dt2 <= 1e-7, (it, de, dt2)


def test_budget_bounds_the_choice():
    report_all, _ = _solve(1.0, 3)
    assert all(ns == 3 for ns, _, _ in report_all)
    report_none, _ = _solve(1e-300, 3)
    assert all(ns == 4 or de == 0.0 for ns, de, _ in report_none)
    report_off, _ = _solve(0.0, 3)
    assert all(ns == 4 and de == 0.0 for ns, de, _ in report_off)
