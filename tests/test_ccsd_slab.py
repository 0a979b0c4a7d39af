"""The CPU baseline's bounded sample (oracle/ccsd_slab.py) does the oracle's own work.

Every statement evaluated on a slab of rows must equal those rows of the oracle's
statement (ccsd_oracle.CCSD.residual, restating src/cc/ccsd.cxx:123-180), on the same
amplitudes; with every row in the slab the sample reproduces the whole residual.
The inputs come from oracle/synth.py, so no engine library is loaded.
"""
import numpy as np
import pytest

from oracle import ccsd_oracle as O
from oracle import ccsd_slab as S
from oracle import synth

NAMES = ["FME", "FMI", "FAE", "WMNIJ", "WMNEJ", "WAMIJ", "WAMEI", "Z1", "Z2"]
OCC_FIRST = {"FME", "FMI", "WMNIJ", "WMNEJ"}


def _state(o, v, seed):
    eps, B, *_ = synth.synth_problem(seed, o, v)
    ref = O.CCSD(O.hamiltonian_from_factor(B, eps, o), diis_order=8)
    ref.iterate()
    ref.iterate()                       # amplitudes with T1 != 0 and a DIIS step behind them
    ref.keep_intermediates = True
    ref.residual(ref.T)
    return eps, B, ref


@pytest.mark.parametrize("o,v,seed,sv,so", [
    (3, 8, 1, [0, 5, 9, 15], [1, 4]),
    (4, 10, 2, [3], [0]),
    (4, 10, 2, [10, 11, 19], [2, 7]),
])
def test_slab_rows_equal_oracle_rows(o, v, seed, sv, so):
    eps, B, ref = _state(o, v, seed)
    I = ref.intermediates
    s = S.SlabIteration(B, eps, o, sv, so)
    s.prepare(ref.T.T1, ref.T.T2, I["Tau"], I)
    times, est = s.run()
    for name in NAMES:
        rows = s.so if name in OCC_FIRST else s.sv
        got, want = s.out[name], I[name][rows]
        assert got.shape == want.shape, name
        assert np.abs(got - want).max() <= 1e-13 * max(1.0, np.abs(want).max()), name
    # fractions: occupied-first rows, virtual-first rows, P(ab) terms twice
    assert times["FME"][1] == len(so) / (2 * o) and times["WAMEI"][1] == len(sv) / (2 * v)
    assert times["Z2 ring"][1] == 2 * len(sv) / (2 * v)
    assert est > 0


def test_all_rows_reproduce_the_residual():
    o, v = 3, 9
    eps, B, ref = _state(o, v, 3)
    I = ref.intermediates
    s = S.SlabIteration(B, eps, o, range(2 * v), range(2 * o))
    s.prepare(ref.T.T1, ref.T.T2, I["Tau"], I)
    s.run()
    assert np.abs(s.out["Z1"] - I["Z1"]).max() < 1e-13
    assert np.abs(s.out["Z2"] - I["Z2"]).max() < 1e-13


def test_slab_blocks_equal_oracle_blocks():
    o, v = 3, 7
    eps, B, *_ = synth.synth_problem(4, o, v)
    H = O.hamiltonian_from_factor(B, eps, o)
    Oi, Vi = np.arange(o), np.arange(o, o + v)
    rows = [1, 6, 8, 13]
    assert np.abs(S.so_block(B, (Vi, Oi, Vi, Vi), rows=rows) - H.VAMEF[rows]).max() < 1e-15
    assert np.abs(S.so_block(B, (Oi, Oi, Vi, Vi)) - H.VMNEF).max() < 1e-15


def test_timing_tail_runs_on_the_slab():
    o, v = 3, 8
    eps, B, *_ = synth.synth_problem(5, o, v)
    s = S.SlabIteration(B, eps, o, [2, 9], [0])
    ring = S.timing_inputs(s, seed=1, diis_order=8)
    times, est = s.run(ring)
    assert "update, energy, DIIS" in times
    assert est >= sum(t for t, _ in times.values())
