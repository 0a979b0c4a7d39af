"""Split (BF16 and INT8 slice) tcgen05 contractions against the native-FP64 path and the oracle.

Tolerances: a single contraction agrees with FP64 to 2e-6 of max|C| with three BF16 slices
per operand (8 bits each, the leading product exact, errors unbiased), 1e-8 with four;
INT8 slices carry 7 bits each (3e-5, 3e-7, 3e-9 for three, four, five).  A full CCSD solve
agrees with the FP64 oracle to |dE| <= 1e-8 Eh and max|dT| <= 1e-7 at every iteration with
three BF16 or four INT8 slices.
"""
import numpy as np
import pytest

import aquarius_b200 as A
from oracle import ccsd_oracle as O
from tests.helpers import random_so, write_full

pytestmark = pytest.mark.gpu

SHAPES = {"abij": ((2, 0), (0, 2)), "abef": ((2, 0), (2, 0)), "amei": ((1, 1), (1, 1)), "mnef": ((0, 2), (2, 0))}


def _contract(precision, o, v, ia, sa, ib, sb, ic, sc, seed, packed_a=False, slices=0):
    rng = np.random.default_rng(seed)
    ctx = A.Context(0)
    try:
        ctx.set_spaces(vrt=[v], occ=[o])
        if precision != "fp64":
            ctx.set_precision(precision, slices=slices)
            ctx.set_split_routing("all")   # these sizes would stay on FP64 otherwise
        tA = ctx.tensor("A", *SHAPES[sa], packed=packed_a)
        tB = ctx.tensor("B", *SHAPES[sb])
        tC = ctx.tensor("C", *SHAPES[sc])
        write_full(tA, random_so(ctx, *SHAPES[sa], rng, scale=0.05))
        write_full(tB, random_so(ctx, *SHAPES[sb], rng, scale=0.01))
        ctx.contract(0.5, tA, ia, tB, ib, 0.0, tC, ic)
        if precision != "fp64":
            assert ctx.split_launches() > 0
        else:
            assert ctx.split_launches() == 0
        return tC.to_full()
    finally:
        ctx.close()


@pytest.mark.parametrize("case", [
    ("abef", "abef", "abij", "efij", "abij", "abij", True),     # particle ladder
    ("amei", "amei", "abij", "ebjm", "abij", "abij", False),    # ring with antisymmetriser images
    ("mnef", "mnef", "abij", "afni", "amei", "amei", False),    # W(am,ei) build
], ids=["ladder", "ring", "wamei"])
@pytest.mark.parametrize("precision,slices,tol", [
    ("split", 3, 2e-6), ("split", 4, 1e-8), ("split_i8", 3, 3e-5), ("split_i8", 4, 3e-7), ("split_i8", 5, 3e-9),
], ids=["bf16x3", "bf16x4", "i8x3", "i8x4", "i8x5"])
def test_split_contraction_matches_fp64(case, precision, slices, tol):
    """BF16: three slices 2e-6 of max|C| (FP32-like inputs), four 1e-8 (2^-8 finer);
    INT8: 7 bits per slice."""
    sa, ia, sb, ib, sc, ic, packed = case
    o, v = 6, 40
    ref = _contract("fp64", o, v, ia, sa, ib, sb, ic, sc, 11, packed)
    got = _contract(precision, o, v, ia, sa, ib, sb, ic, sc, 11, packed, slices=slices)
    scale = np.abs(ref).max()
    assert scale > 0
    assert np.abs(got - ref).max() <= tol * scale


@pytest.mark.parametrize("precision,slices,etol,ttol", [
    ("split", 3, 1e-8, 1e-7), ("split", 4, 1e-10, 1e-9), ("split_i8", 3, 2e-7, 2e-6), ("split_i8", 4, 1e-8, 1e-7),
    ("split_i8", 5, 1e-10, 1e-9),
], ids=["bf16x3", "bf16x4", "i8x3", "i8x4", "i8x5"])
@pytest.mark.parametrize("o,v,seed", [(4, 40, 21), (6, 48, 22)])
def test_split_solve_matches_oracle_every_iteration(o, v, seed, precision, slices, etol, ttol):
    eps, B, *_ = A.synth_problem(seed, o, v)
    ref = O.CCSD(O.hamiltonian_from_factor(B, eps, o), diis_order=8)
    ctx = A.Context(0)
    try:
        ctx.set_spaces(vrt=[v], occ=[o])
        ctx.set_split_routing("all")
        H = ctx.hamiltonian_from_factor(B, eps)
        s = ctx.solver(H, diis_order=8, precision=precision, slices=slices)
        for it in range(10):
            e_ref, _ = ref.iterate()
            e, _ = s.iterate()
            assert abs(e - e_ref) <= etol, (it, e, e_ref)
        assert ctx.split_launches() > 0
        assert np.abs(s.T2.to_full() - ref.T.T2).max() <= ttol
        assert np.abs(s.T1.to_full() - ref.T.T1).max() <= ttol
        s.close()
    finally:
        ctx.close()


@pytest.mark.parametrize("precision", ["split", "split_i8"])
def test_refinement_moves_to_four_slices_and_converges(precision):
    """refine_tol: 3-slice contractions until conv < refine_tol, then 4 slices (and 5 INT8
    slices on a stall); the solve reaches conv_tol and the oracle's converged energy."""
    o, v, seed = 4, 40, 23
    eps, B, *_ = A.synth_problem(seed, o, v)
    ref = O.CCSD(O.hamiltonian_from_factor(B, eps, o), diis_order=8)
    e_ref = ref.run(1e-10, 80)
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=[v], occ=[o])
        ctx.set_split_routing("all")
        H = ctx.hamiltonian_from_factor(B, eps)
        s = ctx.solver(H, diis_order=8, precision=precision, conv_tol=1e-10, max_iter=80, refine_tol=1e-6)
        e, c, it = s.run()
        assert c < 1e-10
        assert abs(e - e_ref) < 1e-10, (e, e_ref)
        s.close()
