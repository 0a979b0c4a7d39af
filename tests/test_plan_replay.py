"""The planner's expansion of every statement of the CCSD iteration (ccsd.cxx:123-180), the
spin-orbital Hbar (st2eoperator.hpp:59-130) and the Lambda-CCSD iteration
(lambdaccsd.cxx:80-124), replayed on the CPU.

Each statement is planned on a planning-only context, exported (ccsd_ctx_plan_export) and
executed with numpy over the engine's block layout (tests/plan_replay.py); the result is
compared with the interface semantics restated over full spin-orbital arrays: implicit
antisymmetrisation, spin cases, irrep blocks, lazy beta (tests/helpers.py).  The same
statements run on the device in tests/test_gpu_planner.py and the solvers' GPU tests.
"""
import numpy as np
import pytest

import aquarius_b200 as A
from tests import plan_replay as R
from tests.helpers import beta_mask, random_so, reference_contract

SHAPES = {
    "ai": ((1, 0), (0, 1)), "me": ((0, 1), (1, 0)), "ae": ((1, 0), (1, 0)), "mi": ((0, 1), (0, 1)),
    "abij": ((2, 0), (0, 2)), "mnef": ((0, 2), (2, 0)), "amef": ((1, 1), (2, 0)), "abej": ((2, 0), (1, 1)),
    "abef": ((2, 0), (2, 0)), "mnij": ((0, 2), (0, 2)), "mnej": ((0, 2), (1, 1)), "amij": ((1, 1), (0, 2)),
    "amei": ((1, 1), (1, 1)),
}
# (C shape, idxC, A shape, idxA, B shape, idxB)
CCSD = [
    ("abij", "abij", "ai", "ai", "ai", "bj"), ("me", "me", "mnef", "mnef", "ai", "fn"),
    ("mi", "mi", "mnef", "mnef", "abij", "efin"), ("mi", "mi", "me", "me", "ai", "ei"),
    ("mi", "mi", "mnej", "nmfi", "ai", "fn"), ("ae", "ae", "mnef", "mnef", "abij", "afmn"),
    ("ae", "ae", "me", "me", "ai", "am"), ("ae", "ae", "amef", "amef", "ai", "fm"),
    ("mnij", "mnij", "mnef", "mnef", "abij", "efij"), ("mnij", "mnij", "mnej", "mnej", "ai", "ei"),
    ("mnej", "mnej", "mnef", "mnef", "ai", "fj"), ("amij", "amij", "amef", "amef", "abij", "efij"),
    ("amij", "amij", "amei", "amej", "ai", "ei"), ("amei", "amei", "mnef", "mnef", "abij", "afni"),
    ("amei", "amei", "amef", "amef", "ai", "fi"), ("amei", "amei", "mnej", "nmei", "ai", "an"),
    ("ai", "ai", "ae", "ae", "ai", "ei"), ("ai", "ai", "mi", "mi", "ai", "am"),
    ("ai", "ai", "amei", "amei", "ai", "em"), ("ai", "ai", "me", "me", "abij", "aeim"),
    ("ai", "ai", "amef", "amef", "abij", "efim"), ("ai", "ai", "mnej", "mnei", "abij", "eamn"),
    ("abij", "abij", "abej", "abej", "ai", "ei"), ("abij", "abij", "amij", "amij", "ai", "bm"),
    ("abij", "abij", "ae", "ae", "abij", "ebij"), ("abij", "abij", "mi", "mi", "abij", "abmj"),
    ("abij", "abij", "abef", "abef", "abij", "efij"), ("abij", "abij", "mnij", "mnij", "abij", "abmn"),
    ("abij", "abij", "amei", "amei", "abij", "ebjm"),
]
# STTwoElectronOperator(H, T, isHbar), in the reference's order
HBAR = [
    ("me", "me", "mnef", "mnef", "ai", "fn"), ("mi", "mi", "mnef", "nmef", "abij", "efni"),
    ("mi", "mi", "me", "me", "ai", "ei"), ("mi", "mi", "mnej", "nmfi", "ai", "fn"),
    ("mnij", "mnij", "mnef", "mnef", "abij", "efij"), ("mnij", "mnij", "mnej", "nmei", "ai", "ej"),
    ("mnej", "mnej", "mnef", "mnef", "ai", "fj"), ("ae", "ae", "mnef", "mnfe", "abij", "famn"),
    ("ae", "ae", "me", "me", "ai", "am"), ("ae", "ae", "amef", "anef", "ai", "fn"),
    ("amij", "amij", "amef", "amef", "abij", "efij"), ("amij", "amij", "amei", "amej", "ai", "ei"),
    ("amei", "amei", "mnef", "mnef", "abij", "afin"), ("amei", "amei", "amef", "amfe", "ai", "fi"),
    ("amei", "amei", "mnej", "nmei", "ai", "an"), ("amij", "amij", "mnej", "nmej", "abij", "aein"),
    ("amij", "amij", "mnij", "nmij", "ai", "an"), ("amij", "amij", "me", "me", "abij", "aeij"),
    ("abej", "abej", "mnej", "mnej", "abij", "abmn"), ("abej", "abej", "amei", "amej", "ai", "bm"),
    ("abej", "abej", "amef", "amef", "abij", "fbmj"), ("abej", "abej", "abef", "abef", "ai", "fj"),
    ("abej", "abej", "me", "me", "abij", "abmj"), ("abef", "abef", "mnef", "mnef", "abij", "abmn"),
    ("abef", "abef", "amef", "amef", "ai", "bm"), ("amef", "amef", "mnef", "nmef", "ai", "an"),
]
# LambdaCCSD::iterate: G(im), G(ea), Z(1)[ia], Z(2)[ijab]
LAMBDA = [
    ("mi", "mn", "abij", "efno", "mnef", "moef"), ("ae", "ef", "abij", "egmn", "mnef", "mnfg"),
    ("me", "ia", "ae", "ea", "me", "ie"), ("me", "ia", "mi", "im", "me", "ma"),
    ("me", "ia", "amei", "eiam", "me", "me"), ("me", "ia", "abej", "efam", "mnef", "imef"),
    ("me", "ia", "amij", "eimn", "mnef", "mnea"), ("me", "ia", "mnej", "inam", "mi", "mn"),
    ("me", "ia", "amef", "fiea", "ae", "ef"),
    ("mnef", "ijab", "me", "ia", "me", "jb"), ("mnef", "ijab", "amef", "ejab", "me", "ie"),
    ("mnef", "ijab", "mnej", "ijam", "me", "mb"), ("mnef", "ijab", "ae", "ea", "mnef", "ijeb"),
    ("mnef", "ijab", "mi", "im", "mnef", "mjab"), ("mnef", "ijab", "abef", "efab", "mnef", "ijef"),
    ("mnef", "ijab", "mnij", "ijmn", "mnef", "mnab"), ("mnef", "ijab", "amei", "eiam", "mnef", "mjbe"),
    ("mnef", "ijab", "mnef", "mjab", "mi", "im"), ("mnef", "ijab", "mnef", "ijeb", "ae", "ea"),
]
CASES = ([("ccsd",) + s for s in CCSD] + [("hbar",) + s for s in HBAR] + [("lambda",) + s for s in LAMBDA])
# <ab||ef> as an operand: packed in H (CCSD, where it is read through restricted pairs only)
# and unpacked in Hbar (whose statements also split its pairs); Lambda reads Hbar's
CASES = [c + (c[3] == "abef" and c[0] == "ccsd",) for c in CASES] + \
        [c + (True,) for c in CASES if c[3] == "abef" and c[0] == "lambda"]


def _ctx(nirrep):
    ctx = A.Context(-1)
    if nirrep == 1:
        ctx.set_spaces(vrt=[5], occ=[3])
    elif nirrep == 2:
        ctx.set_spaces(vrt=[3, 2], occ=[2, 1])
    else:
        # irrep 3 has no occupied orbital: blocks exist but are empty
        ctx.set_spaces(vrt=[2, 1, 2, 1], occ=[1, 1, 1, 0])
    return ctx


def _replay_one(ctx, tensors, fulls, path):
    dump = R.load(path)
    store = {}
    for h, t in dump.tensors.items():
        if not t.view_of:
            store[h] = R.to_storage(ctx, t, fulls[h])
    R.replay(dump, store)
    return dump, store


@pytest.mark.parametrize("nirrep", [1, 2, 4])
@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}:{c[2]}+={c[4]}*{c[6]}{'(packed)' if c[7] else ''}"
                                              for c in CASES])
def test_planned_statement_replays_to_reference(case, nirrep, tmp_path):
    _, cs, ic, as_, ia, bs, ib, packed = case
    rng = np.random.default_rng(abs(hash((nirrep,) + case)) % 2**32)
    with _ctx(nirrep) as ctx:
        tA = ctx.tensor("A", *SHAPES[as_], packed=packed)
        tB = ctx.tensor("B", *SHAPES[bs])
        tC = ctx.tensor("C", *SHAPES[cs])
        fa = random_so(ctx, *SHAPES[as_], rng)
        fb = random_so(ctx, *SHAPES[bs], rng)
        fc = random_so(ctx, *SHAPES[cs], rng)
        alpha, beta = 0.75, -1.25
        ctx.contract(alpha, tA, ia, tB, ib, beta, tC, ic)
        ctx.plan_export(tmp_path / "plan.txt")
        dump, store = _replay_one(ctx, None, {tA.h: fa, tB.h: fb, tC.h: fc}, tmp_path / "plan.txt")
        ref = reference_contract(alpha, fa, ia, fb, ib, 1.0, fc, ic, tC.group)
        bm = beta_mask(ctx, (SHAPES[as_], SHAPES[bs], SHAPES[cs]), ia, ib, ic)
        ref = ref + np.where(bm, (beta - 1.0) * fc, 0.0)
        want = R.to_storage(ctx, dump.tensors[tC.h], ref)
        got = store[tC.h]
        assert np.abs(got - want).max() < 1e-13 * max(1.0, np.abs(want).max())
        assert not np.array_equal(got, R.to_storage(ctx, dump.tensors[tC.h], fc))   # the statement did something


@pytest.mark.parametrize("nirrep", [1, 4])
@pytest.mark.parametrize("sh", [("me", "ia", "ai", "ai"), ("mnef", "ijab", "abij", "abij"),
                                ("abij", "abij", "abij", "baji")])
def test_planned_sum_replays_to_reference(sh, nirrep, tmp_path):
    """The Lambda initial guess L(1)[ia] = T(1)[ai], L(2)[ijab] = T(2)[abij] moves lines
    between upper and lower groups; a relabelled sum keeps the values of every element."""
    cs, ic, as_, ia = sh
    rng = np.random.default_rng(7 + nirrep)
    with _ctx(nirrep) as ctx:
        tA = ctx.tensor("A", *SHAPES[as_])
        tC = ctx.tensor("C", *SHAPES[cs])
        fa = random_so(ctx, *SHAPES[as_], rng)
        fc = random_so(ctx, *SHAPES[cs], rng)
        ctx.sum(0.5, tA, ia, 2.0, tC, ic)
        ctx.plan_export(tmp_path / "plan.txt")
        dump, store = _replay_one(ctx, None, {tA.h: fa, tC.h: fc}, tmp_path / "plan.txt")
        ref = 2.0 * fc + 0.5 * np.einsum(f"{ia}->{ic}", fa)
        want = R.to_storage(ctx, dump.tensors[tC.h], ref)
        assert np.abs(store[tC.h] - want).max() < 1e-14


def test_export_without_a_statement_is_an_error(tmp_path):
    with _ctx(1) as ctx:
        with pytest.raises(A.CcsdError):
            ctx.plan_export(tmp_path / "plan.txt")
