"""Indexed-tensor statements through the C ABI versus the reference semantics restated in
numpy over full spin-orbital arrays (implicit antisymmetrisation, spin cases, irrep blocks)."""
import numpy as np
import pytest

import aquarius_b200 as A
from tests.helpers import beta_mask, random_so, reference_contract, write_full

pytestmark = pytest.mark.gpu

# (C shape, idxC, A shape, idxA, B shape, idxB) -- every contraction pattern of ccsd.cxx:123-180
SHAPES = {
    "ai": ((1, 0), (0, 1)), "me": ((0, 1), (1, 0)), "ae": ((1, 0), (1, 0)), "mi": ((0, 1), (0, 1)),
    "abij": ((2, 0), (0, 2)), "mnef": ((0, 2), (2, 0)), "amef": ((1, 1), (2, 0)), "abej": ((2, 0), (1, 1)),
    "abef": ((2, 0), (2, 0)), "mnij": ((0, 2), (0, 2)), "mnej": ((0, 2), (1, 1)), "amij": ((1, 1), (0, 2)),
    "amei": ((1, 1), (1, 1)),
}
STATEMENTS = [
    ("abij", "abij", "ai", "ai", "ai", "bj"),        # Tau += 1/2 P(ab)P(ij) t t
    ("me", "me", "mnef", "mnef", "ai", "fn"),
    ("mi", "mi", "mnef", "mnef", "abij", "efin"),
    ("mi", "mi", "me", "me", "ai", "ei"),
    ("mi", "mi", "mnej", "nmfi", "ai", "fn"),
    ("ae", "ae", "mnef", "mnef", "abij", "afmn"),
    ("ae", "ae", "me", "me", "ai", "am"),
    ("ae", "ae", "amef", "amef", "ai", "fm"),
    ("mnij", "mnij", "mnef", "mnef", "abij", "efij"),
    ("mnij", "mnij", "mnej", "mnej", "ai", "ei"),
    ("mnej", "mnej", "mnef", "mnef", "ai", "fj"),
    ("amij", "amij", "amef", "amef", "abij", "efij"),
    ("amij", "amij", "amei", "amej", "ai", "ei"),
    ("amei", "amei", "mnef", "mnef", "abij", "afni"),
    ("amei", "amei", "amef", "amef", "ai", "fi"),
    ("amei", "amei", "mnej", "nmei", "ai", "an"),
    ("ai", "ai", "ae", "ae", "ai", "ei"),
    ("ai", "ai", "mi", "mi", "ai", "am"),
    ("ai", "ai", "amei", "amei", "ai", "em"),
    ("ai", "ai", "me", "me", "abij", "aeim"),
    ("ai", "ai", "amef", "amef", "abij", "efim"),
    ("ai", "ai", "mnej", "mnei", "abij", "eamn"),
    ("abij", "abij", "abej", "abej", "ai", "ei"),
    ("abij", "abij", "amij", "amij", "ai", "bm"),
    ("abij", "abij", "ae", "ae", "abij", "ebij"),
    ("abij", "abij", "mi", "mi", "abij", "abmj"),
    ("abij", "abij", "abef", "abef", "abij", "efij"),
    ("abij", "abij", "mnij", "mnij", "abij", "abmn"),
    ("abij", "abij", "amei", "amei", "abij", "ebjm"),
]


def _ctx(nirrep):
    ctx = A.Context(0)
    if nirrep == 1:
        ctx.set_spaces(vrt=[5], occ=[3])
    else:
        # irrep 3 has no occupied orbital: blocks exist but are empty
        ctx.set_spaces(vrt=[2, 1, 2, 1] if nirrep == 4 else [3, 2], occ=[1, 1, 1, 0] if nirrep == 4 else [2, 1])
    return ctx


@pytest.mark.parametrize("path", ["auto", "tiled"])
@pytest.mark.parametrize("nirrep", [1, 2, 4])
@pytest.mark.parametrize("stmt", STATEMENTS, ids=[f"{s[1]}+={s[3]}*{s[5]}" for s in STATEMENTS])
def test_statement_matches_reference(nirrep, stmt, path, monkeypatch):
    """At these sizes every product has an extent <= 32, so "auto" runs the skinny FP64
    kernel and "tiled" (CCSD_FP64_TILED=1) the 128x64 DMMA kernel."""
    monkeypatch.setenv("CCSD_FP64_TILED", "1" if path == "tiled" else "0")
    cs, ic, as_, ia, bs, ib = stmt
    rng = np.random.default_rng(abs(hash((nirrep,) + stmt)) % 2**32)
    ctx = _ctx(nirrep)
    try:
        tA = ctx.tensor("A", *SHAPES[as_], packed=(as_ == "abef"))
        tB = ctx.tensor("B", *SHAPES[bs])
        tC = ctx.tensor("C", *SHAPES[cs])
        fa = random_so(ctx, *SHAPES[as_], rng)
        fb = random_so(ctx, *SHAPES[bs], rng)
        fc = random_so(ctx, *SHAPES[cs], rng)
        write_full(tA, fa)
        write_full(tB, fb)
        write_full(tC, fc)
        alpha, beta = 0.75, -1.25
        ctx.contract(alpha, tA, ia, tB, ib, beta, tC, ic)
        got = tC.to_full()
        ref = reference_contract(alpha, fa, ia, fb, ib, 1.0, fc, ic, tC.group)
        # beta reaches only the C blocks that receive a contribution (lazy beta)
        bm = beta_mask(ctx, (SHAPES[as_], SHAPES[bs], SHAPES[cs]), ia, ib, ic)
        ref = ref + np.where(bm, (beta - 1.0) * fc, 0.0)
        assert np.abs(got - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())
    finally:
        ctx.close()


@pytest.mark.parametrize("nirrep", [1, 2])
def test_sum_dot_scale_norm(nirrep):
    rng = np.random.default_rng(3)
    ctx = _ctx(nirrep)
    try:
        t = ctx.tensor("T", (2, 0), (0, 2))
        u = ctx.tensor("U", (2, 0), (0, 2))
        ft, fu = random_so(ctx, (2, 0), (0, 2), rng), random_so(ctx, (2, 0), (0, 2), rng)
        write_full(t, ft)
        write_full(u, fu)
        # B["abij"] = 2 B + 0.5 A["baji"]
        ctx.sum(0.5, t, "baji", 2.0, u, "abij")
        ref = 2.0 * fu + 0.5 * ft.transpose(1, 0, 3, 2)
        assert np.abs(u.to_full() - ref).max() < 1e-13
        # full spin-orbital dot (SpinorbitalTensor::dot)
        d = ctx.dot(t, "abij", u, "abij")
        assert abs(d - np.sum(ft * ref)) < 1e-11 * max(1, abs(d))
        ctx.scale(u, -3.0)
        assert np.abs(u.to_full() + 3.0 * ref).max() < 1e-12
        assert abs(u.norm(0) - np.abs(3.0 * ref).max()) < 1e-12
    finally:
        ctx.close()


def test_weight_zero_rule_on_device():
    ctx = _ctx(1)
    try:
        t = ctx.tensor("T", (1, 0), (0, 1))
        rng = np.random.default_rng(0)
        f = random_so(ctx, (1, 0), (0, 1), rng)
        write_full(t, f)
        dv = np.array([-1.0, -2.0, -3.0, -4.0, -5.0])
        do = np.array([1.0, 2.0, 3.00001])
        ctx.weight(t, dv, do)
        den = np.concatenate([dv, dv])[:, None] + np.concatenate([do, do])[None, :]
        ref = np.where(np.abs(den) < 1e-4, 0.0, f / den)
        assert np.abs(t.to_full() - ref).max() < 1e-14
    finally:
        ctx.close()


def test_key_value_write_fills_antisymmetric_images():
    ctx = _ctx(1)
    try:
        t = ctx.tensor("T", (2, 0), (0, 2))
        # AA case: alpha counts (2,0,0,2); key of (a=1,b=3,i=0,j=2) in a 5x5x3x3 block
        key = 1 + 5 * (3 + 5 * (0 + 3 * 2))
        t.write((2, 0, 0, 2), [key], [0.5])
        full = t.to_full()
        assert full[1, 3, 0, 2] == 0.5 and full[3, 1, 0, 2] == -0.5
        assert full[1, 3, 2, 0] == -0.5 and full[3, 1, 2, 0] == 0.5
        assert t.read((2, 0, 0, 2), [key])[0] == 0.5
    finally:
        ctx.close()


def test_bad_index_string_is_an_error():
    ctx = _ctx(1)
    try:
        a = ctx.tensor("A", (1, 0), (0, 1))
        b = ctx.tensor("B", (1, 0), (0, 1))
        c = ctx.tensor("C", (1, 0), (0, 1))
        with pytest.raises(A.CcsdError):
            ctx.contract(1.0, a, "aij", b, "ai", 0.0, c, "ai")
        with pytest.raises(A.CcsdError):
            ctx.contract(1.0, a, "ai", b, "bj", 0.0, c, "ak")
    finally:
        ctx.close()
