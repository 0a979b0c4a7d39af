"""The skinny FP64 kernel (one extent <= 32) against the numpy statement semantics, at
sizes where it splits K over CTAs and where the long operand is A or B, contiguous
along rows or along k."""
import numpy as np
import pytest

import aquarius_b200 as A
from tests.helpers import random_so, reference_contract, write_full

pytestmark = pytest.mark.gpu

SHAPES = {"ai": ((1, 0), (0, 1)), "me": ((0, 1), (1, 0)), "mi": ((0, 1), (0, 1)), "ae": ((1, 0), (1, 0)),
          "abij": ((2, 0), (0, 2)), "mnef": ((0, 2), (2, 0)), "amef": ((1, 1), (2, 0)), "amei": ((1, 1), (1, 1)),
          "abej": ((2, 0), (1, 1))}

CASES = [
    # C, idxC, A, idxA, B, idxB
    ("mi", "mi", "mnef", "mnef", "abij", "efin"),    # long K: split-K with a fold
    ("ai", "ai", "amef", "amef", "abij", "efim"),    # N = o, long K
    ("amei", "amei", "amef", "amef", "ai", "fi"),    # long rows of A, N = o
    ("abij", "abij", "mi", "mi", "abij", "abmj"),    # long rows of B (M = o)
    ("ae", "ae", "amef", "amef", "ai", "fm"),        # N = 1
    ("abij", "abij", "abej", "abej", "ai", "ei"),    # long rows of a view
]


@pytest.mark.parametrize("o,v", [(6, 40), (8, 64), (12, 31)], ids=["o6v40", "o8v64", "o12v31"])
@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}+={c[2]}*{c[4]}" for c in CASES])
def test_skinny_matches_reference_and_tiled(case, o, v, monkeypatch):
    """o8v64: hundreds of row tiles with 16-byte copies; o12v31: odd extents, so that
    neighbouring elements are often misaligned and take the 8-byte path."""
    cs, ic, as_, ia, bs, ib = case
    out = {}
    for path in ("auto", "tiled"):
        monkeypatch.setenv("CCSD_FP64_TILED", "1" if path == "tiled" else "0")
        rng = np.random.default_rng(17)
        ctx = A.Context(0)
        try:
            ctx.set_spaces(vrt=[v], occ=[o])
            tA = ctx.tensor("A", *SHAPES[as_])
            tB = ctx.tensor("B", *SHAPES[bs])
            tC = ctx.tensor("C", *SHAPES[cs])
            fa = random_so(ctx, *SHAPES[as_], rng)
            fb = random_so(ctx, *SHAPES[bs], rng)
            fc = random_so(ctx, *SHAPES[cs], rng)
            write_full(tA, fa)
            write_full(tB, fb)
            write_full(tC, fc)
            ctx.contract(0.5, tA, ia, tB, ib, 1.0, tC, ic)
            out[path] = tC.to_full()
            ref = reference_contract(0.5, fa, ia, fb, ib, 1.0, fc, ic, tC.group)
        finally:
            ctx.close()
        scale = max(1.0, np.abs(ref).max())
        assert np.abs(out[path] - ref).max() < 1e-12 * scale, path
    assert np.abs(out["auto"] - out["tiled"]).max() < 1e-12 * max(1.0, np.abs(out["tiled"]).max())
