"""The short-product kernel (both extents <= 64, long K; partials per CTA added by the fold
in plan order) against the numpy statement semantics and the tiled FP64 path.

Short products arise wherever a statement's block products have two small external
extents and a long sum, e.g. F(mi) += <mn||ef> t(ef,in) and Z(ai) += <am||ef> tau(ef,im)
over irrep blocks.  The cases cover one destination per element, antisymmetriser
variants on both sides (m, n and i, j each split between the factors), and symmetry
blocks with uneven irrep counts, where the products of one output block sum over many k
blocks and used to run one launch per level."""
import numpy as np
import pytest

import aquarius_b200 as A
from tests.helpers import random_so, reference_contract, write_full

pytestmark = pytest.mark.gpu

SHAPES = {"ai": ((1, 0), (0, 1)), "mi": ((0, 1), (0, 1)), "mnij": ((0, 2), (0, 2)),
          "abij": ((2, 0), (0, 2)), "mnef": ((0, 2), (2, 0)), "amef": ((1, 1), (2, 0)),
          "amei": ((1, 1), (1, 1))}

CASES = [
    # C, idxC, A, idxA, B, idxB, sizes
    ("mi", "mi", "mnef", "mnef", "abij", "efin", "long"),
    ("ai", "ai", "amef", "amef", "abij", "efim", "long"),
    ("mnij", "mnij", "mnef", "mnef", "abij", "efij", "long"),
    # the ring term at a few orbitals per irrep: P(ab) P(ij), four variants per element
    ("abij", "abij", "amei", "amei", "abij", "ebjm", "few"),
]

SPACES = {
    "long": {"c1": ([24], [4]),
             "d2h": ([5, 3, 4, 2, 4, 3, 2, 3], [2, 1, 1, 0, 1, 1, 0, 1]),
             "c2v-wide": ([14, 9, 11, 6], [3, 2, 2, 1])},
    "few": {"c1": ([4], [2]),
            "d2h": ([2, 1, 1, 1, 2, 1, 1, 1], [1, 1, 1, 0, 1, 0, 1, 0]),
            "c2v-wide": ([3, 2, 2, 1], [2, 1, 1, 1])},
}


@pytest.mark.parametrize("spaces", ["c1", "c2v-wide", "d2h"])
@pytest.mark.parametrize("case", CASES, ids=[f"{c[1]}+={c[3]}*{c[5]}" for c in CASES])
def test_short_products_match_reference_and_tiled(case, spaces, monkeypatch):
    cs, ic, as_, ia, bs, ib, sizes = case
    vrt, occ = SPACES[sizes][spaces]
    out = {}
    # every K takes the short kernel here: the symmetry blocks of these sizes sum over a few
    # hundred k at most, below the default threshold
    monkeypatch.setenv("CCSD_SHORT_MIN_K", "1")
    for path in ("auto", "tiled"):
        monkeypatch.setenv("CCSD_FP64_TILED", "1" if path == "tiled" else "0")
        rng = np.random.default_rng(23)
        ctx = A.Context(0)
        try:
            ctx.set_spaces(vrt=vrt, occ=occ)
            tA = ctx.tensor("A", *SHAPES[as_])
            tB = ctx.tensor("B", *SHAPES[bs])
            tC = ctx.tensor("C", *SHAPES[cs])
            fa = random_so(ctx, *SHAPES[as_], rng)
            fb = random_so(ctx, *SHAPES[bs], rng)
            fc = random_so(ctx, *SHAPES[cs], rng)
            write_full(tA, fa)
            write_full(tB, fb)
            write_full(tC, fc)
            ctx.contract(0.75, tA, ia, tB, ib, 1.0, tC, ic)
            # a second statement on the same tensors replays the recorded schedule
            ctx.contract(-0.25, tA, ia, tB, ib, 1.0, tC, ic)
            out[path] = tC.to_full()
            ref = reference_contract(0.5, fa, ia, fb, ib, 1.0, fc, ic, tC.group)
        finally:
            ctx.close()
        scale = max(1.0, np.abs(ref).max())
        assert np.abs(out[path] - ref).max() < 1e-12 * scale, path
    assert np.abs(out["auto"] - out["tiled"]).max() < 1e-12 * max(1.0, np.abs(out["tiled"]).max())
