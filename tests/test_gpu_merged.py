"""Merged symmetry-blocked products on the split path (csrc/merged.cpp).

The block products of one irrep class of a symmetry-blocked statement (every row block
with every column block over every k block of one pair irrep) run as one INT8 split GEMM
over rectangles of the merged operands, instead of hundreds of block GEMMs too small for
the tensor cores.  At these sizes no single block product reaches the split kernel, so
every split launch is a merged one.  The solve matches the oracle (src/cc/ccsd.cxx:91-193)
at every iteration with the split path's bar: |dE| <= 1e-8 Eh, max|dT2| <= 1e-7.
"""
import numpy as np
import pytest

import aquarius_b200 as A
from oracle import ccsd_oracle as O

pytestmark = pytest.mark.gpu


def _solve(o, v, seed, nirrep, iters, ref=None):
    eps, B, occ, vrt, aux = A.synth_problem(seed, o, v, nirrep=nirrep)
    rows = []
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=vrt, occ=occ)
        H = ctx.hamiltonian_from_factor(B, eps, aux_per_irrep=aux)
        s = ctx.solver(H, diis_order=8, precision="split_i8", slices=4)
        n0 = ctx.split_launches()
        energies = []
        for _ in range(iters):
            e, _ = s.iterate()
            energies.append(e)
            if ref is not None:
                e_ref, _ = ref.iterate()
                rows.append((abs(e - e_ref), float(np.abs(s.T2.to_full() - ref.T.T2).max())))
        split = ctx.split_launches() - n0
        s.close()
        H.destroy()
    return rows, split, energies


@pytest.mark.parametrize("o,v,seed,nirrep", [(12, 72, 7, 2), (12, 96, 8, 4), (16, 128, 9, 8)],
                         ids=["2irreps", "4irreps", "8irreps"])
def test_merged_split_matches_oracle_every_iteration(o, v, seed, nirrep, monkeypatch):
    monkeypatch.setenv("CCSD_MERGED", "1")
    eps, B, *_ = A.synth_problem(seed, o, v, nirrep=nirrep)
    ref = O.CCSD(O.hamiltonian_from_factor(B, eps, o), diis_order=8)
    rows, split, _ = _solve(o, v, seed, nirrep, 6, ref)
    assert split > 0
    for it, (de, dt2) in enumerate(rows):
        assert de <= 1e-8 and dt2 <= 1e-7, (it, de, dt2)


def test_without_merging_these_products_stay_on_fp64(monkeypatch):
    monkeypatch.setenv("CCSD_MERGED", "0")
    _, split, e_off = _solve(12, 72, 7, 2, 3)
    assert split == 0
    monkeypatch.setenv("CCSD_MERGED", "1")
    _, split_on, e_on = _solve(12, 72, 7, 2, 3)
    assert split_on > 0
    assert max(abs(a - b) for a, b in zip(e_off, e_on)) <= 1e-8
