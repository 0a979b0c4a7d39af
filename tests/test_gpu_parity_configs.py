"""Parity at the benchmark's own problem sizes, with the engine's natural routing.

The other GPU tests compare with the oracle at small sizes and, for the split path, with
every product forced onto the tensor-core kernel.  Here the synthetic problems have the
sizes the benchmark runs, and the split solver keeps its default routing: large block
products on the tcgen05 split kernel, skinny and small ones on the FP64 kernels, cached
slices of the constant H operands and split-K folds, exactly as the timed solve does.

* o=16 v=128 C1 (the FP64 plain-path configuration): the native-FP64 solver and the
  4-slice INT8 split solver run side by side with the oracle (src/cc/ccsd.cxx:91-193)
  for 8 iterations.  FP64: |dE| <= 1e-11 Eh and max|dT1|, max|dT2| <= 1e-11 at every
  iteration.  Split: |dE| <= 1e-8 Eh and max|dT2| <= 1e-7 at every iteration.
* o=16 v=96 with 8 irreps (D2h, uneven seeded irrep counts): the same bars.
"""
import numpy as np
import pytest

import aquarius_b200 as A
from oracle import ccsd_oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _lockstep(o, v, seed, nirrep, iters):
    eps, B, occ, vrt, aux = A.synth_problem(seed, o, v, nirrep=nirrep)
    ref = O.CCSD(O.hamiltonian_from_factor(B, eps, o), diis_order=8)
    rows = []
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=vrt, occ=occ)
        H = ctx.hamiltonian_from_factor(B, eps, aux_per_irrep=aux if nirrep > 1 else None)
        s64 = ctx.solver(H, diis_order=8, precision="fp64")
        s8 = ctx.solver(H, diis_order=8, precision="split_i8", slices=4)
        assert abs(s64.mp2 - ref.mp2) < 1e-12 and abs(s8.mp2 - ref.mp2) < 1e-12
        n0 = ctx.split_launches()
        for it in range(iters):
            e_ref, c_ref = ref.iterate()
            e64, c64 = s64.iterate()
            e8, c8 = s8.iterate()
            rows.append(dict(
                it=it, e_ref=e_ref, c_ref=c_ref,
                de64=abs(e64 - e_ref), dc64=abs(c64 - c_ref),
                dt1_64=np.abs(s64.T1.to_full() - ref.T.T1).max(),
                dt2_64=np.abs(s64.T2.to_full() - ref.T.T2).max(),
                de8=abs(e8 - e_ref),
                dt1_8=np.abs(s8.T1.to_full() - ref.T.T1).max(),
                dt2_8=np.abs(s8.T2.to_full() - ref.T.T2).max()))
        split = ctx.split_launches() - n0
        s8.close()
        s64.close()
        H.destroy()
    return rows, split


def _check(rows):
    for r in rows:
        it = r["it"]
        assert r["de64"] <= 1e-11, (it, r)
        assert r["dc64"] <= 1e-9 * max(1e-3, r["c_ref"]), (it, r)
        assert r["dt1_64"] <= 1e-11 and r["dt2_64"] <= 1e-11, (it, r)
        assert r["de8"] <= 1e-8, (it, r)
        assert r["dt1_8"] <= 1e-7 and r["dt2_8"] <= 1e-7, (it, r)


def test_o16_v128_c1_fp64_and_split_match_oracle_every_iteration():
    rows, split = _lockstep(16, 128, 2, 1, 8)
    # natural routing sends the particle ladder (M = v^2, N = o^2, K = v^2 block products)
    # and the other large products to the tcgen05 split kernel
    assert split > 0
    _check(rows)


def test_o16_v96_d2h_fp64_and_split_match_oracle_every_iteration():
    rows, _ = _lockstep(16, 96, 6, 8, 8)
    _check(rows)
