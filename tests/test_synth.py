"""Seeded synthetic inputs (host code in the product library; no device needed)."""
import numpy as np

import aquarius_b200 as A


def test_factor_is_symmetric_and_deterministic(built_lib):
    e1, B1, *_ = A.synth_problem(7, 3, 9)
    e2, B2, *_ = A.synth_problem(7, 3, 9)
    assert np.array_equal(B1, B2) and np.array_equal(e1, e2)
    assert np.array_equal(B1, B1.transpose(0, 2, 1))
    assert B1.shape == (3 * 12, 12, 12)


def test_orbital_energy_ranges(built_lib):
    eps, _, occ, vrt, _ = A.synth_problem(3, 5, 20, with_B=False)
    assert np.all((eps[:5] >= -1.2) & (eps[:5] <= -0.4))
    assert np.all((eps[5:] >= 0.3) & (eps[5:] <= 4.0))
    assert np.all(np.diff(eps[:5]) >= 0) and np.all(np.diff(eps[5:]) >= 0)


def test_d2h_split_and_zero_pattern(built_lib):
    eps, B, occ, vrt, aux = A.synth_problem(11, 12, 40, nirrep=8)
    assert occ.sum() == 12 and vrt.sum() == 40 and aux.sum() == 3 * 52
    assert (occ >= 1).all() and (vrt >= 1).all() and (aux >= 1).all()
    irr = np.concatenate([np.repeat(np.arange(8), occ), np.repeat(np.arange(8), vrt)])
    airr = np.repeat(np.arange(8), aux)
    allowed = (irr[None, :, None] ^ irr[None, None, :]) == airr[:, None, None]
    assert np.all(B[~allowed] == 0)
    assert np.count_nonzero(B[allowed]) > 0.99 * allowed.sum()


def test_different_seeds_differ(built_lib):
    _, B1, *_ = A.synth_problem(1, 3, 6)
    _, B2, *_ = A.synth_problem(2, 3, 6)
    assert not np.allclose(B1, B2)


def test_rhf_plan_query_plans_every_statement():
    """Host-only planning of the closed-shell iteration (no device): every RHFCCSD
    statement plans, in C1 and with D2h blocks, at about half the spin-orbital flops."""
    import aquarius_b200 as A
    f_rhf, b_rhf = A.rhf_plan_query([256], [32], precision="split")
    f_so, b_so = A.plan_query([256], [32], precision="split")
    assert 0 < f_rhf < 0.5 * f_so
    assert b_rhf > 8 * 256 ** 4   # the unpacked <Ab|Cd> block alone
    f8, b8 = A.rhf_plan_query([6, 3, 4, 5, 2, 3, 4, 5], [2, 0, 1, 1, 1, 0, 1, 0])
    assert f8 > 0 and b8 > 0
    # a solve that may refine to 4 slices reserves the larger slice cache
    _, b_ref = A.rhf_plan_query([256], [32], precision="split", refine_tol=1e-7)
    assert b_ref >= b_rhf


import pytest


@pytest.mark.parametrize("seed,o,v,nirrep", [(2, 16, 128, 1), (6, 16, 96, 8), (3, 5, 19, 4), (11, 12, 40, 2)])
def test_numpy_restatement_is_bit_identical(built_lib, seed, o, v, nirrep):
    """oracle/synth.py (which the CPU benchmark legs use, loading no engine library) gives
    the same bits as ccsd_synth_problem: orbital energies, irrep counts and the factor."""
    from oracle import synth as S
    e1, B1, occ1, vrt1, aux1 = A.synth_problem(seed, o, v, nirrep=nirrep)
    e2, B2, occ2, vrt2, aux2 = S.synth_problem(seed, o, v, nirrep=nirrep)
    for x, y in ((occ1, occ2), (vrt1, vrt2), (aux1, aux2)):
        assert np.array_equal(x, y)
    assert np.array_equal(e1.view(np.uint64), e2.view(np.uint64))
    assert np.array_equal(B1.view(np.uint64), B2.view(np.uint64))


def test_numpy_restatement_irrep_counts_at_the_d2h_benchmark_size(built_lib):
    from oracle import synth as S
    for seed in (4, 5, 1000, 1001):
        got = S.synth_irreps(seed, 8, 48, 336)
        ref = A.synth_irreps(seed, 8, 48, 336)
        for x, y in zip(got, ref):
            assert np.array_equal(x, y)
