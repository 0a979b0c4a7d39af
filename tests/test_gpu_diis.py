"""DIIS over caller tensors (ccsd_diis_*) against the oracle's restatement of the
reference's DIIS (src/convergence/diis.hpp:70-227).

The oracle's CCSD iteration runs as usual; every (x, dx) pair it hands to its DIIS is
also written into engine tensors and given to the device DIIS.  After each call the
device's x and dx (the extrapolated T and the extrapolated residual, diis.hpp:205-226)
and its coefficients must equal the oracle's.

Tolerance: the error matrices are dots of the same vectors summed in different orders
(agreeing to ~1e-16 relative), and the bordered systems are solved by two backward-stable
methods (LAPACK dsysv with Bunch-Kaufman pivoting in the oracle, Gaussian elimination
with partial pivoting on the device), whose solutions agree to about cond(E) * eps.  The
coefficients are compared to 1e-12 + 64 eps cond(E) max|c|, where cond(E) is the
condition number of the oracle's bordered matrix at that call (up to ~1e9 late in a
solve), and x, dx to the same bound times the sum of the stored vectors' max-abs.
"""
import numpy as np
import pytest

import aquarius_b200 as A
from oracle import ccsd_oracle as O
from tests.helpers import write_full

pytestmark = pytest.mark.gpu

T1S, T2S = ((1, 0), (0, 1)), ((2, 0), (0, 2))


def _recorded_pairs(o, v, seed, order, start, damping, iters):
    eps, B, *_ = A.synth_problem(seed, o, v)
    ref = O.CCSD(O.hamiltonian_from_factor(B, eps, o), diis_order=order, diis_start=start, diis_damping=damping)
    rec = []
    inner = ref.diis.extrapolate

    def spy(x, dx):
        before = (x.copy(), dx.copy())
        inner(x, dx)
        n = min(order, sum(1 for d in ref.diis.old_dx if d is not None))
        extrapolated = n >= 2 and ref.diis.start <= 1      # the call reached the bordered solve
        c = ref.diis.c[:order].copy()
        tol_c = tol_x = 1e-12
        if extrapolated:
            kappa = np.linalg.cond(ref.diis.e[:n + 1, :n + 1])
            tol_c = 1e-12 + 64 * np.finfo(float).eps * kappa * np.abs(c[:n]).max()
            spread = sum(max(np.abs(v.T1).max(), np.abs(v.T2).max())
                         for vs in (ref.diis.old_x, ref.diis.old_dx) for v in vs[:n])
            tol_x = 1e-12 + tol_c * spread
        rec.append((before, (x.copy(), dx.copy()), c, n, extrapolated, tol_c, tol_x))

    ref.diis.extrapolate = spy
    for _ in range(iters):
        ref.iterate()
    return rec


@pytest.mark.parametrize("order,start,damping", [(8, 1, 0.0), (3, 1, 0.0), (5, 3, 0.0), (4, 3, 0.25)],
                         ids=["order8", "ring-wraps", "late-start", "damping"])
def test_device_diis_matches_oracle_every_call(order, start, damping):
    o, v, seed = 4, 12, 31
    rec = _recorded_pairs(o, v, seed, order, start, damping, 9)
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=[v], occ=[o])
        X1, X2 = ctx.tensor("X1", *T1S), ctx.tensor("X2", *T2S)
        D1, D2 = ctx.tensor("D1", *T1S), ctx.tensor("D2", *T2S)
        d = ctx.diis(order=order, start=start, damping=damping)
        assert any(r[4] for r in rec) and not rec[0][4]
        for k, ((x, dx), (x_out, dx_out), c_ref, nref, extrapolated, tol_c, tol_x) in enumerate(rec):
            write_full(X1, x.T1)
            write_full(X2, x.T2)
            write_full(D1, dx.T1)
            write_full(D2, dx.T2)
            d.extrapolate([X1, X2], [D1, D2])
            n, c = d.coefficients()
            assert n == nref, (k, n, nref)
            if extrapolated:
                assert np.abs(c[:n] - c_ref[:n]).max() <= tol_c, (k, c[:n] - c_ref[:n], tol_c)
            else:   # x and dx kept: the stored newest pair alone
                assert c[0] == 1.0 and not np.any(c[1:]), (k, c)
            assert np.abs(X1.to_full() - x_out.T1).max() <= tol_x, k
            assert np.abs(X2.to_full() - x_out.T2).max() <= tol_x, k
            assert np.abs(D1.to_full() - dx_out.T1).max() <= tol_x, k
            assert np.abs(D2.to_full() - dx_out.T2).max() <= tol_x, k
        d.close()


def test_explicit_weights_equal_the_default():
    """weights (1, 1/4) are the ExcitationOperator::dot weights the NULL default takes."""
    o, v = 3, 9
    rec = _recorded_pairs(o, v, 32, 5, 1, 0.0, 6)
    outs = []
    for weights in (None, [1.0, 0.25]):
        with A.Context(0) as ctx:
            ctx.set_spaces(vrt=[v], occ=[o])
            X1, X2 = ctx.tensor("X1", *T1S), ctx.tensor("X2", *T2S)
            D1, D2 = ctx.tensor("D1", *T1S), ctx.tensor("D2", *T2S)
            d = ctx.diis(order=5)
            for (x, dx), *_ in rec:
                write_full(X1, x.T1)
                write_full(X2, x.T2)
                write_full(D1, dx.T1)
                write_full(D2, dx.T2)
                d.extrapolate([X1, X2], [D1, D2], weights=weights)
            outs.append(X2.to_full())
            d.close()
    assert np.abs(outs[0] - outs[1]).max() <= 1e-13


def test_mismatched_pieces_are_refused():
    with A.Context(0) as ctx:
        ctx.set_spaces(vrt=[6], occ=[2])
        X1, X2 = ctx.tensor("X1", *T1S), ctx.tensor("X2", *T2S)
        d = ctx.diis(order=4)
        with pytest.raises(A.CcsdError) as e:
            d.extrapolate([X1], [X2])
        assert e.value.code == 1
        d.extrapolate([X1, X2], [ctx.tensor("D1", *T1S), ctx.tensor("D2", *T2S)])
        with pytest.raises(A.CcsdError):
            d.extrapolate([X1], [ctx.tensor("D3", *T1S)])     # fewer pieces than the first call
        d.close()
