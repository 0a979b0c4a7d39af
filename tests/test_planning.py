"""Planner checks without a GPU, on planning-only contexts (device < 0).

Statements plan exactly as on the device (spin cases, irrep blocks, pair restrictions),
so flop counts, accounting and error paths of the indexed-tensor interface
(src/tensor/indexable_tensor.hpp:133-155) are testable on the host.
"""
from math import comb

import pytest

import aquarius_b200 as A


def _ctx(vrt, occ):
    c = A.Context(-1)
    c.set_spaces(vrt=vrt, occ=occ)
    return c


@pytest.mark.parametrize("o,v", [(2, 6), (4, 20), (5, 13)])
def test_spin_orbital_ladder_flops(o, v):
    """Z2 += 1/2 V_abef Tau_efij over packed V: same-spin pairs counted once,
    4 C(v,2)^2 C(o,2) + 2 v^4 o^2 (the stored-unique convention of the reference)."""
    with _ctx([v], [o]) as c:
        V = c.tensor("V", (2, 0), (2, 0), packed=True)
        T = c.tensor("T", (2, 0), (0, 2))
        Z = c.tensor("Z", (2, 0), (0, 2))
        Z["abij"] += 0.5 * V["abef"] * T["efij"]
        assert c.plan_flops() == 4 * comb(v, 2) ** 2 * comb(o, 2) + 2 * v ** 4 * o ** 2


@pytest.mark.parametrize("o,v", [(2, 6), (4, 20)])
def test_plain_ladder_flops(o, v):
    """closed-shell ladder Z2 += 1/2 VABCD Tau (rhfccsd.cxx:310): 2 v^4 o^2"""
    with _ctx([v], [o]) as c:
        V = c.tensor("V", (2, 0), (2, 0), plain=True)
        T = c.tensor("T", (2, 0), (0, 2), plain=True)
        Z = c.tensor("Z", (2, 0), (0, 2), plain=True)
        Z["abij"] += 0.5 * V["abef"] * T["efij"]
        assert c.plan_flops() == 2 * v ** 4 * o ** 2


def test_symmetry_blocks_reduce_flops():
    """D2h blocks: the same statement costs less than in C1 over the same orbitals."""
    occ, vrt = [2, 1, 1, 0, 1, 1, 0, 1], [4, 3, 2, 3, 3, 2, 3, 2]
    flops = {}
    for name, (v, o) in {"c1": ([sum(vrt)], [sum(occ)]), "d2h": (vrt, occ)}.items():
        with _ctx(v, o) as c:
            W = c.tensor("W", (1, 1), (1, 1))
            T = c.tensor("T", (2, 0), (0, 2))
            Z = c.tensor("Z", (2, 0), (0, 2))
            Z["abij"] += W["amei"] * T["ebjm"]
            flops[name] = c.plan_flops()
    assert 0 < flops["d2h"] < flops["c1"] / 4


def test_tensor_bytes_are_accounted():
    with _ctx([6], [3]) as c:
        b0 = c.device_bytes()
        T = c.tensor("T", (2, 0), (0, 2))
        # spin cases aa, ab, bb of [v, v, o, o] stored unpacked
        assert c.device_bytes() - b0 == 8 * 3 * (6 * 6 * 3 * 3)
        P = c.tensor("P", (2, 0), (0, 2), plain=True)
        assert c.device_bytes() - b0 == 8 * 4 * (6 * 6 * 3 * 3)
        del T, P


def test_mixing_plain_and_spin_orbital_tensors_is_rejected():
    with _ctx([6], [3]) as c:
        V = c.tensor("V", (2, 0), (2, 0))
        T = c.tensor("T", (2, 0), (0, 2), plain=True)
        Z = c.tensor("Z", (2, 0), (0, 2))
        with pytest.raises(A.CcsdError) as e:
            Z["abij"] += V["abef"] * T["efij"]
        assert e.value.code == 4   # CCSD_ERR_PLAN


def test_bad_index_strings_are_rejected():
    with _ctx([6], [3]) as c:
        V = c.tensor("V", (2, 0), (2, 0))
        T = c.tensor("T", (2, 0), (0, 2))
        Z = c.tensor("Z", (2, 0), (0, 2))
        with pytest.raises(A.CcsdError):
            Z["abij"] += V["abex"] * T["efij"]      # x summed without a partner
        with pytest.raises(A.CcsdError):
            Z["abij"] += V["abef"] * T["efaj"]      # a in A, B and C
        with pytest.raises(A.CcsdError):
            Z["abij"] += V["abie"] * T["efij"]      # occupied letter on a virtual position


def test_planning_context_holds_no_data():
    with _ctx([6], [3]) as c:
        T = c.tensor("T", (2, 0), (0, 2))
        for call in (lambda: T.fill(1.0), lambda: T.norm(0), lambda: T.read_block((2, 0, 0, 2))):
            with pytest.raises(A.CcsdError) as e:
                call()
            assert e.value.code == 9   # CCSD_ERR_UNSUPPORTED


def test_closed_shell_iteration_plans_in_every_point_group():
    for nirrep in (1, 2, 4, 8):
        occ, vrt, _ = A.synth_irreps(5, nirrep, 10, 40)
        f, b = A.rhf_plan_query(vrt, occ)
        assert f > 0 and b > 0


@pytest.mark.parametrize("o,v", [(2, 6), (4, 20)])
def test_lambda_ladder_flops(o, v):
    """Lambda's Z2[ijab] += 1/2 WABEF[efab] L2[ijef] (lambdaccsd.cxx:122) over an unpacked
    W: the same restricted-pair count as the CCSD ladder."""
    with _ctx([v], [o]) as c:
        W = c.tensor("W", (2, 0), (2, 0))
        L2 = c.tensor("L2", (0, 2), (2, 0))
        Z = c.tensor("Z", (0, 2), (2, 0))
        Z["ijab"] += 0.5 * W["efab"] * L2["ijef"]
        assert c.plan_flops() == 4 * comb(v, 2) ** 2 * comb(o, 2) + 2 * v ** 4 * o ** 2


def test_lambda_plan_query():
    """CCSD + spin-orbital Hbar + Lambda plan on the host: every Hbar and Lambda statement
    plans, one Lambda iteration costs more than its ladder, forming Hbar more than one
    Lambda iteration, and D2h blocks cost less than C1 over the same orbitals."""
    o, v = 4, 20
    hf, fl, by = A.lambda_plan_query([v], [o])
    ladder = 4 * comb(v, 2) ** 2 * comb(o, 2) + 2 * v ** 4 * o ** 2
    assert fl > ladder and hf > fl and by > 0
    occ, vrt = [2, 1, 1, 0, 1, 1, 0, 1], [4, 3, 2, 3, 3, 2, 3, 2]
    hf8, fl8, by8 = A.lambda_plan_query(vrt, occ)
    hf1, fl1, by1 = A.lambda_plan_query([sum(vrt)], [sum(occ)])
    assert 0 < fl8 < fl1 / 4 and 0 < hf8 < hf1 / 4 and by8 < by1


def test_rejected_options_leave_no_state():
    """A solver whose options are rejected gives back what its constructor took; the
    same query then succeeds."""
    for bad in ({"diis_order": 20}, {"precision": "split", "diis_order": 0}):
        with pytest.raises(A.CcsdError) as e:
            A.plan_query([6], [2], **bad)
        assert e.value.code == 1   # CCSD_ERR_ARG
        with pytest.raises(A.CcsdError):
            A.lambda_plan_query([6], [2], **bad)
    assert A.lambda_plan_query([6], [2])[1] > 0
