"""The solvers' own recorded statement lists, replayed on the CPU against the oracles.

One CCSD iteration (ccsd.cxx:123-180), the spin-orbital Hbar (st2eoperator.hpp:59-130,
isHbar), one Lambda-CCSD iteration (lambdaccsd.cxx:80-124), the energy reductions, and the
closed-shell iteration and Hbar (rhfccsd.cxx:110-186, 237-316) are planned on the host for C1
and D2h sizes and for the UHF triplet CH2 (alpha and beta spaces differ) (ccsd_plan_export_solver), executed with numpy over the engine's block layout
(tests/plan_replay.py) and compared with oracle/ccsd_oracle.py, oracle/lambda_ccsd.py and
oracle/rhf_ccsd.py.  This checks the statement lists in csrc/solver.cpp -- their
order, assignments, factors and signs -- with the planner's expansion, without a device.
"""
import numpy as np
import pytest

import aquarius_b200 as A
from oracle import ccsd_oracle as O
from oracle import lambda_ccsd as LC
from tests import plan_replay as R

H_NAMES = {"f(ai)": "fAI", "f(ia)": "fME", "f(ab)": "fAE", "f(ij)": "fMI", "<ij||kl>": "VMNIJ",
           "<ai||jk>": "VAMIJ", "<ij||ab>": "VMNEF", "<ai||bj>": "VAMEI", "<ai||bc>": "VAMEF",
           "<ab||cd>": "VABEF"}
HBAR_NAMES = {"Hbar f(ai)": "ai", "Hbar F(me)": "ia", "Hbar F(ae)": "ab", "Hbar F(mi)": "ij",
              "Hbar W(mn,ij)": "ijkl", "Hbar W(am,ij)": "aijk", "Hbar W(mn,ej)": "ijak",
              "Hbar W(ab,ij)": "abij", "Hbar W(mn,ef)": "ijab", "Hbar W(am,ei)": "aibj",
              "Hbar W(am,ef)": "aibc", "Hbar W(ab,ej)": "abci", "Hbar W(ab,ef)": "abcd"}
SIZES = {1: (3, 6), 4: (5, 12), 8: (8, 16)}


@pytest.fixture(scope="module", params=[1, 4, 8], ids=["C1", "4-irreps", "D2h"])
def problem(request):
    nirrep = request.param
    o, v = SIZES[nirrep]
    eps, B, occ, vrt, _ = A.synth_problem(31 + nirrep, o, v, nirrep=nirrep)
    H = O.hamiltonian_from_factor(B, eps, o, ladder_literal=True)
    cc = O.CCSD(H, diis_order=8)
    for _ in range(3):
        cc.iterate()                     # amplitudes away from the MP1 guess
    Hb = LC.hbar(H, cc.T.T1, cc.T.T2)
    lam = LC.LambdaCCSD(Hb, cc.T.T1, cc.T.T2, diis_order=8)
    lam.iterate()                        # Lambda amplitudes away from L = T
    return occ, vrt, H, cc, Hb, lam


def _replay(problem, method, which, arrays, tmp_path):
    return _replay_spaces(dict(vrt=problem[1], occ=problem[0]), method, which, arrays, tmp_path)


def _replay_spaces(spaces, method, which, arrays, tmp_path):
    path = tmp_path / f"{method}-{which}.txt"
    A.plan_export_solver(method, spaces["vrt"], spaces["occ"], which, path, spaces.get("vrt_beta"),
                         spaces.get("occ_beta"))
    dump = R.load(path)
    ctx = A.Context(-1)
    ctx.set_spaces(**spaces)
    store = {}
    for h, t in dump.tensors.items():
        if t.view_of:
            continue
        full = arrays.get(t.name)
        store[h] = R.to_storage(ctx, t, full) if full is not None else np.zeros(max(t.total, 1))
    acc = R.replay(dump, store)
    by_name = {t.name: (t, store[h]) for h, t in dump.tensors.items() if not t.view_of}

    def check(name, want, tol=1e-12):
        t, got = by_name[name]
        w = R.to_storage(ctx, t, want)
        err = np.abs(got - w).max()
        assert err < tol * max(1.0, np.abs(w).max()), (name, err)

    return check, acc, by_name, ctx


def _h_arrays(H):
    return {n: getattr(H, k) for n, k in H_NAMES.items()}


def test_ccsd_iteration_plan(problem, tmp_path):
    _, _, H, cc, _, _ = problem
    arrays = _h_arrays(H)
    arrays.update({"T(1)": cc.T.T1, "T(2)": cc.T.T2})
    check, _, _, ctx = _replay(problem, "ccsd", "iteration", arrays, tmp_path)
    Z1, Z2 = cc.residual(cc.T)
    check("Tau", O.CCSD.make_tau(cc.T))
    check("Z(1)", Z1)
    check("Z(2)", Z2)
    ctx.close()


def test_ccsd_energy_plan(problem, tmp_path):
    _, _, H, cc, _, _ = problem
    arrays = _h_arrays(H)
    arrays.update({"T(1)": cc.T.T1, "Tau": O.CCSD.make_tau(cc.T)})
    _, e, _, ctx = _replay(problem, "ccsd", "energy", arrays, tmp_path)
    assert abs(e - cc.energy_of(cc.T)) < 1e-13
    ctx.close()


def test_hbar_plan(problem, tmp_path):
    _, _, H, cc, Hb, _ = problem
    arrays = _h_arrays(H)
    arrays.update({"T(1)": cc.T.T1, "T(2)": cc.T.T2})
    check, _, by_name, ctx = _replay(problem, "ccsd", "hbar", arrays, tmp_path)
    written = [n for n in HBAR_NAMES if n in by_name]
    # f(ai) and <ab||ij> of Hbar are zero and no statement writes them
    assert sorted(set(HBAR_NAMES) - set(written)) == ["Hbar W(ab,ij)", "Hbar f(ai)"]
    for name in written:
        check(name, Hb[HBAR_NAMES[name]])
    ctx.close()


def test_lambda_iteration_plan(problem, tmp_path):
    _, _, _, cc, Hb, lam = problem
    arrays = {n: Hb[k] for n, k in HBAR_NAMES.items()}
    arrays.update({"T(2)": cc.T.T2, "L(1)": lam.L.T1, "L(2)": lam.L.T2})
    check, _, _, ctx = _replay(problem, "lambda", "iteration", arrays, tmp_path)
    Z1, Z2 = lam.residual(lam.L.T1, lam.L.T2)
    check("Z(1)", Z1)
    check("Z(2)", Z2)
    ctx.close()


def test_lambda_energy_plan(problem, tmp_path):
    _, _, _, _, Hb, lam = problem
    arrays = {n: Hb[k] for n, k in HBAR_NAMES.items()}
    arrays.update({"L(2)": lam.L.T2})
    _, e, _, ctx = _replay(problem, "lambda", "energy", arrays, tmp_path)
    assert abs(e - 0.25 * float(np.vdot(Hb["ijab"], lam.L.T2))) < 1e-13
    ctx.close()


# closed shell (rhfccsd.cxx): plain spatial tensors; VAIJB, VAIJBSA and W(Am,Ie) hold their
# [a, i, j, b] elements at [a, i, b, j]
RHF_NAMES = {"fAI": "fAI", "fAB": "fAB", "fIJ": "fIJ", "<Ab|Cd>": "VABCD", "<Ab|Ci>": "VABCI", "<Ab|Ij>": "VABIJ",
             "<Ai|Bj>": "VAIBJ", "<Ai|Jk>": "VAIJK", "<Ij|Kl>": "VIJKL", "VABIJSA": "VABIJSA"}
RHF_HBAR = {"F(ME)": "FME", "F(MI)": "FMI", "F(AE)": "FAE", "W(Mn,Ij)": "WMNIJ", "W(Mn,Ej)": "WMNEJ",
            "W(Am,Ij)": "WAMIJ", "W(Am,Ei)": "WAMEI", "W(Ab,Ej)": "WABEJ"}


@pytest.fixture(scope="module", params=[1, 4, 8], ids=["C1", "4-irreps", "D2h"])
def rhf_problem(request):
    from oracle import rhf_ccsd as RH
    nirrep = request.param
    o, v = SIZES[nirrep]
    eps, B, occ, vrt, _ = A.synth_problem(41 + nirrep, o, v, nirrep=nirrep)
    ref = RH.RHFCCSD(np.diag(eps), O.eri_from_factor(B), o, diis_order=8)
    for _ in range(3):
        ref.iterate()
    return occ, vrt, ref


def _rhf_arrays(ref):
    arrays = {n: getattr(ref, k) for n, k in RHF_NAMES.items()}
    arrays["<Ai|Jb>"] = ref.VAIJB.transpose(0, 1, 3, 2)
    arrays["VAIJBSA"] = ref.VAIJBSA.transpose(0, 1, 3, 2)
    arrays.update({"T1": ref.T1, "T2": ref.T2})
    return arrays


def test_rhf_iteration_plan(rhf_problem, tmp_path):
    occ, vrt, ref = rhf_problem
    check, _, _, ctx = _replay(rhf_problem, "rhf", "iteration", _rhf_arrays(ref), tmp_path)
    Z1, Z2 = ref.residual(ref.T1, ref.T2)
    check("Tau", ref.T2 + np.einsum("ai,bj->abij", ref.T1, ref.T1))
    check("Z1", Z1)
    check("Z2", Z2)
    ctx.close()


def test_rhf_hbar_plan(rhf_problem, tmp_path):
    occ, vrt, ref = rhf_problem
    check, _, _, ctx = _replay(rhf_problem, "rhf", "hbar", _rhf_arrays(ref), tmp_path)
    want = ref.hbar()
    for name, key in RHF_HBAR.items():
        check(name, want[key])
    check("W(Am,Ie)", want["WAMIE"].transpose(0, 1, 3, 2))
    ctx.close()


@pytest.fixture(scope="module")
def uhf_problem():
    """CH2/cc-pVDZ triplet (test/input.aq:47-71): UHF, alpha and beta spaces differ."""
    import json
    from pathlib import Path
    from oracle import scf
    fixture = json.loads((Path(__file__).parent / "golden" / "molecules.json").read_text())
    res, Hao, eri = scf.solve_scf(fixture, "ch2-pvdz")
    H = scf.SpinOrbitalHamiltonian(res, Hao, eri)
    (na, nb), (va, vb) = H.nocc, H.nvrt
    cc = O.CCSD(H, diis_order=8)
    for _ in range(3):
        cc.iterate()
    Hb = LC.hbar(H, cc.T.T1, cc.T.T2)
    lam = LC.LambdaCCSD(Hb, cc.T.T1, cc.T.T2, diis_order=8)
    lam.iterate()
    return dict(vrt=[va], occ=[na], vrt_beta=[vb], occ_beta=[nb]), H, cc, Hb, lam


def test_uhf_ccsd_iteration_plan(uhf_problem, tmp_path):
    spaces, H, cc, _, _ = uhf_problem
    arrays = _h_arrays(H)
    arrays.update({"T(1)": cc.T.T1, "T(2)": cc.T.T2})
    check, _, _, ctx = _replay_spaces(spaces, "ccsd", "iteration", arrays, tmp_path)
    Z1, Z2 = cc.residual(cc.T)
    check("Z(1)", Z1)
    check("Z(2)", Z2)
    ctx.close()


def test_uhf_hbar_and_lambda_plans(uhf_problem, tmp_path):
    spaces, H, cc, Hb, lam = uhf_problem
    arrays = _h_arrays(H)
    arrays.update({"T(1)": cc.T.T1, "T(2)": cc.T.T2})
    check, _, by_name, ctx = _replay_spaces(spaces, "ccsd", "hbar", arrays, tmp_path)
    for name in HBAR_NAMES:
        if name in by_name:
            check(name, Hb[HBAR_NAMES[name]])
    ctx.close()
    arrays = {n: Hb[k] for n, k in HBAR_NAMES.items()}
    arrays.update({"T(2)": cc.T.T2, "L(1)": lam.L.T1, "L(2)": lam.L.T2})
    check, _, _, ctx = _replay_spaces(spaces, "lambda", "iteration", arrays, tmp_path)
    Z1, Z2 = lam.residual(lam.L.T1, lam.L.T2)
    check("Z(1)", Z1)
    check("Z(2)", Z2)
    ctx.close()


def test_rhf_export_refuses_beta_spaces(tmp_path):
    with pytest.raises(A.CcsdError):
        A.plan_export_solver("rhf", [4], [2], "iteration", tmp_path / "p.txt", vrt_beta=[5], occ_beta=[1])


def test_replay_tells_a_changed_statement_apart(problem, tmp_path):
    """The replayed Lambda plan against an oracle residual with one statement's sign
    flipped (the ring term W(am,ei) L2, lambdaccsd.cxx:124) no longer matches.  `ring` is
    the statement's full contribution: LC.contract applies the statement's implicit
    antisymmetriser P(ij)P(ab) to the output lines that come from both factors, so
    Z2 - 2 * ring is the residual with that term's sign flipped."""
    _, _, _, cc, Hb, lam = problem
    arrays = {n: Hb[k] for n, k in HBAR_NAMES.items()}
    arrays.update({"T(2)": cc.T.T2, "L(1)": lam.L.T1, "L(2)": lam.L.T2})
    check, _, _, ctx = _replay(problem, "lambda", "iteration", arrays, tmp_path)
    _, Z2 = lam.residual(lam.L.T1, lam.L.T2)
    ring = LC.contract(1.0, Hb["aibj"], "eiam", lam.L.T2, "mjbe", "ijab", LC.SHAPES["ijab"])
    assert np.abs(ring).max() > 1e-6
    check("Z(2)", Z2)
    with pytest.raises(AssertionError):
        check("Z(2)", Z2 - 2.0 * ring)
    ctx.close()
