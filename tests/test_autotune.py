"""The slice autotuner's selection rule (ccsd_slice_choice, host only): statements take one
slice fewer smallest measured energy change first, while the sum of the chosen changes
stays within the budget."""
import numpy as np

import aquarius_b200 as A


def test_smallest_first_within_budget(built_lib):
    dE = [3e-10, -1e-11, 5e-9, 2e-10, -4e-10]
    # sorted |dE|: 1e-11, 2e-10, 3e-10, 4e-10, 5e-9 -> cumulative 1e-11, 2.1e-10, 5.1e-10, 9.1e-10, 5.9e-9
    assert A.slice_choice(dE, 1e-9).tolist() == [True, True, False, True, True]
    assert A.slice_choice(dE, 5.2e-10).tolist() == [True, True, False, True, False]
    assert not A.slice_choice(dE, 1e-12).any()
    assert A.slice_choice(dE, 1.0).all()


def test_ties_keep_statement_order(built_lib):
    dE = [1e-10, 1e-10, 1e-10]
    assert A.slice_choice(dE, 2.5e-10).tolist() == [True, True, False]


def test_non_finite_changes_stop_the_choice(built_lib):
    assert A.slice_choice([1e-12, np.nan, 2e-12], 1.0).tolist() == [True, False, True]
    assert not A.slice_choice([np.inf], 1e300).any()


def test_empty_and_bad_arguments(built_lib):
    assert A.slice_choice([], 1.0).size == 0
    import ctypes
    assert built_lib.ccsd_slice_choice(-1, None, 1.0, None) == 1
