"""C-ABI boundary: the library builds, loads, and exports every declared entry point
(no device calls)."""
import re
from pathlib import Path

import aquarius_b200 as A

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "ccsd_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ccsd_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_expected_entry_points():
    assert set(declared_symbols()) == set(A.EXPORTS)


def test_library_exports_every_declared_symbol(built_lib):
    for name in declared_symbols():
        assert hasattr(built_lib, name), name


def test_context_create_without_device_fails_cleanly(built_lib):
    import torch
    if torch.cuda.is_available():
        return
    import pytest
    with pytest.raises(A.CcsdError):
        A.Context(0)


def test_options_defaults_match_reference_spec(built_lib):
    # src/cc/ccsd.cxx:267-287: convergence 1e-9, max_iterations 50, diis order 5 start 1 damping 0
    o = A.Options()
    built_lib.ccsd_options_default(o)
    assert o.conv_tol == 1e-9 and o.max_iter == 50
    assert o.diis_order == 5 and o.diis_start == 1 and o.diis_damping == 0.0
