"""FCIDUMP parsing on the host (ccsd_fcidump_read), no device needed.

Semantics checked against src/operator/fcidump.cxx:50-277: header keys, core energy,
skipped orbital-energy records, mirrored one-electron records (unless "1eints full"),
two-electron records taken from their canonical image only and set on all eight.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from helpers import write_fcidump

FIXTURE = json.loads((Path(__file__).parent / "golden" / "molecules.json").read_text())


@pytest.fixture(scope="module")
def h2o_mo():
    from oracle import scf
    res, H, eri = scf.solve_scf(FIXTURE, "h2o-pvdz")
    h, mo = scf.mo_integrals(res, H, eri)
    return res, h, mo


def test_round_trip_canonical_records(built_lib, h2o_mo, tmp_path):
    import aquarius_b200 as A
    res, h, mo = h2o_mo
    p = tmp_path / "FCIDUMP"
    write_fcidump(p, h, mo, nelec=10, ecore=res.enuc)
    d = A.fcidump_read(p)
    assert d["norb"] == 24 and d["nelec"] == 10
    assert d["ecore"] == res.enuc
    assert np.array_equal(d["h"], h)
    assert np.array_equal(d["eri"], mo)


def test_all_images_and_full_fock_give_the_same_arrays(built_lib, h2o_mo, tmp_path):
    import aquarius_b200 as A
    res, h, mo = h2o_mo
    p = tmp_path / "FCIDUMP.all"
    write_fcidump(p, h, mo, nelec=10, ecore=res.enuc, all_images=True, full_fock=True)
    d = A.fcidump_read(p, full_fock=True)
    assert np.array_equal(d["eri"], mo)
    assert np.array_equal(d["h"], h)
    # the full one-electron matrix read in the symmetric mode double-counts off-diagonals
    d2 = A.fcidump_read(p)
    off = ~np.eye(24, dtype=bool)
    assert np.array_equal(d2["h"][off], 2 * h[off])


def test_header_variants_and_orbital_energy_records(built_lib, tmp_path):
    import aquarius_b200 as A
    p = tmp_path / "FCIDUMP.small"
    p.write_text(" $fci norb = 2 , nelec= 2,\n  orbsym=1,1,\n $end\n"
                 "0.5 1 1 1 1\n0.25 2 1 1 1\n0.125 1 1 2 1\n"
                 "-1.0 1 1 0 0\n-0.5 2 1 0 0\n"
                 "-0.7 1 0 0 0\n"
                 "1.5D+00 0 0 0 0\n")
    d = A.fcidump_read(p)
    assert d["norb"] == 2 and d["nelec"] == 2 and d["ecore"] == 1.5
    eri = d["eri"]
    assert eri[0, 0, 0, 0] == 0.5
    # (21|11) is canonical: all eight images; (11|21) is its pair-swapped image: skipped
    for idx in [(1, 0, 0, 0), (0, 1, 0, 0), (0, 0, 1, 0), (0, 0, 0, 1)]:
        assert eri[idx] == 0.25
    assert np.array_equal(d["h"], np.array([[-1.0, -0.5], [-0.5, 0.0]]))


@pytest.mark.parametrize("text,msg", [
    ("&FCI NELEC=2,\n&END\n", "NORB"),
    ("&FCI NORB=2,\n&END\n", "NELEC"),
    ("&FCI NORB=2, NELEC=2\n", "terminator"),
    ("&FCI NORB=2, NELEC=2,\n&END\n0.5 1 1 3 1\n", "out of range"),
    ("&FCI NORB=2, NELEC=2,\n&END\n0.5 1 1\n", "malformed"),
])
def test_bad_files_are_rejected(built_lib, tmp_path, text, msg):
    import aquarius_b200 as A
    p = tmp_path / "FCIDUMP.bad"
    p.write_text(text)
    with pytest.raises(A.CcsdError, match=msg):
        A.fcidump_read(p)


def test_missing_file(built_lib, tmp_path):
    import aquarius_b200 as A
    with pytest.raises(A.CcsdError, match="cannot open"):
        A.fcidump_read(tmp_path / "nope")
