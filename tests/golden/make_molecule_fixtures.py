"""Generate tests/golden/molecules.json from the reference's end-to-end test inputs.

Reads, from a checkout of the reference (path given as the first argument):
  * test/input.aq     -- the sections whose CCSD energy the reference checks
                         (h2o-pvdz: lines 1-24, ch2-pvdz: lines 47-71): geometry (bohr),
                         multiplicity, basis-set name and the compared SCF / MP2 / CCSD
                         and Lambda-CCSD energies with their tolerance;
  * basis/<name>      -- the contracted shells of every element used.
Writes a small JSON fixture so that the tests never read the reference at run time.

usage: python tests/golden/make_molecule_fixtures.py <reference-checkout>
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import scf  # noqa: E402

SECTIONS = ["h2o-pvdz", "ch2-pvdz"]
KEYS = {"localaoscf:energy": "scf", "ccsd:mp2": "mp2", "ccsd:energy": "ccsd", "lambdaccsd:energy": "lambda"}


def parse_sections(text):
    out = {}
    lines = text.splitlines()
    i = 0
    while i < len(lines):
        m = re.match(r"\s*section\s+(\S+)", lines[i])
        if not m:
            i += 1
            continue
        name, start = m.group(1), i + 1
        j = start
        while j < len(lines) and not re.match(r"\s*section\s+", lines[j]):
            j += 1
        body = lines[start - 1:j]
        atoms, mult, basis, known = [], 1, None, {}
        for ln in body:
            a = re.search(r"atom\s*\{\s*(\w+)\s*,\s*([-\d.]+)\s*,\s*([-\d.]+)\s*,\s*([-\d.]+)\s*\}", ln)
            if a:
                atoms.append([a.group(1), float(a.group(2)), float(a.group(3)), float(a.group(4))])
            m2 = re.search(r"multiplicity\s+(\d+)", ln)
            if m2:
                mult = int(m2.group(1))
            b = re.search(r"basis_set\s+(\S+)", ln)
            if b:
                basis = b.group(1)
            c = re.search(r"val1 from\s+(\S+)\s*,\s*using val2\s*=\s*([-\d.]+)\s*,\s*tolerance\s+([\d.eE+-]+)", ln)
            if c and c.group(1) in KEYS:
                known[KEYS[c.group(1)]] = float(c.group(2))
                known["tolerance"] = float(c.group(3))
        out[name] = {"atoms": atoms, "multiplicity": mult, "basis_set": basis, "known": known,
                     "source": f"test/input.aq:{start}-{j}"}
        i = j
    return out


def main(ref_root):
    ref = Path(ref_root)
    sections = parse_sections((ref / "test" / "input.aq").read_text())
    fixture = {"units": "bohr", "molecules": {}, "basis": {}}
    for name in SECTIONS:
        s = sections[name]
        fixture["molecules"][name] = s
        bname = s["basis_set"]
        text = (ref / "basis" / bname).read_text()
        bs = fixture["basis"].setdefault(bname, {})
        for sym in {a[0].upper() for a in s["atoms"]}:
            bs[sym] = [[l, list(map(float, e)), list(map(float, c))] for l, e, c in scf.parse_basis(text, sym)]
    (HERE / "molecules.json").write_text(json.dumps(fixture, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_molecule_fixtures.py <path of the reference checkout>")
    main(sys.argv[1])
