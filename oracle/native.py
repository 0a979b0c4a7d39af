"""Build and load the oracle's C integral code (gaussian_ints.c).

TEST INFRASTRUCTURE ONLY: part of the oracle.  `build()` compiles the C source with
gcc into oracle/_build/libgints.so; `lib()` loads it with ctypes.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "gaussian_ints.c"
OUT = HERE / "_build" / "libgints.so"

_lib = None


def build() -> Path:
    OUT.parent.mkdir(exist_ok=True)
    if not OUT.exists() or SRC.stat().st_mtime > OUT.stat().st_mtime:
        tmp = OUT.with_suffix(".so.tmp")
        subprocess.run(["gcc", "-O2", "-shared", "-fPIC", "-std=gnu99", "-Wall", str(SRC), "-o", str(tmp), "-lm"],
                       check=True)
        tmp.replace(OUT)
    return OUT


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(OUT))
        vp, i = ctypes.c_void_p, ctypes.c_int
        L.one_electron.argtypes = [i, vp, vp, vp, vp, vp, i, vp, vp, vp, vp, vp]
        L.one_electron.restype = i
        L.two_electron.argtypes = [i, vp, vp, vp, vp, vp, vp]
        L.two_electron.restype = i
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def cartesian_integrals(shells, charges, nuclei):
    """S, T, V (n x n) and (mu nu|la si) (n^4) over Cartesian shell components.

    shells: list of (l, center[3], exps[], coefs[]) with coefs including primitive norms.
    """
    L = lib()
    l = np.array([s[0] for s in shells], dtype=np.int32)
    npr = np.array([len(s[2]) for s in shells], dtype=np.int32)
    cen = np.ascontiguousarray(np.array([s[1] for s in shells], dtype=np.float64).reshape(-1))
    ex = np.ascontiguousarray(np.concatenate([np.asarray(s[2], dtype=np.float64) for s in shells]))
    co = np.ascontiguousarray(np.concatenate([np.asarray(s[3], dtype=np.float64) for s in shells]))
    n = int(sum((x + 1) * (x + 2) // 2 for x in l))
    Z = np.ascontiguousarray(np.asarray(charges, dtype=np.float64))
    C = np.ascontiguousarray(np.asarray(nuclei, dtype=np.float64).reshape(-1))
    S, T, V = (np.zeros((n, n)) for _ in range(3))
    L.one_electron(len(shells), _p(l), _p(npr), _p(cen), _p(ex), _p(co), len(Z), _p(Z), _p(C), _p(S), _p(T), _p(V))
    eri = np.zeros((n, n, n, n))
    L.two_electron(len(shells), _p(l), _p(npr), _p(cen), _p(ex), _p(co), _p(eri))
    return S, T, V, eri
