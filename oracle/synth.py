"""Seeded synthetic closed-shell problem, restated in numpy.

TEST INFRASTRUCTURE ONLY (the checker side; see ccsd_oracle.py).  The CPU legs of the
benchmark and the CPU tests build their inputs here, so that they load nothing of the
engine's library.  It restates the engine's generator value for value:

  orbital energies  occ ~ U[-1.2,-0.4] Eh, vrt ~ U[0.3,4.0] Eh, sorted ascending within
                    each irrep, Fock = diag(eps) (occupied first, irrep-major);
  factor            B[P,p,q] = B[P,q,p] = N(0,1) * 0.25/sqrt(NP) * exp(-|p-q|/n), NP = 3 n,
                    nonzero only when irrep(P) = irrep(p) ^ irrep(q);
  irrep counts      (D2h) a Dirichlet(1.5) split of o, v and NP (Marsaglia-Tsang gamma
                    draws), rounded with largest remainders, every irrep at least one.

Every value comes from a counter-based draw: the splitmix64 finaliser applied to a hash
of (seed, stream, index), so any element can be produced on its own.  Uniforms take the
top 53 bits; normals are one Box-Muller pair per index.  tests/test_synth.py checks that
this module and ccsd_synth_problem give identical bits.
"""
from __future__ import annotations

import math

import numpy as np

_GOLD = np.uint64(0x9E3779B97F4A7C15)
_C1 = np.uint64(0xBF58476D1CE4E5B9)
_C2 = np.uint64(0x94D049BB133111EB)
_SEEDMUL = 0xD1B54A32D192ED03
_IDXMUL = np.uint64(0x8CB92BA72F3D8DD7)


def _mix64(z):
    """splitmix64 finaliser on uint64 arrays (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        z = z + _GOLD
        z = (z ^ (z >> np.uint64(30))) * _C1
        z = (z ^ (z >> np.uint64(27))) * _C2
        return z ^ (z >> np.uint64(31))


def _draw(seed: int, stream: int, idx):
    base = _mix64(np.array([(seed * _SEEDMUL + stream) & ((1 << 64) - 1)], dtype=np.uint64))[0]
    with np.errstate(over="ignore"):
        return _mix64(base ^ (np.asarray(idx, dtype=np.uint64) * _IDXMUL))


def uniform(seed: int, stream: int, idx):
    """U[0,1): the top 53 bits of the draw times 2^-53."""
    return (_draw(seed, stream, idx) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def _libm(f, x):
    """f applied element by element through the C library (Python's math module): numpy's
    vectorised log and exp differ from it in the last bit for some arguments."""
    x = np.asarray(x, dtype=np.float64)
    return np.fromiter(map(f, x.ravel().tolist()), dtype=np.float64, count=x.size).reshape(x.shape)


def gauss(seed: int, stream: int, idx):
    """N(0,1), Box-Muller over the draws 2*idx and 2*idx+1."""
    idx = np.asarray(idx, dtype=np.uint64)
    u1 = 1.0 - uniform(seed, stream, np.uint64(2) * idx)
    u2 = uniform(seed, stream, np.uint64(2) * idx + np.uint64(1))
    return np.sqrt(-2.0 * _libm(math.log, u1)) * _libm(math.cos, 6.283185307179586 * u2)


def _gauss1(seed, stream, idx):
    u1 = 1.0 - float(uniform(seed, stream, 2 * idx))
    u2 = float(uniform(seed, stream, 2 * idx + 1))
    return math.sqrt(-2.0 * math.log(u1)) * math.cos(6.283185307179586 * u2)


def _gamma(seed, stream, ctr, alpha):
    d = alpha - 1.0 / 3.0
    c = 1.0 / math.sqrt(9.0 * d)
    for _ in range(1000):
        x = _gauss1(seed, stream, ctr)
        ctr += 1
        v = 1.0 + c * x
        if v <= 0:
            continue
        v = v * v * v
        u = float(uniform(seed, stream + 1000, ctr))
        ctr += 1
        if math.log(u) < 0.5 * x * x + d - d * v + d * math.log(v):
            return d * v, ctr
    return d, ctr


def dirichlet_split(seed: int, stream: int, total: int, nirrep: int):
    if nirrep == 1:
        return [total]
    g, ctr = [], 0
    for _ in range(nirrep):
        x, ctr = _gamma(seed, stream, ctr, 1.5)
        g.append(x)
    s = 0.0
    for x in g:
        s += x
    rest = total - nirrep
    share = [rest * x / s for x in g]
    cnt = [int(math.floor(x)) for x in share]
    used = sum(cnt)
    order = sorted(range(nirrep), key=lambda h: -(share[h] - cnt[h]))   # stable, like std::stable_sort
    k = 0
    while used < rest:
        cnt[order[k % nirrep]] += 1
        k += 1
        used += 1
    return [c + 1 for c in cnt]


def synth_irreps(seed: int, nirrep: int, o: int, v: int):
    """(occ, vrt, aux) orbital counts per irrep."""
    if nirrep not in (1, 2, 4, 8) or o < nirrep or v < nirrep:
        raise ValueError("nirrep must be 1, 2, 4 or 8 with at least one orbital per irrep")
    naux = 3 * (o + v)
    return (np.array(dirichlet_split(seed, 4, o, nirrep), np.int32),
            np.array(dirichlet_split(seed, 5, v, nirrep), np.int32),
            np.array(dirichlet_split(seed, 6, naux, nirrep), np.int32))


def synth_problem(seed: int, o: int, v: int, nirrep: int = 1, with_B: bool = True):
    """(eps[n], B[naux, n, n] or None, occ, vrt, aux): the engine's synth_problem."""
    if nirrep == 1:
        occ, vrt = np.array([o], np.int32), np.array([v], np.int32)
        aux = np.array([3 * (o + v)], np.int32)
    else:
        occ, vrt, aux = synth_irreps(seed, nirrep, o, v)
    n = o + v
    naux = int(aux.sum())
    irr = np.concatenate([np.repeat(np.arange(nirrep), occ), np.repeat(np.arange(nirrep), vrt)])
    auxirr = np.repeat(np.arange(nirrep), aux)
    p = np.arange(n)
    eps = np.where(p < o, -1.2 + 0.8 * uniform(seed, 1, p), 0.3 + 3.7 * uniform(seed, 2, p))
    start = 0
    for cnts in (occ, vrt):
        for c in cnts:
            eps[start:start + c] = np.sort(eps[start:start + c])
            start += c
    B = None
    if with_B:
        scale = 0.25 / math.sqrt(naux)
        B = np.zeros((naux, n, n))
        pp, qq = np.triu_indices(n)
        damp = _libm(math.exp, -np.arange(n, dtype=np.float64) / n)[qq - pp]
        for P in range(naux):
            keep = (irr[pp] ^ irr[qq]) == auxirr[P]
            idx = (np.uint64(P) * np.uint64(n) + pp.astype(np.uint64)) * np.uint64(n) + qq.astype(np.uint64)
            val = np.where(keep, gauss(seed, 3, idx) * scale * damp, 0.0)
            B[P, pp, qq] = val
            B[P, qq, pp] = val
    return eps, B, occ, vrt, aux
