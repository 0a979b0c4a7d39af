"""Host-side replay of a planned statement (test infrastructure).

Reads the text that ccsd_ctx_plan_export writes (record format: the header of
aquarius_b200/csrc/plan_export.cpp) and executes its steps with numpy over flat arrays in
the engine's block layout.  This checks the planner's expansion of a statement -- spin
cases, irrep blocks, pair restrictions, antisymmetriser images, lazy beta -- on the CPU,
against the interface semantics restated over full spin-orbital arrays (tests/helpers.py).
It is the checker only: nothing in the library calls it.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class BlockLayout:
    irrep: list
    len: list
    stride: list
    offset: int
    size: int
    pairs: list            # (p, q, kind, stride)


@dataclass
class TensorLayout:
    handle: int
    ndim: int
    total: int
    view_of: int
    name: str
    group: list = field(default_factory=list)
    cases: list = field(default_factory=list)     # (alpha[4], spin per position, [BlockLayout])


@dataclass
class PlanDump:
    scratch: int
    tensors: dict
    steps: list


def load(path) -> PlanDump:
    lines = open(path).read().splitlines()
    tensors, steps = {}, []
    scratch = 0
    cur = None
    i = 0

    def ints(line, tag):
        w = line.split()
        assert w[0] == tag, (tag, line)
        return np.array([int(x) for x in w[1:]], dtype=np.int64)

    while i < len(lines):
        w = lines[i].split()
        kind = w[0]
        if kind == "scratch":
            scratch = int(w[1])
        elif kind == "tensor":
            cur = TensorLayout(int(w[1]), int(w[2]), int(w[3]), int(w[4]), " ".join(w[6:]))
            tensors[cur.handle] = cur
        elif kind == "group":
            cur.group = [int(x) for x in w[1:]]
        elif kind == "case":
            cur.cases.append(([int(x) for x in w[1:5]], [int(x) for x in w[5:]], []))
        elif kind == "block":
            n = cur.ndim
            v = [int(x) for x in w[1:]]
            irrep, ln, st = v[:n], v[n:2 * n], v[2 * n:3 * n]
            off, size, npair = v[3 * n], v[3 * n + 1], v[3 * n + 2]
            pr = [tuple(v[3 * n + 3 + 4 * k:3 * n + 7 + 4 * k]) for k in range(npair)]
            cur.cases[-1][2].append(BlockLayout(irrep, ln, st, off, size, pr))
        elif kind == "gemm":
            tA, tB, tC, M, N, K = (int(x) for x in w[1:7])
            alpha = float(w[7])
            nvm, nvn = int(w[8]), int(w[9])
            vsign = [float(x) for x in w[10:14]]
            tabs = {}
            for tag in ("Am", "Ak", "Bk", "Bn", "Cm0", "Cm1", "Cn0", "Cn1"):
                i += 1
                tabs[tag] = ints(lines[i], tag)
            steps.append(("gemm", tA, tB, tC, M, N, K, alpha, nvm, nvn, vsign, tabs))
        elif kind in ("sum", "dot"):
            tA, tX, nd = int(w[1]), int(w[2]), int(w[3])
            alpha, offA, offX = float(w[4]), int(w[5]), int(w[6])
            ln = ints(lines[i + 1], "len")
            sA = ints(lines[i + 2], "sA")
            sX = ints(lines[i + 3], "sC" if kind == "sum" else "sB")
            i += 3
            steps.append((kind, tA, tX, nd, alpha, offA, offX, ln, sA, sX))
        elif kind == "scale":
            steps.append(("scale", int(w[1]), int(w[2]), int(w[3]), float(w[4])))
        else:
            raise ValueError(f"unknown record {kind!r}")
        i += 1
    return PlanDump(scratch, tensors, steps)


def _block_positions(b: BlockLayout):
    """(mask over the block's index grid, storage position of every grid point)"""
    grids = np.indices(b.len, dtype=np.int64) if b.len else np.zeros((0,), np.int64)
    pos = np.full(tuple(b.len), b.offset, dtype=np.int64)
    mask = np.ones(tuple(b.len), dtype=bool)
    in_pair = set()
    for p, q, kind, st in b.pairs:
        x, y = grids[p], grids[q]
        in_pair.update((p, q))
        if kind == 1:
            mask &= x < y
            pos = pos + st * (y * (y - 1) // 2 + x)
        else:
            pos = pos + st * (x + b.len[p] * y)
    for p in range(len(b.len)):
        if p not in in_pair:
            pos = pos + b.stride[p] * grids[p]
    return mask, pos


def _full_index(ctx, t: TensorLayout, spins, b: BlockLayout):
    idx = []
    for p in range(t.ndim):
        sp = t.group[p] % 2
        lo = ctx.spin_start(sp, spins[p]) + ctx.offset(sp, b.irrep[p], spins[p])
        idx.append(lo + np.arange(b.len[p]))
    return np.ix_(*idx)


def to_storage(ctx, t: TensorLayout, full):
    """Flat storage of a full spin-orbital array in the tensor's block layout."""
    st = np.zeros(max(t.total, 1))
    for _, spins, blocks in t.cases:
        for b in blocks:
            if b.size == 0:
                continue
            mask, pos = _block_positions(b)
            st[pos[mask]] = full[_full_index(ctx, t, spins, b)][mask]
    return st


def replay(dump: PlanDump, store: dict):
    """Execute the steps on `store` (handle -> flat array; views read their base's array).
    Returns the sum of the dot steps."""
    scratch = np.zeros(max(dump.scratch, 1))

    def arr(h):
        if h == -1:
            return scratch
        t = dump.tensors[h]
        return store[t.view_of if t.view_of else h]

    acc = 0.0
    for s in dump.steps:
        if s[0] == "gemm":
            _, tA, tB, tC, M, N, K, alpha, nvm, nvn, vsign, tb = s
            Am = arr(tA)[tb["Am"][:, None] + tb["Ak"][None, :]]
            Bm = arr(tB)[tb["Bk"][:, None] + tb["Bn"][None, :]]
            P = alpha * (Am @ Bm)
            C = arr(tC)
            for im in range(nvm):
                for jn in range(nvn):
                    where = tb["Cm%d" % im][:, None] + tb["Cn%d" % jn][None, :]
                    np.add.at(C, where, vsign[im * nvn + jn] * P)
        elif s[0] in ("sum", "dot"):
            kind, tA, tX, nd, alpha, offA, offX, ln, sA, sX = s
            g = np.indices(tuple(ln), dtype=np.int64).reshape(nd, -1)
            ia = offA + (sA[:, None] * g).sum(axis=0)
            ix = offX + (sX[:, None] * g).sum(axis=0)
            if kind == "sum":
                np.add.at(arr(tX), ix, alpha * arr(tA)[ia])
            else:
                acc += alpha * float(np.dot(arr(tA)[ia], arr(tX)[ix]))
        else:
            _, tC, off, n, beta = s
            C = arr(tC)
            if beta == 0.0:
                C[off:off + n] = 0.0
            else:
                C[off:off + n] *= beta
    return acc
