"""Shared test helpers: full spin-orbital arrays <-> engine blocks, and the reference
semantics of an indexed-tensor statement restated in numpy (the planner's checker)."""
from __future__ import annotations

import itertools
import math

import numpy as np


def so_info(ctx, nout, nin):
    group = [0] * nout[0] + [1] * nout[1] + [2] * nin[0] + [3] * nin[1]
    space = [g % 2 for g in group]
    dims = [2 * ctx.total(s) for s in space]
    return group, space, dims


def index_spin_irrep(ctx, space, n):
    """spin and irrep of every full spin-orbital index of a space."""
    tot = ctx.total(space)
    spin = np.repeat([0, 1], tot)
    irr = np.concatenate([np.repeat(np.arange(ctx.nirrep), ctx._counts[(space, 0)])] * 2)
    return spin, irr


def random_so(ctx, nout, nin, rng, scale=1.0):
    """Random spin-orbital tensor (full array): spin-conserving, totally symmetric,
    antisymmetric inside each (space, upper/lower) group."""
    group, space, dims = so_info(ctx, nout, nin)
    X = rng.standard_normal(dims) * scale
    nd = len(dims)
    spins, irreps = [], []
    for p in range(nd):
        s, h = index_spin_irrep(ctx, space[p], dims[p])
        spins.append(s)
        irreps.append(h)
    # spin conservation: #alpha(lower) - #alpha(upper) = (nin - nout)/2
    nup = nout[0] + nout[1]
    alpha_up = sum(np.ix_(*[(1 - spins[p]) if p < nup else np.zeros(dims[p], int) for p in range(nd)]))
    alpha_lo = sum(np.ix_(*[(1 - spins[p]) if p >= nup else np.zeros(dims[p], int) for p in range(nd)]))
    want = (sum(nin) - sum(nout)) // 2
    mask = (alpha_lo - alpha_up) == want
    x = 0
    for p in range(nd):
        sh = [1] * nd
        sh[p] = dims[p]
        x = np.bitwise_xor(x, irreps[p].reshape(sh))
    mask = mask & (x == 0)
    X = X * mask
    # antisymmetrise within groups
    for g in range(4):
        pos = [p for p in range(nd) if group[p] == g]
        if len(pos) < 2:
            continue
        acc = np.zeros_like(X)
        for perm in itertools.permutations(range(len(pos))):
            axes = list(range(nd))
            for a, b in zip(pos, perm):
                axes[a] = pos[b]
            acc += perm_sign(perm) * np.transpose(X, axes)
        X = acc / math.factorial(len(pos))
    return X


def perm_sign(p):
    p = list(p)
    s = 1
    for i in range(len(p)):
        while p[i] != i:
            j = p[i]
            p[i], p[j] = p[j], p[i]
            s = -s
    return s


def write_full(T, full):
    """Write the canonical blocks of a full spin-orbital array into engine tensor T."""
    ctx = T.ctx
    for alpha in T.spin_cases():
        spins = T.case_spins(alpha)
        for irr in itertools.product(range(ctx.nirrep), repeat=T.ndim):
            x = 0
            for h in irr:
                x ^= h
            if x or T.block_size(alpha, irr) == 0:
                continue
            shape = T.block_shape(alpha, irr)
            sl = []
            for p in range(T.ndim):
                sp = T.group[p] % 2
                lo = ctx.spin_start(sp, spins[p]) + ctx.offset(sp, irr[p], spins[p])
                sl.append(slice(lo, lo + shape[p]))
            blk = full[tuple(sl)]
            if getattr(T, "packed", False):
                keys = np.arange(blk.size, dtype=np.int64)
                T.write(alpha, keys, blk.reshape(-1, order="F"), irreps=irr)
            else:
                T.write_block(alpha, blk, irr)


def shuffles(cpos_groups):
    """Antisymmetriser terms: list of (axis permutation of C, sign)."""
    per_group = []
    for pos, sub in cpos_groups:
        n = len(pos)
        terms = []
        if len(set(sub)) <= 1:
            terms.append((list(pos), 1))
        else:
            for perm in itertools.permutations(range(n)):
                ok = all(not (sub[a] == sub[b] and perm[a] > perm[b]) for a in range(n) for b in range(a + 1, n))
                if ok:
                    terms.append(([pos[perm[a]] for a in range(n)], perm_sign(perm)))
        per_group.append((pos, terms))
    out = []
    for combo in itertools.product(*[t for _, t in per_group]):
        m = {}
        sign = 1
        for (pos, _), (tgt, s) in zip(per_group, combo):
            for a, p in enumerate(pos):
                m[p] = tgt[a]
            sign *= s
        out.append((m, sign))
    return out


def reference_contract(alpha, A, ia, B, ib, beta, C, ic, groupC):
    """C = beta*C + alpha * P[ einsum(A,B) ] with the implicit antisymmetriser of
    src/tensor/spinorbital_tensor.cxx:637-669 restated over full arrays."""
    X = np.einsum(f"{ia},{ib}->{ic}", A, B)
    groups = []
    for g in range(4):
        pos = [p for p in range(len(ic)) if groupC[p] == g]
        if not pos:
            continue
        sub = [0 if ic[p] in ia else (1 if ic[p] in ib else 2) for p in pos]
        groups.append((pos, sub))
    acc = np.zeros_like(X)
    for m, sign in shuffles(groups):
        # letter at C position p is evaluated at C position m[p]
        axes = [0] * len(ic)
        for p in range(len(ic)):
            axes[m[p]] = p
        acc += sign * np.transpose(X, axes)
    return beta * C + alpha * acc


def _spin_cases(nout, nin):
    gs = [nout[0], nout[1], nin[0], nin[1]]
    out = []
    for a in itertools.product(*[range(g + 1) for g in gs]):
        if a[2] + a[3] == a[0] + a[1] + (sum(nin) - sum(nout)) // 2:
            out.append(a)
    return out


def _case_exists(nout, nin, spins):
    """spins per position -> does the spin case exist (spin conservation)"""
    group = [0] * nout[0] + [1] * nout[1] + [2] * nin[0] + [3] * nin[1]
    a = [0, 0, 0, 0]
    for p, s in enumerate(spins):
        if s == 0:
            a[group[p]] += 1
    return a[2] + a[3] == a[0] + a[1] + (sum(nin) - sum(nout)) // 2


def beta_mask(ctx, shapes, ia, ib, ic):
    """Full-array mask of C elements whose block receives beta: blocks (spin case, irrep
    tuple) of C for which some antisymmetriser term, internal spin and internal irrep
    assignment has symmetry-allowed A and B blocks (symblocked_tensor.cxx:1033-1062)."""
    (anout, anin), (bnout, bnin), (cnout, cnin) = shapes
    cgroup = [0] * cnout[0] + [1] * cnout[1] + [2] * cnin[0] + [3] * cnin[1]
    cspace = [g % 2 for g in cgroup]
    internal = sorted(set(ia) & set(ib))
    groups = []
    for g in range(4):
        pos = [p for p in range(len(ic)) if cgroup[p] == g]
        if pos:
            groups.append((pos, [0 if ic[p] in ia else (1 if ic[p] in ib else 2) for p in pos]))
    terms = shuffles(groups)
    dims = [2 * ctx.total(s) for s in cspace]
    mask = np.zeros(dims, dtype=bool)
    nirr = ctx.nirrep
    for case in _spin_cases((cnout[0], cnout[1]), (cnin[0], cnin[1])):
        cspins = []
        for g, gs in enumerate([cnout[0], cnout[1], cnin[0], cnin[1]]):
            cspins += [0] * case[g] + [1] * (gs - case[g])
        for cirr in itertools.product(range(nirr), repeat=len(ic)):
            x = 0
            for h in cirr:
                x ^= h
            if x:
                continue
            hit = False
            for m, _sign in terms:
                for ispin in itertools.product((0, 1), repeat=len(internal)):
                    for iirr in itertools.product(range(nirr), repeat=len(internal)):
                        sp, hh = {}, {}
                        for p in range(len(ic)):
                            sp[ic[p]] = cspins[m[p]]
                            hh[ic[p]] = cirr[m[p]]
                        for k, l in enumerate(internal):
                            sp[l] = ispin[k]
                            hh[l] = iirr[k]
                        xa = 0
                        for l in ia:
                            xa ^= hh[l]
                        xb = 0
                        for l in ib:
                            xb ^= hh[l]
                        if xa or xb:
                            continue
                        if not _case_exists(anout, anin, [sp[l] for l in ia]):
                            continue
                        if not _case_exists(bnout, bnin, [sp[l] for l in ib]):
                            continue
                        hit = True
                        break
                    if hit:
                        break
                if hit:
                    break
            if not hit:
                continue
            sl = []
            for p in range(len(ic)):
                lo = cspins[p] * ctx.total(cspace[p]) + ctx.offset(cspace[p], cirr[p])
                sl.append(slice(lo, lo + ctx.count(cspace[p], cspins[p], cirr[p])))
            # every arrangement of the block inside its groups shares the block's beta
            gpos = [[p for p in range(len(ic)) if cgroup[p] == g] for g in range(4)]
            for combo in itertools.product(*[list(itertools.permutations(gp)) for gp in gpos]):
                perm = list(range(len(ic)))
                for gp, pg in zip(gpos, combo):
                    for a_, b_ in zip(gp, pg):
                        perm[a_] = b_
                mask[tuple(sl[perm[q]] for q in range(len(ic)))] = True
    return mask


def write_fcidump(path, h, eri, nelec, ecore, all_images=False, full_fock=False, ms2=0):
    """Write spatial integrals as an FCIDUMP (1-based indices, canonical records
    p>=q, r>=s, pq>=rs unless all_images; h lower triangle unless full_fock)."""
    n = h.shape[0]
    lines = [f"&FCI NORB={n},NELEC={nelec},MS2={ms2},", "ORBSYM=" + "1," * n, "ISYM=1,", "&END"]
    for p in range(n):
        for q in range(n):
            for r in range(n):
                for s in range(n):
                    v = eri[p, q, r, s]
                    if v == 0.0:
                        continue
                    if not all_images and not (p >= q and r >= s and (p > r or (p == r and q >= s))):
                        continue
                    lines.append(f"{float(v)!r} {p + 1} {q + 1} {r + 1} {s + 1}")
    for p in range(n):
        for q in range(n):
            if full_fock or p >= q:
                if h[p, q] != 0.0:
                    lines.append(f"{float(h[p, q])!r} {p + 1} {q + 1} 0 0")
    lines.append(f"{float(ecore)!r} 0 0 0 0")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
