"""The allocation-free batched dot (ccsd_dot_batch_noalloc) against the regular entry
point.

It exists for callers that cannot let the library allocate device memory: an
application that owns all device memory through its own arena, or code that issues the
call while a stream is being captured into a CUDA graph.  The inputs and outputs here
are caller-owned device buffers (torch tensors); the regular path (ccsd_dot on engine
tensors holding the same values, which uses library-allocated reduction scratch) is the
reference.  Two calls in a row check that the shared fixed scratch carries nothing
over from one call to the next.  This file is collected last.
"""
import numpy as np
import pytest

import aquarius_b200 as A

pytestmark = pytest.mark.gpu

V, O = 300, 40          # "ai" tensors: alpha block + beta block = 2*V*O = 24000 values
TOL = 1e-12             # relative; the two paths sum in different orders


def _engine_dots(ctx, xs, ys):
    """ccsd_dot(X["ai"], Y_j["ai"]) for engine tensors holding xs / ys."""
    def tensor_of(vals):
        t = ctx.tensor("t", (1, 0), (0, 1))
        half = V * O
        t.write_block((1, 0, 0, 1), vals[:half].reshape((V, O), order="F"))   # alpha case
        t.write_block((0, 0, 0, 0), vals[half:].reshape((V, O), order="F"))   # beta case
        return t
    tx = tensor_of(xs)
    return np.array([ctx.dot(tx, "ai", tensor_of(y), "ai") for y in ys])


def _noalloc_dots(torch, xs, ys):
    dev = torch.device("cuda", 0)
    x = torch.from_numpy(xs).to(dev)
    yt = [torch.from_numpy(y).to(dev) for y in ys]
    out = torch.full((len(ys),), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    A.dot_batch_noalloc(stream.cuda_stream, x.data_ptr(), [y.data_ptr() for y in yt], x.numel(), out.data_ptr())
    stream.synchronize()
    return out.cpu().numpy()


def test_noalloc_dot_batch_matches_regular_entry_point_twice():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    rng = np.random.default_rng(2024)
    ctx = A.Context(0)
    try:
        ctx.set_spaces(vrt=[V], occ=[O])
        for ny in (7, 16):          # two calls in a row, different data and widths
            xs = rng.standard_normal(2 * V * O)
            ys = [rng.standard_normal(2 * V * O) for _ in range(ny)]
            ref = _engine_dots(ctx, xs, ys)
            got = _noalloc_dots(torch, xs, ys)
            assert np.all(np.isfinite(got))
            assert np.all(np.abs(got - ref) <= TOL * np.maximum(1.0, np.abs(ref))), (ny, got - ref)
    finally:
        ctx.close()


def test_noalloc_rejects_too_many_vectors():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    x = torch.zeros(8, dtype=torch.float64, device=dev)
    out = torch.zeros(17, dtype=torch.float64, device=dev)
    with pytest.raises(A.CcsdError) as e:
        A.dot_batch_noalloc(torch.cuda.current_stream(dev).cuda_stream, x.data_ptr(), [x.data_ptr()] * 17, 8,
                            out.data_ptr())
    assert e.value.code == 1 and "1..16" in str(e.value)
