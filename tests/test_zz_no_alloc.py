"""The allocation-free batched dot (ccsd_dot_batch_noalloc) against the regular entry
point and against numpy.

It exists for callers that cannot let the library allocate device memory: an
application that owns all device memory through its own arena or pool and forbids
libraries to allocate behind its back.  The inputs and outputs here are caller-owned
device buffers (torch tensors); the regular path (ccsd_dot on engine tensors holding
the same values, which uses library-allocated reduction scratch) and a numpy dot of the
same host arrays are the references.  Two calls in a row check that the shared fixed
scratch carries nothing over from one call to the next, and the device's free memory
is the same before and after further calls.  This file is collected last.
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
            host = np.array([np.dot(xs, y) for y in ys])
            assert np.all(np.isfinite(got))
            assert np.all(np.abs(got - ref) <= TOL * np.maximum(1.0, np.abs(ref))), (ny, got - ref)
            assert np.all(np.abs(got - host) <= TOL * np.maximum(1.0, np.abs(host))), (ny, got - host)
    finally:
        ctx.close()


def test_noalloc_calls_leave_free_device_memory_unchanged():
    """After a first call (which may load the kernels), further calls change the device's
    free memory by nothing: every buffer here is allocated before the measurement."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(7)
    n, ny = 1 << 20, 16
    x = torch.from_numpy(rng.standard_normal(n)).to(dev)
    ys = [torch.from_numpy(rng.standard_normal(n)).to(dev) for _ in range(ny)]
    out = torch.zeros(ny, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    call = lambda: A.dot_batch_noalloc(stream.cuda_stream, x.data_ptr(), [y.data_ptr() for y in ys], n,
                                       out.data_ptr())
    call()
    stream.synchronize()
    free0, _ = torch.cuda.mem_get_info(dev)
    for _ in range(5):
        call()
    stream.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0, (free0, free1)
    xh = x.cpu().numpy()
    host = np.array([np.dot(xh, y.cpu().numpy()) for y in ys])
    got = out.cpu().numpy()
    assert np.all(np.abs(got - host) <= TOL * np.maximum(1.0, np.abs(host)))


def test_noalloc_rejects_too_many_vectors():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    x = torch.zeros(8, dtype=torch.float64, device=dev)
    out = torch.zeros(17, dtype=torch.float64, device=dev)
    with pytest.raises(A.CcsdError) as e:
        A.dot_batch_noalloc(torch.cuda.current_stream(dev).cuda_stream, x.data_ptr(), [x.data_ptr()] * 17, 8,
                            out.data_ptr())
    assert e.value.code == 1 and "1..16" in str(e.value)
