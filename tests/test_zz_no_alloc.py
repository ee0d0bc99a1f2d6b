"""solve_matrix_batched_noalloc: the batched solve for callers that cannot let a
library allocate device memory (a host code that reserves the GPU's memory for
its own arena, or must avoid the device-wide synchronisation of cudaMalloc /
cudaFree).  It must give the same results and codes as solve_matrix_batched,
call after call, while its factorisation scratch is a static device array
shared by every call.  This file is collected last so that a run stopping at
its first failure has already run every other test."""
import ctypes
from ctypes import c_void_p

import numpy as np
import pytest

from python_b200 import workloads as wl
from tests.helpers import same_values

pytestmark = pytest.mark.gpu

MAX_N = 512   # SIROCCO_NOALLOC_MAX_N


def _batch(seed):
    rng = np.random.default_rng(seed)
    sizes = [1, 2, 5, 27, 61, 129, 200, 301, MAX_N] + list(rng.integers(1, MAX_N + 1, 23))
    rng.shuffle(sizes)
    b = wl.dense_batch("solve", sizes, seed=seed, log_spread=3.0)
    # a singular system rides along: its code must come back as the reference's
    k = int(np.argmax(b.n > 3))
    o, n = int(b.offA[k]), int(b.n[k])
    m = b.A[o:o + n * n].reshape(n, n)
    m[1] = m[0]
    return b


def _reference(engine, batch):
    import torch
    dev = torch.device("cuda")
    A = torch.from_numpy(batch.A).to(dev)
    bb = torch.from_numpy(batch.b).to(dev)
    x = torch.full_like(bb, float("nan"))
    st = torch.full((batch.nsys,), -99, dtype=torch.int32, device=dev)
    n = np.ascontiguousarray(batch.n, np.int32)
    rc = engine.load().solve_matrix_batched(batch.nsys, n.ctypes.data_as(c_void_p), batch.offA.ctypes.data_as(c_void_p),
                                            c_void_p(A.data_ptr()), batch.offv.ctypes.data_as(c_void_p),
                                            c_void_p(bb.data_ptr()), c_void_p(x.data_ptr()), c_void_p(st.data_ptr()))
    assert rc == 0, engine.last_error()
    torch.cuda.synchronize()
    return x.cpu().numpy(), st.cpu().numpy()


def _noalloc(engine, batch, nmax, x=None):
    import torch
    dev = torch.device("cuda")
    n = torch.from_numpy(np.ascontiguousarray(batch.n, np.int32)).to(dev)
    oa = torch.from_numpy(batch.offA).to(dev)
    ov = torch.from_numpy(batch.offv).to(dev)
    A = torch.from_numpy(batch.A).to(dev)
    bb = torch.from_numpy(batch.b).to(dev)
    if x is None:
        x = torch.full_like(bb, float("nan"))
    st = torch.full((batch.nsys,), -99, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    rc = engine.load().solve_matrix_batched_noalloc(batch.nsys, nmax, c_void_p(n.data_ptr()), c_void_p(oa.data_ptr()),
                                                    c_void_p(A.data_ptr()), c_void_p(ov.data_ptr()),
                                                    c_void_p(bb.data_ptr()), c_void_p(x.data_ptr()),
                                                    c_void_p(st.data_ptr()), c_void_p(stream))
    torch.cuda.synchronize()
    return rc, x.cpu().numpy(), st.cpu().numpy()


def test_noalloc_matches_batched_entry_point_on_consecutive_calls(engine):
    # two different batches in a row, then the first again: each call must see
    # nothing of what the previous call left in the shared scratch
    b1, b2 = _batch(11), _batch(12)
    for batch in (b1, b2, b1):
        xr, sr = _reference(engine, batch)
        rc, x, st = _noalloc(engine, batch, int(batch.n.max()))
        assert rc == 0, engine.last_error()
        np.testing.assert_array_equal(st, sr)
        keep = np.repeat(sr != 4, batch.n)
        assert same_values(x[keep], xr[keep]).all()
        assert 4 in set(sr.tolist())


def test_noalloc_rejects_orders_beyond_its_scratch(engine):
    b = wl.dense_batch("solve", [MAX_N + 1], seed=3)
    rc, _, _ = _noalloc(engine, b, MAX_N + 1)
    assert rc == -2                      # SIROCCO_ESIZE
    assert "scratch" in engine.last_error()
    # a system larger than the nmax it was promised is refused, not overrun
    b = wl.dense_batch("solve", [40, 80], seed=4)
    rc, _, st = _noalloc(engine, b, 40)
    assert rc == 0 and st[0] == 0 and st[1] == -1


def test_noalloc_full_size_systems_share_slabs(engine):
    # at the largest order the static array holds 8 slabs, so 20 systems of
    # order 512 run on 8 CTAs that each reuse one slab for several systems
    b = wl.dense_batch("solve", [MAX_N] * 20, seed=21, log_spread=2.0)
    xr, sr = _reference(engine, b)
    for _ in range(2):
        rc, x, st = _noalloc(engine, b, MAX_N)
        assert rc == 0, engine.last_error()
        np.testing.assert_array_equal(st, sr)
        assert same_values(x, xr).all()


def test_noalloc_matches_the_oracle(engine):
    from oracle import oracle
    b = _batch(13)
    rc, x, st = _noalloc(engine, b, int(b.n.max()))
    assert rc == 0, engine.last_error()
    xo, so = oracle.solve(b, "port", threads=oracle.host_threads())
    np.testing.assert_array_equal(st, so)
    keep = np.repeat(so != 4, b.n)
    assert same_values(x[keep], xo[keep]).all()
