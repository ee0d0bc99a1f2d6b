"""Host-side validation of the batched entry points: malformed layouts, null
pointers and unknown modes are refused with a library code before anything
touches the device, so these tests need no GPU.  The contract they protect is
the reference's failure behaviour for bad calls (source/matrix_cpu.c:134-146):
an error code, never a read or write outside the caller's buffers."""
import ctypes
from ctypes import c_int, c_void_p

import numpy as np
import pytest

from python_b200 import build, engine

EINVAL, ESIZE, EMODE = -1, -2, -3


@pytest.fixture(scope="module")
def lib():
    build.build_engine()
    return engine.load()


def ptr(a):
    return None if a is None else a.ctypes.data_as(c_void_p)


def layout(sizes, gap=0):
    n = np.array(sizes, np.int32)
    offA = np.zeros(n.size, np.int64)
    offv = np.zeros(n.size, np.int64)
    if n.size > 1:
        offA[1:] = np.cumsum(n[:-1].astype(np.int64) ** 2 + gap)
        offv[1:] = np.cumsum(n[:-1].astype(np.int64) + gap)
    return n, offA, offv


def solve(lib, n, offA, offv, A=None, b=None, x=None, st=None, nsys=None):
    nsys = n.size if nsys is None else nsys
    A = np.zeros(max(1, int((offA + n.astype(np.int64) ** 2).max()))) if A is None else A
    b = np.zeros(max(1, int((offv + n).max()))) if b is None else b
    x = np.zeros_like(b) if x is None else x
    st = np.zeros(max(1, n.size), np.int32) if st is None else st
    return lib.solve_matrix_batched(nsys, ptr(n), ptr(offA), ptr(A), ptr(offv), ptr(b), ptr(x), ptr(st))


def invert(lib, n, offA, A=None, out=None, st=None, nsys=None):
    nsys = n.size if nsys is None else nsys
    A = np.zeros(max(1, int((offA + n.astype(np.int64) ** 2).max()))) if A is None else A
    out = np.zeros_like(A) if out is None else out
    st = np.zeros(max(1, n.size), np.int32) if st is None else st
    return lib.invert_matrix_batched(nsys, ptr(n), ptr(offA), ptr(A), ptr(out), ptr(st))


def test_zero_order_is_refused(lib):
    n, oa, ov = layout([3, 0, 2])
    assert solve(lib, n, oa, ov) == EINVAL
    assert invert(lib, n, oa) == EINVAL
    assert "order 0" in engine.last_error()


def test_order_beyond_the_engine_is_refused(lib):
    n, oa, ov = layout([3, 1025])
    assert solve(lib, n, oa, ov) == ESIZE
    assert invert(lib, n, oa) == ESIZE


def test_negative_count_and_null_pointers(lib):
    n, oa, ov = layout([3, 4])
    assert solve(lib, n, oa, ov, nsys=-1) == EINVAL
    assert lib.solve_matrix_batched(2, None, ptr(oa), ptr(np.zeros(25)), ptr(ov), ptr(np.zeros(7)),
                                    ptr(np.zeros(7)), ptr(np.zeros(2, np.int32))) == EINVAL
    assert lib.solve_matrix_batched(2, ptr(n), ptr(oa), ptr(np.zeros(25)), None, ptr(np.zeros(7)),
                                    ptr(np.zeros(7)), ptr(np.zeros(2, np.int32))) == EINVAL
    assert lib.solve_matrix_batched(2, ptr(n), ptr(oa), ptr(np.zeros(25)), ptr(ov), None,
                                    ptr(np.zeros(7)), ptr(np.zeros(2, np.int32))) == EINVAL
    assert lib.invert_matrix_batched(2, ptr(n), ptr(oa), None, ptr(np.zeros(25)),
                                     ptr(np.zeros(2, np.int32))) == EINVAL
    assert lib.invert_matrix_batched(2, ptr(n), ptr(oa), ptr(np.zeros(25)), ptr(np.zeros(25)), None) == EINVAL


def test_empty_batch_is_a_no_op(lib):
    n, oa, ov = layout([])
    assert lib.solve_matrix_batched(0, None, None, None, None, None, None, None) == 0
    assert lib.invert_matrix_batched(0, None, None, None, None, None) == 0


def test_negative_offsets_are_refused(lib):
    n, oa, ov = layout([3, 4])
    oa2 = oa.copy()
    oa2[1] = -16
    assert invert(lib, n, oa2, A=np.zeros(25)) == EINVAL
    assert solve(lib, n, oa2, ov, A=np.zeros(25)) == EINVAL
    ov2 = ov.copy()
    ov2[0] = -3
    assert solve(lib, n, oa, ov2, b=np.zeros(7)) == EINVAL
    assert "negative offset" in engine.last_error()


def test_overlapping_outputs_are_refused(lib):
    n, oa, ov = layout([3, 4])
    oa2 = oa.copy()
    oa2[1] = 8                                   # the second inverse starts inside the first
    assert invert(lib, n, oa2, A=np.zeros(24)) == EINVAL
    assert "overlap" in engine.last_error()
    ov2 = ov.copy()
    ov2[1] = 2                                   # the second solution overlaps the first
    assert solve(lib, n, oa, ov2, b=np.zeros(6)) == EINVAL
    # unsorted but disjoint inverses pass the layout check
    n3, oa3, _ = layout([2, 2, 2])
    oa3 = oa3[::-1].copy()
    rc = invert(lib, n3, oa3)
    assert rc not in (EINVAL, ESIZE, EMODE)


def test_solve_matrices_may_share_storage(lib):
    # matrices are only read: two systems may use the same A
    n = np.array([3, 3], np.int32)
    oa = np.zeros(2, np.int64)
    ov = np.array([0, 3], np.int64)
    rc = solve(lib, n, oa, ov, A=np.eye(3).ravel().copy(), b=np.ones(6))
    assert rc not in (EINVAL, ESIZE, EMODE)


def test_unknown_precision_mode(lib):
    assert lib.sirocco_set_precision(7) == EMODE
    n, oa, ov = layout([3])
    h = c_void_p()
    assert lib.sirocco_plan_create(ctypes.byref(h), 1, 1, ptr(n), ptr(oa), ptr(ov), 7) == EMODE
    assert lib.sirocco_plan_create(ctypes.byref(h), 5, 1, ptr(n), ptr(oa), ptr(ov), 0) == EINVAL


def test_plan_layout_checked_before_the_device(lib):
    n, oa, ov = layout([3, 4])
    oa[1] = -1
    h = c_void_p()
    assert lib.sirocco_plan_create(ctypes.byref(h), 1, 2, ptr(n), ptr(oa), ptr(ov), 0) == EINVAL
    assert lib.sirocco_plan_create(None, 1, 2, ptr(n), ptr(oa), ptr(ov), 0) == EINVAL


def test_matom_layout_checked(lib):
    n, oa, ov = layout([3, 4])
    ov[1] = -2
    N = np.zeros(25)
    R = np.zeros(7)
    assert lib.matom_matrices_batched(2, ptr(n), ptr(oa), ptr(ov), ptr(N), ptr(R), ptr(np.zeros(25)), None,
                                      ptr(np.zeros(2, np.int32))) == EINVAL
