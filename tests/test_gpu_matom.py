"""Macro-atom epilogue and draws on the GPU (matom_matrices_batched,
matom_sample_batched) against the reference's formulas: B = N^-1 diag(R)
(source/macro_accelerate.c:325-334) and the running-total walk of
matom_deactivation_from_matrix (macro_accelerate.c:995-1008)."""
import ctypes

import numpy as np
import pytest

from oracle import oracle
from python_b200 import workloads as wl

SIZES = [5, 20, 33, 61, 61, 64, 65, 96, 128, 150, 200, 256, 300]


def reference_walk(row_b, z):
    """matom_deactivation_from_matrix's loop on one row of B."""
    j, total = 0, 0.0
    while total < z:
        if j == len(row_b):
            return -1
        total += row_b[j]
        j += 1
    return j - 1 if j > 0 else 0


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["FP64", "FAST"])
def test_matom_matrices_match_inverse_times_r(engine, mode):
    """B equals the engine's own inverse in the same mode times R, bit for bit,
    and C its left-to-right running totals; in SIROCCO_FAST the certified
    kernel forms both itself (orders 33-224 here), the GSL-exact path and the
    epilogue kernel the rest."""
    m = getattr(engine, mode)
    batch, R, offv = wl.matom_cells(SIZES, seed=11)
    B, C, st = engine.matom_matrices(batch, R, offv, mode=m)
    inv, sti = engine.invert_batched(batch, m)
    ir, sr = oracle.invert(batch, "port", threads=oracle.host_threads())
    np.testing.assert_array_equal(st, sti)
    np.testing.assert_array_equal(st, sr)
    for s in range(batch.nsys):
        n, o, v = int(batch.n[s]), int(batch.offA[s]), int(offv[s])
        r = R[v:v + n]
        b = B[o:o + n * n].reshape(n, n)
        # bit for bit: the engine's own inverse times R, and the left-to-right running totals
        want = inv[o:o + n * n].reshape(n, n) * r[None, :]
        assert np.array_equal(b, want), s
        assert np.array_equal(C[o:o + n * n].reshape(n, n), np.cumsum(b, axis=1)), s
        # against the GSL inverse: rounding only
        ref = ir[o:o + n * n].reshape(n, n) * r[None, :]
        assert np.max(np.abs(b - ref)) <= 1e-12 * np.max(np.abs(ref)), s
        # absorbing probabilities: every row of B sums to one
        assert np.allclose(b.sum(axis=1), 1.0, rtol=0, atol=1e-10), s


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["FP64", "FAST"])
def test_matom_singular_cell_gives_zero_matrices(engine, mode):
    batch, R, offv = wl.matom_cells([12, 40], seed=3)
    m = batch.matrix(1).copy()
    m[7] = 0.0                       # a zero row: exactly singular
    mats = [batch.matrix(0), m]
    sb = wl.from_matrices("invert", mats)
    B, C, st = engine.matom_matrices(sb, R, offv, mode=getattr(engine, mode))
    _, sr = oracle.invert(sb, "port", threads=1)
    np.testing.assert_array_equal(st, sr)
    assert st[1] == 1 and st[0] == 0
    o = int(sb.offA[1])
    assert (B[o:o + 1600] == 0).all() and (C[o:o + 1600] == 0).all()


@pytest.mark.gpu
def test_matom_draws_follow_the_reference_walk(engine):
    batch, R, offv = wl.matom_cells(SIZES, seed=5)
    B, C, st = engine.matom_matrices(batch, R, offv)
    rng = np.random.default_rng(9)
    nq = 20000
    sys = rng.integers(0, batch.nsys, nq).astype(np.int32)
    level = np.array([rng.integers(0, batch.n[s]) for s in sys], np.int32)
    z = rng.random(nq)
    # exact hits on running totals, the ends of the interval and bad queries
    for i in range(0, 200):
        s, u = int(sys[i]), int(level[i])
        n, o = int(batch.n[s]), int(batch.offA[s])
        z[i] = C[o + u * n + int(rng.integers(0, n))]
    z[200], z[201], z[202] = 0.0, -1.0, 1.5
    level[203], sys[204] = -1, batch.nsys
    t = engine.matom_sample(batch.n, batch.offA, C, sys, level, z)
    for i in range(nq):
        s, u = int(sys[i]), int(level[i])
        if not (0 <= s < batch.nsys) or not (0 <= u < batch.n[s]):
            assert t[i] == -2
            continue
        n, o = int(batch.n[s]), int(batch.offA[s])
        assert t[i] == reference_walk(B[o + u * n:o + (u + 1) * n], z[i]), i


@pytest.mark.gpu
def test_matom_device_pointers(engine):
    import torch
    batch, R, offv = wl.matom_cells([61] * 64 + [150] * 8, seed=21)
    B, C, st = engine.matom_matrices(batch, R, offv)
    dev = torch.device("cuda", 0)
    dN = torch.from_numpy(batch.A).to(dev)
    dR = torch.from_numpy(R).to(dev)
    dB = torch.empty_like(dN)
    dC = torch.empty_like(dN)
    dst = torch.empty(batch.nsys, dtype=torch.int32, device=dev)
    n = np.ascontiguousarray(batch.n, np.int32)
    offA = np.ascontiguousarray(batch.offA, np.int64)
    ov = np.ascontiguousarray(offv, np.int64)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    d = lambda t_: ctypes.c_void_p(t_.data_ptr())
    lib = engine.load()
    assert lib.matom_matrices_batched(batch.nsys, p(n), p(offA), p(ov), d(dN), d(dR), d(dB), d(dC), d(dst)) == 0
    assert np.array_equal(dB.cpu().numpy(), B) and np.array_equal(dC.cpu().numpy(), C)
    assert np.array_equal(dst.cpu().numpy(), st)
    rng = np.random.default_rng(2)
    sys = torch.from_numpy(rng.integers(0, batch.nsys, 4096).astype(np.int32)).to(dev)
    level = torch.from_numpy(rng.integers(0, 61, 4096).astype(np.int32)).to(dev)
    z = torch.from_numpy(rng.random(4096)).to(dev)
    tgt = torch.empty(4096, dtype=torch.int32, device=dev)
    assert lib.matom_sample_batched(4096, batch.nsys, p(n), p(offA), d(dC), d(sys), d(level), d(z), d(tgt)) == 0
    want = engine.matom_sample(batch.n, batch.offA, C, sys.cpu().numpy(), level.cpu().numpy(), z.cpu().numpy())
    assert np.array_equal(tgt.cpu().numpy(), want)


@pytest.mark.gpu
def test_matom_matrices_tiled_blocks(engine):
    # every block within 48 KB: the epilogue stages each system in shared memory
    batch, R, offv = wl.matom_cells([61] * 40 + [1, 5, 33, 47, 78], seed=13)
    B, C, st = engine.matom_matrices(batch, R, offv)
    inv, sti = engine.invert_batched(batch)
    np.testing.assert_array_equal(st, sti)
    for s in range(batch.nsys):
        n, o, v = int(batch.n[s]), int(batch.offA[s]), int(offv[s])
        b = B[o:o + n * n].reshape(n, n)
        assert np.array_equal(b, inv[o:o + n * n].reshape(n, n) * R[v:v + n][None, :]), s
        assert np.array_equal(C[o:o + n * n].reshape(n, n), np.cumsum(b, axis=1)), s
