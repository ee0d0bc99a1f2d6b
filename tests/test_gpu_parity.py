"""Parity of the CUDA engine with the reference, through the C ABI.

FP64 mode: the factorisation is GSL's bit for bit, so solutions and every
return code must equal the reference build's exactly; inverses agree to
rounding (GSL groups the inverse's sums recursively).
Mixed mode: codes exactly; populations above 1e-20 of each system's total
within 1e-10 relative; normwise backward error within n * 1e-15.
"""
import numpy as np
import pytest

from oracle import oracle
from python_b200 import workloads as wl
from tests.helpers import (backward_err, batch_from_golden, inverse_rel_err, population_rel_err,
                           same_values)

pytestmark = pytest.mark.gpu

POP_TOL = 1e-10
INV_TOL = 1e-10   # inverses: max |X - X_ref| / max |X_ref| per matrix


def ref_which():
    return "ref" if oracle.available("ref") else "port"


def solved_mask(batch, st):
    return np.repeat(st != 4, batch.n)


# ------------------------------------------------------------------ FP64 ----
def test_fp64_golden_solves_bit_exact(engine, golden_solve):
    batch = batch_from_golden(golden_solve, "solve")
    x, st = engine.solve_batched(batch, engine.FP64)
    np.testing.assert_array_equal(st, golden_solve["status_ref"])
    m = solved_mask(batch, st)
    assert same_values(x[m], golden_solve["x_ref"][m]).all()


def test_fp64_golden_inverses(engine, golden_invert):
    batch = batch_from_golden(golden_invert, "invert")
    inv, st = engine.invert_batched(batch, engine.FP64)
    np.testing.assert_array_equal(st, golden_invert["status_ref"])
    assert inverse_rel_err(inv, golden_invert["inv_ref"], batch.n, batch.offA, st == 0) < 1e-9


def test_dropin_reference_fixtures(engine, golden_fixtures):
    g = golden_fixtures
    for name in ("small_matrix", "matrix_ion"):
        code, x = engine.solve_matrix(g[f"{name}_A"], g[f"{name}_b"])
        assert code == g[f"{name}_code_ref"][0]
        assert same_values(x, g[f"{name}_x_ref"]).all()
        np.testing.assert_allclose(x, g[f"{name}_x_fixture"], rtol=1e-6, atol=1e-6)
    for name in ("inverse_small", "inverse_macro"):
        code, inv = engine.invert_matrix(g[f"{name}_M"])
        assert code == g[f"{name}_code_ref"][0] == 0
        ref = g[f"{name}_inv_ref"]
        assert np.max(np.abs(inv - ref)) <= 1e-12 * np.max(np.abs(ref))
        np.testing.assert_allclose(inv, g[f"{name}_inv_fixture"], rtol=2e-4, atol=1e-6)


def test_dropin_singular_leaves_output_untouched(engine):
    a = np.array([[1.0, 2.0], [2.0, 4.0]])
    x0 = np.full(2, 7.0)
    code, x = engine.solve_matrix(a, np.ones(2), x0.copy())
    assert code == 4 and (x == x0).all()
    code, inv = engine.invert_matrix(a, np.full((2, 2), 7.0))
    assert code == 1 and (inv == 7.0).all()


@pytest.mark.parametrize("sizes", [list(range(1, 33)), [33, 40, 47, 48, 50, 63, 64, 65, 80, 96, 100, 127, 128],
                                   [129, 150, 160, 161, 178, 192, 193, 200, 208, 209, 224, 225, 256, 257],
                                   [320, 321, 384, 385, 448, 449, 512, 513, 640, 641, 768, 769, 896, 897, 1024]])
def test_fp64_every_size_class_matches_oracle(engine, sizes):
    rng = np.random.default_rng(sum(sizes))
    reps = 3 if max(sizes) <= 128 else 1
    szs = [n for n in sizes for _ in range(reps)]
    batch = wl.dense_batch("solve", szs, seed=int(rng.integers(1 << 30)), log_spread=4.0)
    x, st = engine.solve_batched(batch, engine.FP64)
    xr, sr = oracle.solve(batch, "port", threads=oracle.host_threads())
    np.testing.assert_array_equal(st, sr)
    m = solved_mask(batch, st)
    assert same_values(x[m], xr[m]).all()
    ib = wl.dense_batch("invert", szs, seed=int(rng.integers(1 << 30)))
    inv, si = engine.invert_batched(ib, engine.FP64)
    ir, sir = oracle.invert(ib, "port", threads=oracle.host_threads())
    np.testing.assert_array_equal(si, sir)
    assert inverse_rel_err(inv, ir, ib.n, ib.offA, si == 0) < INV_TOL


def test_fp64_config0_full_size_bit_exact(engine):
    batch = wl.config0()
    x, st = engine.solve_batched(batch, engine.FP64)
    xr, sr = oracle.solve(batch, "port", threads=oracle.host_threads())
    np.testing.assert_array_equal(st, sr)
    assert same_values(x, xr).all()
    # conservation row: populations of each system sum to 1
    sums = np.add.reduceat(x, batch.offv.astype(np.intp))
    assert np.max(np.abs(sums - 1.0)) < 1e-12


def test_fp64_config1_full_size(engine):
    batch = wl.config1()
    inv, st = engine.invert_batched(batch, engine.FP64)
    assert (st == 0).all()
    sub = wl.Batch("invert", batch.n[:512], batch.offA[:512], batch.A[:batch.offA[512]])
    ir, sr = oracle.invert(sub, "port", threads=oracle.host_threads())
    assert inverse_rel_err(inv[:sub.A.size], ir, sub.n, sub.offA) < 1e-12
    # size-independent checks on every system: M M^-1 = I, and the absorbing
    # row sums of N^-1 (1 - q) = 1 for the jumping matrix N = I - Q
    worst_id = 0.0
    for s in range(0, batch.nsys, 97):
        M = batch.matrix(s)
        X = inv[batch.offA[s]:batch.offA[s] + M.size].reshape(M.shape)
        worst_id = max(worst_id, np.max(np.abs(M @ X - np.eye(M.shape[0]))))
        pdeact = M.sum(axis=1)                       # 1 - row sum of Q
        np.testing.assert_allclose(X @ pdeact, np.ones(M.shape[0]), rtol=1e-10)
    assert worst_id < 1e-10


def test_batched_device_plan_and_graph(engine):
    import torch
    batch = wl.config0(nsys=1000)
    dev = torch.device("cuda")
    A = torch.from_numpy(batch.A).to(dev)
    b = torch.from_numpy(batch.b).to(dev)
    x = torch.empty_like(b)
    st = torch.full((batch.nsys,), -1, dtype=torch.int32, device=dev)
    plan = engine.Plan(batch, engine.FP64)
    plan.execute(A, x, st, b=b)
    torch.cuda.synchronize()
    xr, sr = oracle.solve(batch, "port")
    assert (st.cpu().numpy() == sr).all() and same_values(x.cpu().numpy(), xr).all()
    # the same sequence captured in a CUDA graph and replayed
    x.zero_()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            plan.execute(A, x, st, b=b, stream=s)
    g.replay()
    torch.cuda.synchronize()
    assert same_values(x.cpu().numpy(), xr).all()
    plan.close()


# ----------------------------------------------------------------- mixed ----
def run_plan(engine, batch, mode):
    import torch
    dev = torch.device("cuda")
    A = torch.from_numpy(batch.A).to(dev)
    b = torch.from_numpy(batch.b).to(dev)
    x = torch.full_like(b, float("nan"))
    st = torch.full((batch.nsys,), -1, dtype=torch.int32, device=dev)
    diag = torch.zeros((batch.nsys,), dtype=torch.int32, device=dev)
    plan = engine.Plan(batch, mode)
    plan.execute(A, x, st, b=b, diag=diag)
    torch.cuda.synchronize()
    plan.close()
    return x.cpu().numpy(), st.cpu().numpy(), diag.cpu().numpy()


def check_mixed(engine, batch, require_accept=None):
    """Codes exact; fallback systems bit-identical to the reference; accepted
    systems within 1e-10 of the reference on significant populations, or, where
    the reference's own FP64 answer is off by more, within 1e-10 of the exact
    solution (80-digit mpmath)."""
    x, st, diag = run_plan(engine, batch, engine.MIXED)
    xr, sr = oracle.solve(batch, "port", threads=oracle.host_threads())
    np.testing.assert_array_equal(st, sr)
    fell_back = (diag & (1 << 8)) != 0
    accepted = 0
    for s in range(batch.nsys):
        n, o = int(batch.n[s]), int(batch.offv[s])
        v, r = x[o:o + n], xr[o:o + n]
        if fell_back[s]:
            if st[s] != 4:
                assert same_values(v, r).all(), s
            continue
        accepted += 1
        assert st[s] == 0
        if population_rel_err(v, r, np.array([n]), np.array([0])) > POP_TOL:
            t = exact_solution(batch.matrix(s), batch.rhs(s))
            assert population_rel_err(v, t, np.array([n]), np.array([0])) <= POP_TOL, s
            assert population_rel_err(r, t, np.array([n]), np.array([0])) > POP_TOL, s
    if require_accept is not None:
        assert accepted >= require_accept * batch.nsys, (accepted, batch.nsys)
    return accepted


def exact_solution(A, b):
    import mpmath
    mpmath.mp.dps = 80
    x = mpmath.lu_solve(mpmath.matrix(A.tolist()), mpmath.matrix(b.tolist()))
    return np.array([float(t) for t in x])


def test_mixed_golden(engine, golden_solve):
    check_mixed(engine, batch_from_golden(golden_solve, "solve"))


def test_mixed_config0(engine):
    check_mixed(engine, wl.config0())


def test_mixed_well_conditioned_sets_accept_and_match(engine):
    rng = np.random.default_rng(77)
    mats = [wl.macro_matrix(rng, int(n)) for n in rng.integers(4, 33, 600)]
    macro = wl.from_matrices("solve", mats, [np.abs(rng.standard_normal(m.shape[0])) for m in mats])
    check_mixed(engine, macro, require_accept=0.5)
    dense = wl.dense_batch("solve", rng.integers(2, 33, 600), seed=78)
    check_mixed(engine, dense, require_accept=0.3)


# ------------------------------------------------------------ non-finite ----
@pytest.mark.parametrize("mode", ["FP64", "FAST"])
def test_nonfinite_codes_match_reference(engine, mode):
    """Matrices with +Inf, -Inf or NaN entries: invert_matrix's codes, 21
    (GSL_ESING, an infinite pivot) included, and solve_matrix's codes equal the
    reference build's (tests/golden/nonfinite_cases.npz); a system whose code is
    not 0 leaves its output untouched through the drop-in call."""
    from tests.conftest import GOLDEN
    g = dict(np.load(GOLDEN / "nonfinite_cases.npz"))
    m = getattr(engine, mode)
    ib = wl.Batch("invert", g["n"].astype(np.int32), g["offA"], g["A"])
    _, si = engine.invert_batched(ib, m)
    np.testing.assert_array_equal(si, g["inv_status_ref"])
    sb = wl.Batch("solve", g["n"].astype(np.int32), g["offA"], g["A"], g["offv"], g["b"])
    _, ss = engine.solve_batched(sb, m)
    np.testing.assert_array_equal(ss, g["solve_status_ref"])
    for s in np.nonzero(g["inv_status_ref"] == 21)[0][:4]:
        code, inv = engine.invert_matrix(ib.matrix(int(s)).copy(), np.full((ib.n[s], ib.n[s]), 7.0))
        assert code == 21 and (inv == 7.0).all()


# --------------------------------------------------- drop-in CUDA names ----
def test_gpu_named_entry_points_match_oracle(engine, golden_solve, golden_invert):
    """gpu_solve_matrix / gpu_invert_matrix, the names of the reference's CUDA
    build (source/matrix_gpu.h:20-21), on the golden cases: codes equal, solves
    bit for bit, inverses to rounding."""
    import ctypes
    lib = engine.load()
    dp = ctypes.POINTER(ctypes.c_double)
    sb = batch_from_golden(golden_solve, "solve")
    for s in range(0, sb.nsys, 7):
        n = int(sb.n[s])
        a = sb.matrix(s).copy()
        b = sb.rhs(s).copy()
        x = np.full(n, 7.0)
        code = lib.gpu_solve_matrix(a.ctypes.data_as(dp), b.ctypes.data_as(dp), n, x.ctypes.data_as(dp))
        assert code == golden_solve["status_ref"][s]
        xr = golden_solve["x_ref"][sb.offv[s]:sb.offv[s] + n]
        if code != 4:
            assert same_values(x, xr).all(), s
        else:
            assert (x == 7.0).all()
    ib = batch_from_golden(golden_invert, "invert")
    for s in range(0, ib.nsys, 5):
        n = int(ib.n[s])
        m = ib.matrix(s).copy()
        out = np.full((n, n), 7.0)
        code = lib.gpu_invert_matrix(m.ctypes.data_as(dp), out.ctypes.data_as(dp), n)
        assert code == golden_invert["status_ref"][s]
        if code == 0:
            r = golden_invert["inv_ref"][ib.offA[s]:ib.offA[s] + n * n].reshape(n, n)
            assert np.max(np.abs(out - r)) <= 1e-10 * np.max(np.abs(r)), s
        else:
            assert (out == 7.0).all()


# ------------------------------------------------ the headline generators ----
@pytest.mark.parametrize("mode", ["FP64", "FAST"])
def test_config3_generator_sample(engine, mode):
    """A sample of the 50k-cell generator (400 cells: 4,000 ion solves of orders
    2-27 and 400 macro-atom inverses of orders 20-200) in both modes: solves bit
    for bit and codes equal to the reference build, inverses within 1e-10."""
    solves, inverses = wl.config3(ncells=400, seed=wl.BASE_SEED + 33)
    m = getattr(engine, mode)
    x, st = engine.solve_batched(solves, m)
    xr, sr = oracle.solve(solves, ref_which(), threads=oracle.host_threads())
    np.testing.assert_array_equal(st, sr)
    keep = solved_mask(solves, st)
    assert same_values(x[keep], xr[keep]).all()
    inv, si = engine.invert_batched(inverses, m)
    ir, sir = oracle.invert(inverses, ref_which(), threads=oracle.host_threads())
    np.testing.assert_array_equal(si, sir)
    assert inverse_rel_err(inv, ir, inverses.n, inverses.offA, si == 0) <= INV_TOL


def test_config4_generator_sample(engine):
    """Large macro atoms (orders 256-1024, the config-4 generator) against the
    reference build: codes equal, inverses within 1e-10."""
    batch = wl.config4(nsys=6, seed=wl.BASE_SEED + 44)
    for mode in (engine.FP64, engine.FAST):
        inv, st = engine.invert_batched(batch, mode)
        ir, sr = oracle.invert(batch, ref_which(), threads=oracle.host_threads())
        np.testing.assert_array_equal(st, sr)
        assert inverse_rel_err(inv, ir, batch.n, batch.offA, st == 0) <= INV_TOL
