"""The CPU oracle against the reference: golden fixtures (always) and the
reference's own GSL build (when oracle/_ref was built in this tree)."""
import numpy as np
import pytest

from oracle import oracle
from python_b200 import workloads as wl
from tests.conftest import GOLDEN
from tests.helpers import batch_from_golden, inverse_rel_err, same_values


def test_reference_unit_fixtures(golden_fixtures):
    g = golden_fixtures
    for name in ("small_matrix", "matrix_ion"):
        batch = wl.from_matrices("solve", [g[f"{name}_A"]], [g[f"{name}_b"]])
        x, st = oracle.solve(batch, "port")
        assert st[0] == g[f"{name}_code_ref"][0] == 0
        # bit-identical to the reference's GSL build on the same input
        assert same_values(x, g[f"{name}_x_ref"]).all()
        # and within the 7 printed digits of the reference's expected answer
        # (test_matrix.c compares with absolute 1e-6; all n values are checked here)
        np.testing.assert_allclose(x, g[f"{name}_x_fixture"], rtol=1e-6, atol=1e-6)
    for name in ("inverse_small", "inverse_macro"):
        M = g[f"{name}_M"]
        batch = wl.from_matrices("invert", [M])
        inv, st = oracle.invert(batch, "port")
        inv = inv.reshape(M.shape)
        assert st[0] == g[f"{name}_code_ref"][0] == 0
        assert np.max(np.abs(inv - g[f"{name}_inv_ref"])) <= 1e-13 * np.max(np.abs(g[f"{name}_inv_ref"]))
        # every entry, not only the first row (test_matrix.c:198 compared n values)
        np.testing.assert_allclose(inv, g[f"{name}_inv_fixture"], rtol=2e-4, atol=1e-6)


def test_golden_solve_cases_bit_exact(golden_solve):
    batch = batch_from_golden(golden_solve, "solve")
    x, st = oracle.solve(batch, "port")
    np.testing.assert_array_equal(st, golden_solve["status_ref"])
    ok = st != 4
    xs = np.concatenate([x[o:o + k] for o, k, m in zip(batch.offv, batch.n, ok) if m])
    xr = np.concatenate([golden_solve["x_ref"][o:o + k] for o, k, m in zip(batch.offv, batch.n, ok) if m])
    assert same_values(xs, xr).all()
    # the fixture set exercises every reference code
    assert set(np.unique(st)) == {0, 2, 3, 4}


def test_golden_invert_cases(golden_invert):
    batch = batch_from_golden(golden_invert, "invert")
    inv, st = oracle.invert(batch, "port")
    np.testing.assert_array_equal(st, golden_invert["status_ref"])
    assert set(np.unique(st)) == {0, 1}
    # GSL groups the inverse's sums recursively for n > 24; the restatement
    # does not, so agreement is to rounding
    assert inverse_rel_err(inv, golden_invert["inv_ref"], batch.n, batch.offA, st == 0) < 1e-9


@pytest.mark.skipif(not oracle.available("ref"), reason="reference build absent (oracle/_ref)")
def test_live_reference_bit_exact_random():
    rng = np.random.default_rng(7)
    mats, rhs = [], []
    for i in range(400):
        n = int(rng.integers(1, 90))
        m = rng.standard_normal((n, n)) * np.exp(rng.uniform(-15, 15, (n, n)))
        if i % 9 == 0:
            m[:, rng.integers(n)] = 0.0
        if i % 13 == 0:
            m = np.round(m)
        mats.append(m)
        rhs.append(rng.standard_normal(n))
    batch = wl.from_matrices("solve", mats, rhs)
    xp, sp = oracle.solve(batch, "port", threads=4)
    xr, sr = oracle.solve(batch, "ref", threads=4)
    np.testing.assert_array_equal(sp, sr)
    keep = np.repeat(sr != 4, batch.n)
    assert same_values(xp[keep], xr[keep]).all()


@pytest.mark.skipif(not oracle.available("ref"), reason="reference build absent (oracle/_ref)")
def test_live_reference_configs():
    b0 = wl.config0(nsys=256)
    xp, sp = oracle.solve(b0, "port")
    xr, sr = oracle.solve(b0, "ref")
    assert (sp == sr).all() and same_values(xp, xr).all()
    b1 = wl.config1(nsys=64)
    ip, tp = oracle.invert(b1, "port")
    ir, tr = oracle.invert(b1, "ref")
    assert (tp == tr).all()
    assert inverse_rel_err(ip, ir, b1.n, b1.offA) < 1e-13


def test_error_strings_match_reference_wording():
    assert oracle.error_string(2) == "some matrix rows failing relative error check"
    assert oracle.error_string(4).startswith("Unsolvable matrix!")


def test_nonfinite_codes_match_reference_golden():
    """Non-finite entries: the restatement returns the reference's codes, 21
    (GSL_ESING) included, which LU_invx raises when an infinite value reaches
    the diagonal of U (tests/golden/nonfinite_cases.npz, made by the reference
    build)."""
    g = dict(np.load(GOLDEN / "nonfinite_cases.npz"))
    ib = wl.Batch("invert", g["n"].astype(np.int32), g["offA"], g["A"])
    _, si = oracle.invert(ib, "port")
    np.testing.assert_array_equal(si, g["inv_status_ref"])
    assert 21 in set(si.tolist()) and 1 in set(si.tolist())
    sb = wl.Batch("solve", g["n"].astype(np.int32), g["offA"], g["A"], g["offv"], g["b"])
    _, ss = oracle.solve(sb, "port")
    np.testing.assert_array_equal(ss, g["solve_status_ref"])
