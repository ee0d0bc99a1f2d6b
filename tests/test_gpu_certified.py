"""Certified inverses (SIROCCO_FAST) against the reference's GSL inverse.

Matrices that pass the certificate (nonsingular M-matrices with a relative
row-dominance margin of at least 1e-5 and diagonal entries within [1/4, 4])
are inverted by Gauss-Jordan without
pivoting: code 0, as GSL's, and the inverse within 1e-10 (max-abs, relative to
the largest entry) of the reference build's.  Orders 33-224 run the
register-resident kernel, orders 225-1024 the streamed one.  Every other
matrix falls back to the GSL-exact path, whose results must equal
SIROCCO_FP64 mode's bit for bit.
"""
import numpy as np
import pytest

from oracle import oracle
from python_b200 import workloads as wl
from tests.helpers import inverse_rel_err, same_values

pytestmark = pytest.mark.gpu

INV_TOL = 1e-10
CERTIFIED_DIAG = 0


def ref_invert(batch):
    which = "ref" if oracle.available("ref") else "port"
    return oracle.invert(batch, which, threads=oracle.host_threads())


def run_plan(engine, batch, mode):
    import torch
    dev = torch.device("cuda")
    A = torch.from_numpy(batch.A).to(dev)
    out = torch.full_like(A, float("nan"))
    st = torch.full((batch.nsys,), -99, dtype=torch.int32, device=dev)
    diag = torch.full((batch.nsys,), -1, dtype=torch.int32, device=dev)
    plan = engine.Plan(batch, mode)
    plan.execute(A, out, st, diag=diag)
    torch.cuda.synchronize()
    plan.close()
    return out.cpu().numpy(), st.cpu().numpy(), diag.cpu().numpy()


def per_system_err(inv, ref, batch):
    return np.array([inverse_rel_err(inv, ref, batch.n[s:s + 1], batch.offA[s:s + 1]) for s in range(batch.nsys)])


def test_certified_config1_sample_matches_gsl(engine):
    batch = wl.config1(nsys=2048)
    inv, st, diag = run_plan(engine, batch, engine.FAST)
    ir, sr = ref_invert(batch)
    np.testing.assert_array_equal(st, sr)
    assert (diag == CERTIFIED_DIAG).all(), "every config-1 matrix is an M-matrix with margin >= 1e-4"
    assert inverse_rel_err(inv, ir, batch.n, batch.offA) <= INV_TOL


@pytest.mark.parametrize("lo,hi", [(33, 64), (65, 128), (129, 192), (193, 224)])
def test_certified_every_class_matches_gsl(engine, lo, hi):
    rng = np.random.default_rng(lo)
    sizes = list(range(lo, hi + 1, 3)) + [lo, hi]
    batch = wl.macro_batch(sizes, seed=int(rng.integers(1 << 30)))
    inv, st, diag = run_plan(engine, batch, engine.FAST)
    ir, sr = ref_invert(batch)
    np.testing.assert_array_equal(st, sr)
    assert (diag == CERTIFIED_DIAG).all()
    err = per_system_err(inv, ir, batch)
    assert err.max() <= INV_TOL, (batch.n[np.argmax(err)], err.max())


# the streamed kernel: 64-column steps, so the orders around multiples of 64
# (partial last tiles and steps) and both ends of its range
STREAMED_ORDERS = [225, 230, 255, 256, 257, 300, 319, 320, 321, 383, 384, 449, 511, 512, 513, 640, 700, 777,
                   895, 960, 1000, 1023, 1024]


def test_certified_streamed_orders_match_gsl(engine):
    batch = wl.macro_batch(STREAMED_ORDERS, seed=225, density=0.10)
    inv, st, diag = run_plan(engine, batch, engine.FAST)
    ir, sr = ref_invert(batch)
    np.testing.assert_array_equal(st, sr)
    assert (diag == CERTIFIED_DIAG).all()
    err = per_system_err(inv, ir, batch)
    assert err.max() <= INV_TOL, (batch.n[np.argmax(err)], err.max())


def test_certified_streamed_fallback_and_odd_layout(engine):
    """Streamed orders that fail the certificate take the exact path (bit-equal
    to SIROCCO_FP64); the good ones are inverted at offsets that leave their
    rows 8-byte but not 16-byte aligned (an odd number of doubles before each)."""
    rng = np.random.default_rng(23)
    good = [wl.macro_matrix(rng, int(n), density=0.10) for n in (226, 260, 402, 514)]
    bad = []
    m = wl.macro_matrix(rng, 300, density=0.10)
    m[17, 40] = 2e-3                            # a positive off-diagonal entry
    bad.append(m)
    m = wl.macro_matrix(rng, 600, density=0.10)
    m[100, :] = 0.0                             # singular: the reference returns 1
    bad.append(m)
    m = wl.macro_matrix(rng, 257, density=0.10)
    m[3, 3] = np.inf
    bad.append(m)
    mats = [good[0], bad[0], good[1], bad[1], good[2], bad[2], good[3]]
    n = np.array([x.shape[0] for x in mats], dtype=np.int32)
    offA = np.zeros(len(mats), dtype=np.int64)
    pos = 1                                     # every matrix starts at an odd element offset
    for s, x in enumerate(mats):
        offA[s] = pos
        pos += x.size + (1 if (pos + x.size) % 2 == 0 else 0)
    A = np.zeros(pos, dtype=np.float64)
    for s, x in enumerate(mats):
        A[offA[s]:offA[s] + x.size] = x.ravel()
    batch = wl.Batch("invert", n, offA, A)
    inv, st, diag = run_plan(engine, batch, engine.FAST)
    inv64, st64, _ = run_plan(engine, batch, engine.FP64)
    ir, sr = ref_invert(batch)
    np.testing.assert_array_equal(st, sr)
    np.testing.assert_array_equal(st, st64)
    fb = (diag & (1 << 8)) != 0
    assert fb.tolist() == [False, True, False, True, False, True, False]
    for s in np.nonzero(fb)[0]:
        o, k = int(offA[s]), int(n[s])
        assert same_values(inv[o:o + k * k], inv64[o:o + k * k]).all(), s
    err = per_system_err(inv, ir, batch)
    assert err[~fb].max() <= INV_TOL


def test_certified_config3_macro_sample(engine):
    rng = np.random.default_rng(3)
    batch = wl.macro_batch(rng.integers(20, 201, 400), seed=33)
    inv, st, _ = run_plan(engine, batch, engine.FAST)
    ir, sr = ref_invert(batch)
    np.testing.assert_array_equal(st, sr)
    assert per_system_err(inv, ir, batch).max() <= INV_TOL


def margin_matrix(rng, n, tau):
    """A dense M-matrix whose every row sits just inside the certificate's
    margin: unit diagonal, off-diagonal row sums 1 - tau (condition ~1/tau)."""
    off = rng.uniform(0.0, 1.0, (n, n))
    np.fill_diagonal(off, 0.0)
    off *= (1.0 - tau) / off.sum(axis=1, keepdims=True)
    return np.eye(n) - off


@pytest.mark.parametrize("tau", [1.5e-5, 1e-3])
def test_certified_pivot_blocks_near_the_margin(engine, tau):
    # condition ~1e5 at tau = 1.5e-5; the one-CTA classes invert each 8 x 8
    # pivot block in FP32 and refine it by FP64 Newton steps, the clusters by
    # FP64 elimination
    rng = np.random.default_rng(int(1 / tau))
    sizes = [33, 40, 47, 56, 61, 64, 72, 90, 104, 119, 128, 150, 200]
    batch = wl.from_matrices("invert", [margin_matrix(rng, n, tau) for n in sizes])
    inv, st, diag = run_plan(engine, batch, engine.FAST)
    ir, sr = ref_invert(batch)
    np.testing.assert_array_equal(st, sr)
    assert (diag == CERTIFIED_DIAG).all()
    err = per_system_err(inv, ir, batch)
    assert err.max() <= INV_TOL, (batch.n[np.argmax(err)], err.max())


def test_certified_diagonal_scale(engine):
    # The fused update adds I to each pivot block's inverse, which is accurate
    # relative to unit scale only: the certificate takes diagonals in [1/4, 4]
    # and leaves every other scale (rows at 2^+-150, whose FP32 pivot start
    # would also overflow or underflow; a whole matrix times 8 or 1/8) to the
    # exact path, bit-equal to SIROCCO_FP64.  Rows scaled within the range stay
    # certified and within 1e-10 of GSL.
    rng = np.random.default_rng(150)
    mats, want_fb = [], []
    for n in (37, 64, 100, 128, 170, 300):
        mats.append(np.ldexp(1.0, rng.choice([-150, 0, 150], n))[:, None] * wl.macro_matrix(rng, n))
        want_fb.append(True)
    for n, f in ((45, 8.0), (90, 0.125), (200, 8.0)):
        mats.append(f * wl.macro_matrix(rng, n))
        want_fb.append(True)
    for n in (40, 61, 120, 150, 260):
        mats.append(np.ldexp(1.0, rng.choice([-2, -1, 0, 1, 2], n))[:, None] * wl.macro_matrix(rng, n))
        want_fb.append(False)
    batch = wl.from_matrices("invert", mats)
    inv, st, diag = run_plan(engine, batch, engine.FAST)
    inv64, st64, _ = run_plan(engine, batch, engine.FP64)
    ir, sr = ref_invert(batch)
    np.testing.assert_array_equal(st, sr)
    np.testing.assert_array_equal(st, st64)
    fb = (diag & (1 << 8)) != 0
    assert fb.tolist() == want_fb, diag
    for k in np.nonzero(fb)[0]:
        o, n = int(batch.offA[k]), int(batch.n[k])
        assert same_values(inv[o:o + n * n], inv64[o:o + n * n]).all(), n
    err = per_system_err(inv, ir, batch)
    assert err[~fb].max() <= INV_TOL, (batch.n[~fb], err[~fb])


def uncertified_matrices(rng):
    """Matrices that must fail the certificate, with the reason."""
    out = []
    m = wl.macro_matrix(rng, 40)
    m[5, :] = 0.0
    m[5, 5] = 1.0
    m[5, 7] = -1.0                              # a level that cannot deactivate: margin 0
    out.append(m)
    m = wl.macro_matrix(rng, 70)
    m[3, 9] = 1e-3                              # a positive off-diagonal entry
    out.append(m)
    m = wl.macro_matrix(rng, 100)
    m[10, 11] = np.nan                          # non-finite entry
    out.append(m)
    m = wl.macro_matrix(rng, 33)
    m[2, :] = 0.0                               # singular: the reference returns 1
    out.append(m)
    m = wl.macro_matrix(rng, 150)
    m[0, 0] = 1.0 - 1e-6 + m[0, 0] - 1.0        # diagonal shrunk below the margin
    m[0, 1:] = 0.0
    m[0, 1] = -(1.0 - 2e-6)
    out.append(m)
    out.append(np.random.default_rng(1).standard_normal((60, 60)))   # general dense
    m = wl.macro_matrix(rng, 200)
    m[199, 198] = np.inf
    out.append(m)
    return out


def test_uncertified_fall_back_to_the_exact_path(engine):
    rng = np.random.default_rng(11)
    bad = uncertified_matrices(rng)
    good = [wl.macro_matrix(rng, int(n)) for n in rng.integers(33, 225, 40)]
    mats = good[:20] + bad + good[20:]
    batch = wl.from_matrices("invert", mats)
    inv, st, diag = run_plan(engine, batch, engine.FAST)
    inv64, st64, _ = run_plan(engine, batch, engine.FP64)
    ir, sr = ref_invert(batch)
    np.testing.assert_array_equal(st, sr)
    np.testing.assert_array_equal(st, st64)
    fb = (diag & (1 << 8)) != 0
    nbad = len(bad)
    assert fb[20:20 + nbad].all(), diag[20:20 + nbad]
    assert not fb[:20].any() and not fb[20 + nbad:].any()
    for s in np.nonzero(fb)[0]:
        o, k = int(batch.offA[s]), int(batch.n[s])
        if st[s] == 0:
            assert same_values(inv[o:o + k * k], inv64[o:o + k * k]).all(), s
    ok = st == 0
    good_idx = np.array([s for s in range(batch.nsys) if not fb[s]])
    sub_err = per_system_err(inv, ir, batch)
    assert sub_err[good_idx].max() <= INV_TOL
    assert ok[good_idx].all()


def test_certified_plan_in_a_cuda_graph(engine):
    import torch
    rng = np.random.default_rng(5)
    mats = [wl.macro_matrix(rng, int(n)) for n in rng.integers(33, 225, 300)]
    mats += [wl.macro_matrix(rng, int(n), density=0.10) for n in (230, 333, 480)]   # the streamed kernel's queue
    bad = uncertified_matrices(rng)
    batch = wl.from_matrices("invert", mats[:150] + bad + mats[150:])
    want, wst, _ = run_plan(engine, batch, engine.FAST)
    dev = torch.device("cuda")
    A = torch.from_numpy(batch.A).to(dev)
    out = torch.zeros_like(A)
    st = torch.full((batch.nsys,), -99, dtype=torch.int32, device=dev)
    plan = engine.Plan(batch, engine.FAST)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        plan.execute(A, out, st, stream=s)   # warm-up outside the capture
        s.synchronize()
        with torch.cuda.graph(g, stream=s):
            plan.execute(A, out, st, stream=s)
    for _ in range(2):
        out.zero_()
        st.fill_(-99)
        g.replay()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_array_equal(st.cpu().numpy(), wst)
        ok = np.repeat(wst == 0, batch.n.astype(np.int64) ** 2)
        assert same_values(got[ok], want[ok]).all()
    plan.close()


def test_certified_host_batched_entry(engine):
    """invert_matrix_batched in SIROCCO_FAST mode through host buffers, including
    the chunked host pipeline (a batch above 32 MiB)."""
    batch = wl.config1(nsys=1400)
    inv, st = engine.invert_batched(batch, engine.FAST)
    ir, sr = ref_invert(batch)
    np.testing.assert_array_equal(st, sr)
    assert inverse_rel_err(inv, ir, batch.n, batch.offA) <= INV_TOL
