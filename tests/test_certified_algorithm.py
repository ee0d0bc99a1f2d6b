"""The certified inverse's arithmetic, restated in numpy (no GPU).

The certified kernels (python_b200/csrc/kernels_cert.cuh) invert M-matrices by
blocked Gauss-Jordan without pivoting in a fused rank-8 form:

    R' = D^-1 R outside the pivot block K, I + D^-1 on K's columns,
    C' = C, minus I on K's rows,
    W <- W - C' R'   on every entry.

One-CTA classes invert each 8 x 8 pivot block D by elimination in FP32 and
refine it by Newton steps X <- X + X (I - D X) in FP64 until the residual's
largest entry is below 2^-27, falling back to FP64 elimination when the first
residual is 1/4 or more or four steps do not converge.  These tests restate
both in numpy (the FP32 elimination with IEEE division where the kernel uses
the hardware's approximate reciprocal, within an FP32 ulp of it; the Newton
steps absorb the difference) and check the two decisions they rest on:
  * the refined pivot inverse is as accurate as the FP64 one, and takes the
    fallback exactly when FP32 cannot give a usable start;
  * the fused update is accurate only for diagonals near unit scale, which is
    why the certificate asks for 1/4 <= a_rr <= 4.
"""
import numpy as np
import pytest

from python_b200 import workloads as wl

HI_QUARTER = 1021 << 20     # high word of 2^-2
HI_CONVERGED = 996 << 20    # high word of 2^-27


def inv8_f64(D):
    """Gauss-Jordan without pivoting, row by row (the kernel's warp_inv8)."""
    X = D.astype(np.float64).copy()
    m = X.shape[0]
    for k in range(m):
        piv = 1.0 / X[k, k]
        nk = X[k, :] * piv
        nk[k] = piv
        for q in range(m):
            if q != k:
                f = X[q, k]
                row = X[q, :].copy()
                row[k] = 0.0
                X[q, :] = row - f * nk
        X[k, :] = nk
    return X


def inv8_f32(D):
    with np.errstate(all="ignore"):
        return inv8_f64(D.astype(np.float32)).astype(np.float64)


def abs_hi(x):
    """|x| as the high 32 bits of a double (NaN and Inf above every finite value)."""
    return (np.abs(x).view(np.uint64) >> np.uint64(32)).astype(np.uint64)


def inv8_refined(D, stats=None):
    """FP32 start, FP64 Newton steps, FP64 elimination as fallback."""
    with np.errstate(all="ignore"):
        X = inv8_f32(D)
        for it in range(4):
            E = np.eye(8) - D @ X
            em = int(abs_hi(E).max())
            if em >= HI_QUARTER:
                break
            X = X + X @ E
            if em < HI_CONVERGED:
                if stats is not None:
                    stats.append(it + 1)
                return X
    if stats is not None:
        stats.append(0)
    return inv8_f64(D)


def certified_gj(A, refined=True, stats=None):
    """The fused blocked Gauss-Jordan on the identity-padded matrix."""
    n = A.shape[0]
    P = (n + 7) // 8 * 8
    W = np.eye(P)
    W[:n, :n] = A
    for kb in range((n + 7) // 8):
        K = slice(8 * kb, 8 * kb + 8)
        D = W[K, K].copy()
        Dinv = inv8_refined(D, stats) if refined else inv8_f64(D)
        R = W[K, :].copy()
        C = W[:, K].copy()
        Rp = Dinv @ R
        Rp[:, K] = np.eye(8) + Dinv
        Cp = C.copy()
        Cp[K, :] -= np.eye(8)
        W = W - Cp @ Rp
    return W[:n, :n]


def rel_err(X, ref):
    return float(np.abs(X - ref).max() / np.abs(ref).max())


def margin_matrix(rng, n, tau):
    off = rng.uniform(0.0, 1.0, (n, n))
    np.fill_diagonal(off, 0.0)
    off *= (1.0 - tau) / off.sum(axis=1, keepdims=True)
    return np.eye(n) - off


def dominant_block(rng, scale_rows=None):
    """An 8 x 8 row-dominant M-matrix block (unit diagonal, margin >= 0.3)."""
    off = rng.uniform(0.0, 1.0, (8, 8))
    np.fill_diagonal(off, 0.0)
    off *= rng.uniform(0.0, 0.7, (8, 1)) / off.sum(axis=1, keepdims=True)
    D = np.eye(8) - off
    return D if scale_rows is None else scale_rows[:, None] * D


def test_refined_pivot_inverse_matches_fp64_elimination():
    rng = np.random.default_rng(8)
    for _ in range(200):
        D = dominant_block(rng)
        steps = []
        X = inv8_refined(D, steps)
        assert steps[0] in (1, 2), steps        # an FP32 start converges in one or two steps
        assert rel_err(X, inv8_f64(D)) <= 4e-16 * 8
        assert rel_err(X, np.linalg.inv(D)) <= 4e-16 * 8


@pytest.mark.parametrize("e", [150, -150])
def test_refined_pivot_inverse_falls_back_outside_fp32(e):
    # a row beyond FP32's range makes the FP32 start Inf or NaN: the first
    # residual is not below 1/4 and the FP64 elimination takes the block
    rng = np.random.default_rng(abs(e))
    s = np.ones(8)
    s[3] = np.ldexp(1.0, e)
    D = dominant_block(rng, s)
    steps = []
    X = inv8_refined(D, steps)
    assert steps == [0]
    assert np.array_equal(X, inv8_f64(D))


def test_certified_gj_on_macro_matrices():
    rng = np.random.default_rng(61)
    for n in (33, 40, 61, 100, 136, 152, 200):
        M = wl.macro_matrix(rng, n)
        ref = np.linalg.inv(M)
        X = certified_gj(M)
        assert rel_err(X, ref) <= 1e-12, n
        assert rel_err(X, certified_gj(M, refined=False)) <= 1e-13, n


@pytest.mark.parametrize("tau,want", [(1e-6, {3}), (1e-7, {3, 4}), (1e-8, {0, 4})])
def test_refined_pivot_inverse_of_ill_conditioned_blocks(tau, want):
    # 8 x 8 blocks whose every row sits at margin tau (condition ~1/tau): the
    # FP32 start is further off, so more Newton steps follow, and at 1e-8 some
    # blocks take the FP64 elimination; the result stays within the
    # elimination's own accuracy (~1e-16 / tau)
    rng = np.random.default_rng(5)
    seen = set()
    for _ in range(40):
        D = margin_matrix(rng, 8, tau)
        steps = []
        X = inv8_refined(D, steps)
        seen.add(steps[0])
        assert rel_err(X, np.linalg.inv(D)) <= 1e-15 / tau
        assert rel_err(X, inv8_f64(D)) <= 1e-15 / tau
    assert seen <= {0, 3, 4} and seen & want, seen


def test_certified_gj_near_the_margin():
    # every row of the matrix at margin 1.5e-5 (condition ~1e5): its 8 x 8
    # pivot blocks stay well conditioned, and the inverse within 1e-10
    rng = np.random.default_rng(15)
    for n in (40, 64, 128):
        M = margin_matrix(rng, n, 1.5e-5)
        steps = []
        X = certified_gj(M, stats=steps)
        assert rel_err(X, np.linalg.inv(M)) <= 1e-10, n
        assert all(k in (1, 2) for k in steps), steps


def test_fused_update_is_accurate_near_unit_scale_only():
    # rows scaled by 2^+-e: within the certificate's range (e = 2) the fused
    # update keeps FP64 accuracy; at e = 20 it loses about e bits, past what
    # 1e-10 allows once the row scales spread further -- hence the range
    rng = np.random.default_rng(20)
    for e, lo, hi in ((2, 0.0, 1e-13), (20, 1e-12, 1.0)):
        worst = 0.0
        for n in (37, 64, 100):
            M = wl.macro_matrix(rng, n)
            s = np.ldexp(1.0, rng.choice([-e, 0, e], n))
            X = certified_gj(s[:, None] * M, refined=False)
            worst = max(worst, rel_err(X, np.linalg.inv(M) / s[None, :]))
        assert lo <= worst <= hi, (e, worst)


def certified_gj_equilibrated(A, refined=True):
    """Rows times the power of two that brings their diagonal into [1, 2),
    the inverse's columns times the same powers (exact).  The kernels do not
    do this: built into the register-resident kernel it cost 5 % at order 64
    even when skipped at run time, so the certificate bounds the diagonal
    instead; this restatement shows what it would restore."""
    s = np.ldexp(1.0, -np.frexp(np.diag(A))[1] + 1)
    return certified_gj(s[:, None] * A, refined) * s[None, :]


@pytest.mark.parametrize("e", [20, 150])
def test_equilibration_restores_accuracy(e):
    rng = np.random.default_rng(e)
    for n in (37, 64, 100):
        M = wl.macro_matrix(rng, n)
        s = np.ldexp(1.0, rng.choice([-e, 0, e], n))
        A = s[:, None] * M
        X = certified_gj_equilibrated(A)
        assert np.all(np.diag(np.ldexp(1.0, -np.frexp(np.diag(A))[1] + 1)[:, None] * A) >= 1.0)
        assert rel_err(X * s[None, :], np.linalg.inv(M)) <= 1e-13, (e, n)
        assert np.array_equal(X * s[None, :], certified_gj(M)), (e, n)   # exact powers of two
