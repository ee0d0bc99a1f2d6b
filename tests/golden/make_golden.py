"""Generate the golden fixtures in this folder from the reference.

Run in a tree where the reference is present (its path in SIROCCO_REFERENCE,
default the mount used when these fixtures were made) after ``make -C oracle ref``:

    python tests/golden/make_golden.py

Writes:
  reference_fixtures.npz  the reference's own unit-test matrices
      (source/tests/test_data/matrix/{small_matrix,matrix_ion,inverse_small,
      inverse_macro}: first token n, then n*n or n values, row-major), with the
      7-digit expected answers from those files AND the full-precision answers
      of the reference's GSL build run here on the same inputs.
  solve_cases.npz / invert_cases.npz  seeded systems (all size classes of the
      engine, ion-balance and macro-atom generators, singular and
      residual-failure constructions) with the reference build's outputs.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import oracle  # noqa: E402
from python_b200 import workloads as wl  # noqa: E402

# the reference checkout: SIROCCO_REFERENCE, else a `reference` directory beside
# this repository's root
REF = Path(os.environ.get("SIROCCO_REFERENCE", str(ROOT.parent / "reference")))
FIX = REF / "source" / "tests" / "test_data" / "matrix"


def read_fixture(path: Path) -> np.ndarray:
    tok = path.read_text().split()
    n = int(tok[0])
    vals = np.array([float(t) for t in tok[1:]], dtype=np.float64)
    return vals.reshape(n, n) if vals.size == n * n else vals


def singular_cases(rng):
    """Matrices the reference must call singular (or nearly so)."""
    mats = []
    for n in (2, 3, 5, 8, 13, 27, 40, 61):
        m = rng.standard_normal((n, n))
        m[:, rng.integers(n)] = 0.0                      # zero column
        mats.append(m)
        m = rng.standard_normal((n, n))
        m[rng.integers(n)] = 0.0                         # zero row
        mats.append(m)
        m = rng.standard_normal((n, n))
        i, j = rng.choice(n, 2, replace=False)
        m[j] = m[i]                                      # duplicate row
        mats.append(m)
        m = rng.integers(-3, 4, (n, n)).astype(float)
        if n > 2:
            m[2] = m[0] + 2 * m[1]                       # exact integer dependence
        mats.append(m)
    # rank-one-deficient rows built with inexact multipliers: depending on the
    # rounding, GSL sees an exact zero pivot or a tiny one
    for _ in range(60):
        n = int(rng.integers(2, 7))
        m = rng.integers(-9, 10, (n, n)).astype(float)
        a, c = rng.integers(1, 9, 2) / rng.integers(1, 9, 2)
        m[n - 1] = a * m[0] + (c * m[1] if n > 2 else 0.0)
        mats.append(m)
    mats.append(np.array([[0.0]]))
    mats.append(np.array([[1.0, 2.0], [2.0, 4.0]]))
    return mats


def residual_failure_cases(rng):
    """Systems whose reference residual check fails (codes 2 / 3) or nearly so."""
    mats, rhs = [], []
    for _ in range(200):
        n = int(rng.integers(3, 30))
        m = rng.standard_normal((n, n)) * np.exp(rng.uniform(-1, 1, (n, n)) * rng.uniform(5, 25))
        b = rng.standard_normal(n) * 10.0 ** rng.uniform(-3, 8)
        if rng.random() < 0.5:
            b = np.abs(b)
        mats.append(m)
        rhs.append(b)
    return mats, rhs


def main() -> None:
    oracle.build_port()
    if not oracle.available("ref"):
        raise SystemExit("build the reference first: make -C oracle ref")
    rng = np.random.default_rng(wl.BASE_SEED + 100)

    # ---- the reference's own fixtures ------------------------------------
    out = {}
    for name in ("small_matrix", "matrix_ion"):
        A = read_fixture(FIX / name / "A.txt")
        b = read_fixture(FIX / name / "b.txt")
        x = read_fixture(FIX / name / "x.txt")
        batch = wl.from_matrices("solve", [A], [b])
        xr, sr = oracle.solve(batch, "ref")
        out[f"{name}_A"], out[f"{name}_b"], out[f"{name}_x_fixture"] = A, b, x
        out[f"{name}_x_ref"], out[f"{name}_code_ref"] = xr, sr
    for name in ("inverse_small", "inverse_macro"):
        M = read_fixture(FIX / name / "matrix.txt")
        Minv = read_fixture(FIX / name / "inverse.txt")
        batch = wl.from_matrices("invert", [M])
        ir, sr = oracle.invert(batch, "ref")
        out[f"{name}_M"], out[f"{name}_inv_fixture"] = M, Minv
        out[f"{name}_inv_ref"], out[f"{name}_code_ref"] = ir.reshape(M.shape), sr
    np.savez_compressed(HERE / "reference_fixtures.npz", **out)

    # ---- seeded solve cases ------------------------------------------------
    mats, rhs = [], []
    for n in list(range(1, 41)) + [44, 48, 56, 64]:
        m = rng.standard_normal((n, n))
        mats.append(m)
        rhs.append(rng.standard_normal(n))
    for conservation in ("last", "first"):
        for n in list(wl.ION_SIZES_PER_CELL) * 4 + [27] * 20 + [64, 178]:
            a, b = wl.ion_matrix(rng, int(n), conservation=conservation)
            mats.append(a)
            rhs.append(b)
    for m in singular_cases(rng):
        mats.append(m)
        rhs.append(rng.standard_normal(m.shape[0]))
    fm, fr = residual_failure_cases(rng)
    mats += fm
    rhs += fr
    sb = wl.from_matrices("solve", mats, rhs)
    xs, ss = oracle.solve(sb, "ref")
    np.savez_compressed(HERE / "solve_cases.npz", n=sb.n, offA=sb.offA, A=sb.A, offv=sb.offv, b=sb.b,
                        x_ref=xs, status_ref=ss)
    print("solve cases:", sb.nsys, "codes", np.bincount(ss, minlength=5))

    # ---- seeded invert cases -----------------------------------------------
    mats = []
    for n in list(range(1, 41)) + [44, 48, 56, 61, 64]:
        mats.append(rng.standard_normal((n, n)))
    for n in [61] * 4 + [20, 33, 76]:
        mats.append(wl.macro_matrix(rng, int(n)))
    mats += singular_cases(rng)
    ib = wl.from_matrices("invert", mats)
    inv, si = oracle.invert(ib, "ref")
    np.savez_compressed(HERE / "invert_cases.npz", n=ib.n, offA=ib.offA, A=ib.A, inv_ref=inv, status_ref=si)
    print("invert cases:", ib.nsys, "codes", np.bincount(si, minlength=2))


def nonfinite_cases(rng):
    """Macro-atom and dense matrices with one +Inf, -Inf or NaN entry, and a few
    with several: the reference's invert_matrix returns 21 (GSL_ESING) where an
    infinite value reaches the diagonal of U, 1 for an exact zero pivot, else 0;
    its solve_matrix returns 4 or 0 and leaves the residual test to NaN."""
    mats = []
    for n in (2, 3, 5, 9, 17, 24, 31, 33, 48, 61, 65, 70):
        for k in range(6):
            m = wl.macro_matrix(rng, n) if k % 2 == 0 else rng.standard_normal((n, n))
            i, j = rng.integers(0, n, 2)
            m[i, j] = (np.inf, -np.inf, np.nan)[k % 3]
            if k == 5 and n > 3:
                m[rng.integers(n), rng.integers(n)] = np.inf
                m[rng.integers(n)] = 0.0
            mats.append(m)
    return mats


def main_nonfinite() -> None:
    rng = np.random.default_rng(wl.BASE_SEED + 101)
    mats = nonfinite_cases(rng)
    ib = wl.from_matrices("invert", mats)
    inv, si = oracle.invert(ib, "ref")
    sb = wl.from_matrices("solve", mats, [rng.standard_normal(m.shape[0]) for m in mats])
    xs, ss = oracle.solve(sb, "ref")
    np.savez_compressed(HERE / "nonfinite_cases.npz", n=ib.n, offA=ib.offA, A=ib.A, inv_ref=inv,
                        inv_status_ref=si, offv=sb.offv, b=sb.b, x_ref=xs, solve_status_ref=ss)
    print("non-finite cases:", ib.nsys, "invert codes", np.unique(si, return_counts=True),
          "solve codes", np.unique(ss, return_counts=True))


if __name__ == "__main__":
    # python tests/golden/make_golden.py [--only nonfinite]
    if sys.argv[1:] == ["--only", "nonfinite"]:
        oracle.build_port()
        main_nonfinite()
    else:
        main()
        main_nonfinite()
