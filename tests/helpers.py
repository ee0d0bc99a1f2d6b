"""Comparison helpers shared by the parity tests."""
import numpy as np

from python_b200 import workloads as wl


def batch_from_golden(g, kind):
    if kind == "solve":
        return wl.Batch("solve", g["n"].astype(np.int32), g["offA"], g["A"], g["offv"], g["b"])
    return wl.Batch("invert", g["n"].astype(np.int32), g["offA"], g["A"])


def same_values(a, b):
    """Elementwise equality that treats NaN == NaN and +0 == -0."""
    return (a == b) | (np.isnan(a) & np.isnan(b))


def population_rel_err(x, ref, n, offv, floor=1e-20):
    """Largest relative error over components above floor * sum|ref| of each system."""
    worst = 0.0
    for s in range(n.size):
        o, k = int(offv[s]), int(n[s])
        r = ref[o:o + k]
        v = x[o:o + k]
        tot = np.sum(np.abs(r))
        sig = np.abs(r) > floor * tot
        if sig.any():
            worst = max(worst, float(np.max(np.abs(v[sig] - r[sig]) / np.abs(r[sig]))))
    return worst


def inverse_rel_err(inv, ref, n, offA, mask=None):
    """Largest normwise (max-abs) relative difference per matrix."""
    worst = 0.0
    for s in range(n.size):
        if mask is not None and not mask[s]:
            continue
        o, k = int(offA[s]), int(n[s])
        r = ref[o:o + k * k]
        v = inv[o:o + k * k]
        worst = max(worst, float(np.max(np.abs(v - r)) / max(np.max(np.abs(r)), 1e-300)))
    return worst


def backward_err(A, x, b):
    """Normwise backward error |b - A x|_inf / (|A|_inf |x|_inf + |b|_inf)."""
    r = b - A @ x
    return float(np.max(np.abs(r)) / (np.max(np.sum(np.abs(A), axis=1)) * np.max(np.abs(x)) + np.max(np.abs(b))))
