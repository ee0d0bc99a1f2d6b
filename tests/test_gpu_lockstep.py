"""Lock-step n_e iteration (ion_populations_lockstep) against a restatement of
the reference's per-cell loop, matrix_ion_populations
(source/matrix_ion.c:219-382), solving each cell's FULL block-diagonal rate
matrix with the oracle: equal statuses, round counts, n_e and populations, bit
for bit."""
import numpy as np
import pytest

from oracle import oracle
from python_b200 import workloads as wl

DENSITY_MIN, FRACTIONAL_ERROR, MAXITERATIONS = 1e-20, 0.03, 200
ELEM_N = np.array([2, 3, 7, 27], np.int32)          # H, He, C, Fe
ELEM_FIRST = np.concatenate([[0], np.cumsum(ELEM_N)[:-1]]).astype(np.int32)
NIONS = int(ELEM_N.sum())
ISTATE = np.concatenate([np.arange(1, k + 1) for k in ELEM_N]).astype(np.int32)
ABUND = np.array([1.0, 0.1, 3e-4, 3e-5])


class Model:
    """Per-cell rates: ionisation out of each stage (He's raised by charge
    exchange with ionised hydrogen) and recombination proportional to n_e."""

    def __init__(self, ncell, seed):
        rng = np.random.default_rng(seed)
        self.ion = np.exp(rng.uniform(np.log(1e-3), np.log(1e2), (ncell, NIONS)))
        self.alpha = np.exp(rng.uniform(np.log(1e-13), np.log(1e-10), (ncell, NIONS)))
        self.chi = np.exp(rng.uniform(np.log(1e-12), np.log(1e-9), ncell))
        nh = np.exp(rng.uniform(np.log(1e8), np.log(1e12), ncell))
        nh[3] = 1e-9                                  # nearly empty cell: n_e below 1e-6 at once
        self.elem_dens = nh[:, None] * ABUND[None, :]
        self.ion[5, ELEM_FIRST[3]:] = 0.0             # a cell whose Fe block has no rates: singular
        self.alpha[5, ELEM_FIRST[3]:] = 0.0

    def blocks(self, c, ne, nh1, nh2):
        out = []
        for e, (f, n) in enumerate(zip(ELEM_FIRST, ELEM_N)):
            m = np.zeros((n, n))
            for k in range(n - 1):
                up = self.ion[c, f + k] + (self.chi[c] * nh2 if e == 1 else 0.0)
                down = self.alpha[c, f + k] * ne
                m[k + 1, k] += up
                m[k, k] -= up
                m[k, k + 1] += down
                m[k + 1, k + 1] -= down
            m[0, :] = 1.0                             # conservation row first (matrix_ion.c:633-655)
            b = np.zeros(n)
            b[0] = 1.0
            out.append((m, b))
        return out

    def assemble(self, cells, ne, nh1, nh2, A, b):
        blk = int((ELEM_N.astype(np.int64) ** 2).sum())
        for i, c in enumerate(cells):
            oa = i * blk
            for e, (m, v) in enumerate(self.blocks(int(c), ne[i], nh1[i], nh2[i])):
                A[oa:oa + m.size] = m.ravel()
                oa += m.size
                b[i * NIONS + ELEM_FIRST[e]:i * NIONS + ELEM_FIRST[e] + m.shape[0]] = v


def reference_cell(model, c, ne0, den0):
    """matrix_ion_populations for one cell on its full nions x nions matrix."""
    xne = ne0
    newden = den0.copy()
    elem_of = np.repeat(np.arange(len(ELEM_N)), ELEM_N)
    for it in range(MAXITERATIONS):
        nh1 = nh2 = 0.0
        for nn in range(NIONS):
            if elem_of[nn] == 0 and ISTATE[nn] == 1:
                nh1 = newden[nn] * model.elem_dens[c, 0]
            if elem_of[nn] == 0 and ISTATE[nn] == 2:
                nh2 = newden[nn] * model.elem_dens[c, 0]
        full = np.zeros((NIONS, NIONS))
        rhs = np.zeros(NIONS)
        for e, (m, v) in enumerate(model.blocks(c, xne, nh1, nh2)):
            f = ELEM_FIRST[e]
            full[f:f + m.shape[0], f:f + m.shape[0]] = m
            rhs[f:f + m.shape[0]] = v
        x, st = oracle.solve(wl.from_matrices("solve", [full], [rhs]), "port", threads=1)
        if st[0] == 4:
            return -1, it + 1, ne0, den0
        newden = np.where(x < DENSITY_MIN, DENSITY_MIN, x)
        xnew = 0.0
        for nn in range(NIONS):
            xnew += newden[nn] * (ISTATE[nn] - 1) * model.elem_dens[c, elem_of[nn]]
        if xnew < DENSITY_MIN:
            xnew = DENSITY_MIN
        if abs((xne - xnew) / xnew) < FRACTIONAL_ERROR or xnew < 1.e-6:
            return 0, it + 1, xnew, newden
        xne = (xnew + xne) / 2.
    return -2, MAXITERATIONS, ne0, den0


@pytest.mark.gpu
def test_lockstep_matches_reference_loop(engine):
    ncell = 48
    model = Model(ncell, seed=4)
    ne = model.elem_dens[:, 0].copy()                # start fully ionised hydrogen
    den = np.concatenate([np.full(k, 1.0 / k) for k in ELEM_N])[None, :].repeat(ncell, 0).copy()
    ne0, den0 = ne.copy(), den.copy()
    status, iters = engine.ion_populations_lockstep(ELEM_FIRST, ELEM_N, ISTATE, 0, model.elem_dens, ne, den,
                                                    model.assemble)
    assert status[5] == -1 and status[3] == 0
    assert (iters > 1).sum() > ncell // 2           # most cells need several rounds
    for c in range(ncell):
        st, it, ref_ne, ref_den = reference_cell(model, c, ne0[c], den0[c])
        assert status[c] == st and iters[c] == it, c
        assert ne[c] == ref_ne, c
        assert np.array_equal(den[c], ref_den), c
