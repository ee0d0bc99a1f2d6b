"""GPU assembly of the ion rate matrices (ion_rate_matrices_batched) against the
restatement of populate_ion_rate_matrix (source/matrix_ion.c:444-659), which
tests/test_oracle_ionmat.py pins to the reference's own build: every block
entry and right-hand side bit for bit.  Then the lock-step driver that
assembles on the GPU (ion_populations_lockstep_rates) against the callback
driver fed the restatement's blocks: equal statuses, rounds, n_e and
populations, bit for bit."""
import numpy as np
import pytest

from oracle import oracle
from python_b200 import engine, workloads as wl

pytestmark = pytest.mark.gpu


def _blocks(tab, A, b, cell):
    """Cell `cell`'s element blocks out of the packed layout."""
    blk = int((tab.elem_n.astype(np.int64) ** 2).sum())
    out, oa = [], cell * blk
    for e in range(tab.nelem):
        n = int(tab.elem_n[e])
        out.append(A[oa:oa + n * n].reshape(n, n))
        oa += n * n
    return out


def _tables():
    yield wl.ion_table(), 64
    yield wl.ion_table(zs=(1, 2, 7, 10, 14, 26, 30), seed=11), 40   # Zn: a 31-ion block
    t = wl.ion_table(zs=(1, 6, 8), seed=12)
    t.cx_nion1, t.cx_nion2 = t.cx_nion1[:0], t.cx_nion2[:0]
    yield t, 16


@pytest.mark.parametrize("case", range(3))
def test_assembly_matches_reference_restatement(case):
    tab, ncell = list(_tables())[case]
    rates = wl.ion_rates(tab, ncell, seed=200 + case)
    rng = np.random.default_rng(7 + case)
    ne = 10 ** rng.uniform(0, 13, ncell)
    nh1, nh2 = 10 ** rng.uniform(-3, 8, ncell), 10 ** rng.uniform(2, 12, ncell)
    A, b = engine.ion_rate_matrices(tab, rates, ne, nh1, nh2)
    for c in range(ncell):
        Ar, br = oracle.ion_rate_matrix(tab, rates, c, float(ne[c]), float(nh1[c]), float(nh2[c]))
        assert b[c].tobytes() == br.tobytes(), (case, c)
        for e, blk in enumerate(_blocks(tab, A, b, c)):
            f, n = int(tab.elem_first[e]), int(tab.elem_n[e])
            assert blk.tobytes() == np.ascontiguousarray(Ar[f:f + n, f:f + n]).tobytes(), (case, c, e)


def test_assembly_rejects_terms_outside_a_block():
    tab = wl.ion_table()
    rates = wl.ion_rates(tab, 4)
    f = int(tab.elem_first[2])                       # the neutral ion of a metal
    rates.cxr[1, f] = 1e-9                           # its charge-exchange term lands in another element
    with pytest.raises(engine.EngineError):
        engine.ion_rate_matrices(tab, rates, np.ones(4), np.ones(4), np.ones(4))
    tab2 = wl.ion_table()
    last = int(tab2.elem_first[3] + tab2.elem_n[3] - 1)
    tab2.cx_nion1 = np.append(tab2.cx_nion1, np.int32(last))   # ionising the bare ion
    tab2.cx_nion2 = np.append(tab2.cx_nion2, np.int32(1))
    rates2 = wl.ion_rates(tab2, 2)
    with pytest.raises(engine.EngineError):
        engine.ion_rate_matrices(tab2, rates2, np.ones(2), np.ones(2), np.ones(2))


def test_lockstep_with_gpu_assembly_matches_callback_driver():
    tab = wl.ion_table()
    ncell = 48
    rates = wl.ion_rates(tab, ncell, seed=300)
    rng = np.random.default_rng(301)
    abund = np.array([1.0, 0.1, 3e-4, 5e-4, 3e-5])
    nh = np.exp(rng.uniform(np.log(1e6), np.log(1e12), ncell))
    nh[3] = 1e-9                                     # a nearly empty cell
    elem_dens = nh[:, None] * abund[None, :]
    den0 = np.zeros((ncell, tab.nions))
    for e in range(tab.nelem):
        den0[:, tab.elem_first[e]] = 1.0             # start neutral
    ne0 = 0.1 * nh
    h_elem = 0
    blk = int((tab.elem_n.astype(np.int64) ** 2).sum())

    def assemble(cells, ne, nh1, nh2, A, b):
        for i, c in enumerate(cells):
            Ar, br = oracle.ion_rate_matrix(tab, rates, int(c), float(ne[i]), float(nh1[i]), float(nh2[i]))
            oa = i * blk
            for e in range(tab.nelem):
                f, n = int(tab.elem_first[e]), int(tab.elem_n[e])
                A[oa:oa + n * n] = Ar[f:f + n, f:f + n].ravel()
                oa += n * n
            b[i * tab.nions:(i + 1) * tab.nions] = br

    ne_a, den_a = ne0.copy(), den0.copy()
    st_a, it_a = engine.ion_populations_lockstep(tab.elem_first, tab.elem_n, tab.ion_istate, h_elem, elem_dens,
                                                 ne_a, den_a, assemble)
    ne_b, den_b = ne0.copy(), den0.copy()
    st_b, it_b = engine.ion_populations_lockstep_rates(tab, rates, h_elem, elem_dens, ne_b, den_b)
    assert np.array_equal(st_a, st_b) and np.array_equal(it_a, it_b)
    assert ne_a.tobytes() == ne_b.tobytes()
    assert den_a.tobytes() == den_b.tobytes()
    assert (st_a == 0).sum() > ncell // 2, st_a
