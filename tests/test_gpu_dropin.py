"""The drop-in at the link level: the reference's own calc_matom_matrix
(source/macro_accelerate.c:31-348, compiled unmodified from the reference tree)
linked against this engine instead of matrix_cpu.c and GSL.  Its call of
invert_matrix (macro_accelerate.c:315) then resolves to the engine's C ABI
(oracle/_ref/libref_matom_dropin.so needs libsirocco_solve.so and no GSL), and
the B it forms must be the reference build's to within the inverse tolerance,
and bit for bit the engine's own inverse of the same N times R."""
import numpy as np
import pytest

from oracle import oracle
from python_b200 import workloads as wl

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (oracle.MATOM_DROPIN_LIB.exists() and oracle.matom_reference_available()),
                                 reason="the reference's macro_accelerate.c builds (oracle/_ref) are not present")]

INV_TOL = 1e-10


@pytest.mark.parametrize("levels,seed", [((12, 20, 16, 9, 1), 7), ((6, 30, 25, 4, 1), 99), ((3, 2, 1), 5)])
def test_reference_routine_on_the_engine(engine, levels, seed):
    m = wl.matom_model(ion_levels=levels, seed=seed)
    nr = m.nlev + 1
    for c in range(3):
        cell = wl.matom_cell(m, 10 * seed + c)
        b_gsl = oracle.ref_matom_b(m, cell)
        b_eng = oracle.ref_matom_b(m, cell, dropin=True)
        assert np.max(np.abs(b_eng - b_gsl)) <= INV_TOL * np.max(np.abs(b_gsl)), (levels, c)
        # the routine's B is the engine's inverse times R, as the routine forms it
        N, R = oracle.matom_rate_matrix(m, cell)
        inv, st = engine.invert_batched(wl.from_matrices("invert", [N.copy()]), engine.FP64)
        assert st[0] == 0
        want = inv.reshape(nr, nr) * R[None, :]
        assert want.tobytes() == b_eng.tobytes(), (levels, c)
