"""The restatement of calc_matom_matrix's Q / R assembly and normalisation
(oracle.matom_rate_matrix) against the reference's own routine, compiled from
source/macro_accelerate.c into oracle/_ref/libref_matom.so: N and R from the
restatement, inverted by the reference's own invert_matrix and multiplied as
the routine does (:314-334), give the routine's B bit for bit.  The models
have simple and macro lines, Auger levels, clamped negative upward bound-free
rates, zero downward ones and lower densities under DENSITY_PHOT_MIN."""
import numpy as np
import pytest

from oracle import oracle
from python_b200 import workloads as wl

pytestmark = pytest.mark.skipif(not (oracle.matom_reference_available() and oracle.available("ref")),
                                reason="the reference's macro_accelerate.c build (oracle/_ref) is not present")


@pytest.mark.parametrize("levels,seed", [((12, 20, 16, 9, 1), 7), ((6, 30, 25, 4, 1), 99), ((3, 2, 1), 5)])
def test_restatement_matches_reference_build(levels, seed):
    m = wl.matom_model(ion_levels=levels, seed=seed)
    nr = m.nlev + 1
    for c in range(3):
        cell = wl.matom_cell(m, 10 * seed + c)
        N, R = oracle.matom_rate_matrix(m, cell)
        inv, st = oracle.invert(wl.from_matrices("invert", [N.copy()]), "ref")
        assert st[0] == 0
        inv = inv.reshape(nr, nr)
        B = np.empty((nr, nr))
        for i in range(nr):
            for j in range(nr):
                B[i, j] = inv[i, j] * R[j]
        assert B.tobytes() == oracle.ref_matom_b(m, cell).tobytes(), (levels, c)
