"""The restatement of populate_ion_rate_matrix (oracle.ion_rate_matrix) against
the reference's own routine, compiled from source/matrix_ion.c into
oracle/_ref/libref_ionmat.so: identical matrices and right-hand sides, bit for
bit, on synthetic atomic tables with direct-ionisation and dielectronic flags,
inner-shell yields (with and without yield data) and charge exchange."""
import numpy as np
import pytest

from oracle import oracle
from python_b200 import workloads as wl

pytestmark = pytest.mark.skipif(not oracle.ion_reference_available(),
                                reason="the reference's matrix_ion.c build (oracle/_ref) is not present")


def _cases():
    yield wl.ion_table(), 6
    yield wl.ion_table(zs=(1, 2, 7, 10, 14, 26, 30), seed=11), 4   # Zn: a 31-ion block
    t = wl.ion_table(zs=(1, 6, 8), seed=12)          # no charge-exchange entries at all
    t.cx_nion1 = t.cx_nion1[:0]
    t.cx_nion2 = t.cx_nion2[:0]
    yield t, 4


@pytest.mark.parametrize("case", range(3))
def test_restatement_matches_reference_build(case):
    tab, ncell = list(_cases())[case]
    rates = wl.ion_rates(tab, ncell, seed=100 + case)
    rng = np.random.default_rng(case)
    for c in range(ncell):
        xne = float(10 ** rng.uniform(0, 13))
        nh1, nh2 = float(10 ** rng.uniform(-3, 8)), float(10 ** rng.uniform(2, 12))
        A, b = oracle.ion_rate_matrix(tab, rates, c, xne, nh1, nh2)
        Ar, br, rc = oracle.ref_ion_rate_matrix(tab, rates, c, xne, nh1, nh2)
        assert rc == 0
        assert A.tobytes() == Ar.tobytes(), (case, c)
        assert b.tobytes() == br.tobytes(), (case, c)
        # block-diagonal by element, as the per-element systems assume
        eo = tab.elem_of()
        assert not np.any(A[eo[:, None] != eo[None, :]])
