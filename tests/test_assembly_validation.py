"""Host-side checks of matom_rate_matrices_batched, which run before any CUDA
call: malformed jump lists are rejected with SIROCCO_EINVAL and a message."""
import numpy as np
import pytest

from python_b200 import engine, workloads as wl


def _inputs():
    m = wl.matom_model()
    return m, wl.matom_jump_inputs(m, [wl.matom_cell(m, 1)])


@pytest.mark.parametrize("key,bad", [("bbu_target", "level"), ("bfd_target", "negative"),
                                     ("kbb_target", "level"), ("bbd_start", "descend")])
def test_malformed_tables_are_rejected(key, bad):
    m, inp = _inputs()
    a = inp[key].copy()
    if bad == "level":
        a[0] = m.nlev                              # the k-packet is no jump target
    elif bad == "negative":
        a[0] = -1
    else:
        a[3] = a[2] - 1                            # starts must not descend
    inp[key] = a
    with pytest.raises(engine.EngineError):
        engine.matom_rate_matrices(inp)
    assert engine.last_error()


def _ion_case(kind):
    tab = wl.ion_table()
    rates = wl.ion_rates(tab, 2)
    if kind == "cxr_neutral":
        rates.cxr[1, int(tab.elem_first[2])] = 1e-9          # lands in another element's block
    elif kind == "cx_last_ion":
        last = int(tab.elem_first[3] + tab.elem_n[3] - 1)
        tab.cx_nion1 = np.append(tab.cx_nion1, np.int32(last))
        tab.cx_nion2 = np.append(tab.cx_nion2, np.int32(1))   # against H II
        rates = wl.ion_rates(tab, 2)
    elif kind == "yield_row":
        tab.inner_yield = tab.inner_yield.copy()
        tab.inner_yield[0] = len(tab.yield_prob)              # no such row
    elif kind == "overlap":
        tab.elem_first = tab.elem_first.copy()
        tab.elem_first[1] = 1                                 # He starts inside H
    return tab, rates


@pytest.mark.parametrize("kind", ["cxr_neutral", "cx_last_ion", "yield_row", "overlap"])
def test_malformed_ion_tables_are_rejected(kind):
    tab, rates = _ion_case(kind)
    with pytest.raises(engine.EngineError):
        engine.ion_rate_matrices(tab, rates, np.ones(2), np.ones(2), np.ones(2))
    assert engine.last_error()
