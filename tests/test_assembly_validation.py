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
