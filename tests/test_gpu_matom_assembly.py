"""GPU assembly of the macro-atom jump matrices (matom_rate_matrices_batched)
against the restatement of calc_matom_matrix's Q / R assembly
(oracle.matom_rate_matrix, pinned to the reference's own build by
tests/test_oracle_matom_assembly.py): N and R bit for bit.  Device outputs
then feed matom_matrices_batched, whose B matches B from the oracle's inverse
within the inverse's tolerance."""
import numpy as np
import pytest

from oracle import oracle
from python_b200 import engine, workloads as wl

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("levels,seed,ncell", [((12, 20, 16, 9, 1), 7, 24), ((6, 30, 25, 4, 1), 99, 12),
                                               ((3, 2, 1), 5, 8),
                                               ((60, 80, 60, 1), 3, 3)])   # 201 levels: rows built in place
def test_assembly_matches_restatement(levels, seed, ncell):
    m = wl.matom_model(ion_levels=levels, seed=seed)
    cells = [wl.matom_cell(m, 1000 * seed + c) for c in range(ncell)]
    N, R = engine.matom_rate_matrices(wl.matom_jump_inputs(m, cells))
    for c, cell in enumerate(cells):
        Nr, Rr = oracle.matom_rate_matrix(m, cell)
        assert N[c].tobytes() == Nr.tobytes(), (levels, c)
        assert R[c].tobytes() == Rr.tobytes(), (levels, c)


def test_device_outputs_feed_the_matom_epilogue():
    import torch
    m = wl.matom_model()
    ncell = 16
    cells = [wl.matom_cell(m, 50 + c) for c in range(ncell)]
    nr = m.nlev + 1
    dN = torch.empty((ncell, nr, nr), dtype=torch.float64, device="cuda")
    dR = torch.empty((ncell, nr), dtype=torch.float64, device="cuda")
    engine.matom_rate_matrices(wl.matom_jump_inputs(m, cells), dN, dR)
    torch.cuda.synchronize()
    N, R = dN.cpu().numpy(), dR.cpu().numpy()
    Nh, Rh = engine.matom_rate_matrices(wl.matom_jump_inputs(m, cells))
    assert N.tobytes() == Nh.tobytes() and R.tobytes() == Rh.tobytes()
    batch = wl.from_matrices("invert", [N[c] for c in range(ncell)])
    offv = np.arange(ncell, dtype=np.int64) * nr
    B, C, st = engine.matom_matrices(batch, R.reshape(-1), offv)
    assert (st == 0).all()
    inv, sto = oracle.invert(batch, "port")
    for c in range(ncell):
        Bo = inv[c * nr * nr:(c + 1) * nr * nr].reshape(nr, nr) * R[c][None, :]
        Bg = B[c * nr * nr:(c + 1) * nr * nr].reshape(nr, nr)
        scale = np.abs(Bo).max()
        assert np.abs(Bg - Bo).max() <= 1e-10 * scale, c


def test_assembly_rejects_bad_targets():
    m = wl.matom_model()
    inp = wl.matom_jump_inputs(m, [wl.matom_cell(m, 1)])
    inp["bbu_target"] = inp["bbu_target"].copy()
    inp["bbu_target"][0] = m.nlev                  # the k-packet is not a jump target
    with pytest.raises(engine.EngineError):
        engine.matom_rate_matrices(inp)
