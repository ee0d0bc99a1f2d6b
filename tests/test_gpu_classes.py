"""Every candidate configuration of a CTA size class returns the same bits.

The engine picks one configuration per padded order from the autotuner's
timings (shared-memory or global-workspace matrix, panel warps, update tiles,
CTAs per SM); a result must not depend on that choice.  Orders are chosen so
that the last panel is short and update chunks straddle the panel."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tune():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    from python_b200 import autotune
    return autotune.load_tune_lib()


@pytest.mark.parametrize("p,n", [(48, 45), (64, 61), (64, 50), (96, 93), (128, 115), (192, 181), (256, 250)])
def test_candidates_agree(tune, p, n):
    import torch

    from python_b200 import workloads as wl
    lib, cands = tune
    from python_b200 import autotune
    mine = [c for c in cands if c[1][0] == p]
    assert len(mine) >= 2, p
    batch = wl.macro_batch([n] * 300, seed=77 + n)
    dev = torch.device("cuda", 0)
    ref = None
    for i, cfg in mine:
        out, st, ms, _ = autotune.run_candidate(lib, i, batch, dev)
        assert out is not None, (cfg, ms)
        assert (st == 0).all(), cfg
        if ref is None:
            ref = (cfg, out, st)
            continue
        assert np.array_equal(st, ref[2]), (cfg, ref[0])
        assert out.tobytes() == ref[1].tobytes(), f"{cfg} differs from {ref[0]} at n={n}"


@pytest.mark.parametrize("p,n", [(64, 57), (112, 105), (192, 185)])
def test_certified_shapes_agree(p, n):
    """Every candidate shape of a certified class (tile-warp grid, R' in
    registers or in shared memory, staging) returns code 0 and inverses within
    1e-12 of the first shape's: the tuner may pick any of them."""
    torch = pytest.importorskip("torch")
    from python_b200 import autotune
    from python_b200 import workloads as wl
    libs = autotune.build_cgj_tune_libs()
    lib, cands = autotune.load_cgj_lib(libs[p])
    assert len(cands) >= 2, p
    db = autotune._DeviceBatch(wl.macro_batch([n] * 400, seed=91 + n), torch.device("cuda", 0))
    ref = None
    for i, cfg in cands:
        out, st, ms, _ = autotune.run_cgj(lib, i, db, 1)
        assert out is not None, (cfg, ms)
        assert (st == 0).all(), cfg
        if ref is None:
            ref = out
            continue
        assert np.max(np.abs(out - ref)) <= autotune.CGJ_AGREE * np.max(np.abs(ref)), cfg
