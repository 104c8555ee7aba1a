"""Double-buffered history upload (pct_stage_reconstruction_histories / pct_use_staged_histories).

Staging a new set of histories while the current one is being reconstructed must not disturb the
running iteration, and using the staged set must give exactly what loading it directly gives.  The
deterministic scatter makes both comparisons bit for bit.
"""
import numpy as np
import pytest

from pct_reconstruction_b200 import Config
from pct_reconstruction_b200 import phantoms as P
from pct_reconstruction_b200.engine import PCTError


def _scan(cfg, seed):
    tr = P.simulate_tracks(P.water_cylinder_phantom(6.0), 40000, seed=seed)
    return {k: v.numpy() for k, v in P.reconstruction_histories(cfg, tr).items()}


@pytest.mark.gpu
def test_staged_histories_match_direct_loading(c1_params):
    import torch
    from pct_reconstruction_b200 import Context
    cfg = Config(**dict(c1_params, SCATTER_MODE="DETERMINISTIC"))
    h1, h2 = _scan(cfg, 91), _scan(cfg, 92)
    n = min(len(h1["WEPL"]), len(h2["WEPL"]))
    h1 = {k: v[:n].copy() for k, v in h1.items()}
    h2 = {k: v[:n].copy() for k, v in h2.items()}
    x = (0.95 + 0.1 * np.random.default_rng(5).random(cfg.NUM_VOXELS)).astype(np.float32)
    with Context(cfg) as ref:
        ref.set_reconstruction_histories(h1)
        ref.x_host_2_GPU(x)
        ref.DROP_full_tx_iteration(1)
        x1 = ref.x_GPU_2_host()
        ref.set_reconstruction_histories(h2)
        ref.DROP_full_tx_iteration(2)
        x2 = ref.x_GPU_2_host()
    pinned = {k: torch.from_numpy(v).pin_memory() for k, v in h2.items()}
    with Context(cfg) as ctx:
        with pytest.raises(PCTError):
            ctx.use_staged_histories()  # nothing staged yet
        ctx.stage_reconstruction_histories(h1)
        ctx.use_staged_histories()
        ctx.x_host_2_GPU(x)
        ctx.stage_reconstruction_histories(pinned)  # uploads while iteration 1 runs on h1
        ctx.DROP_full_tx_iteration(1)
        y1 = ctx.x_GPU_2_host()
        ctx.use_staged_histories()
        ctx.DROP_full_tx_iteration(2)
        y2 = ctx.x_GPU_2_host()
    np.testing.assert_array_equal(y1, x1)
    np.testing.assert_array_equal(y2, x2)
    assert np.abs(x2 - x1).max() > 0
