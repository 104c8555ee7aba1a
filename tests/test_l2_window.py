"""L2 persistence window (pct_set_l2_window).

The window only changes which L2 lines the hardware keeps, never an arithmetic result: with the
deterministic scatter the images with and without it are bit-identical, and switching it off again
restores the plain captured iteration.
"""
import numpy as np
import pytest

from pct_reconstruction_b200 import Config
from pct_reconstruction_b200 import phantoms as P


@pytest.mark.gpu
def test_l2_window_leaves_images_bit_identical(c1_params):
    from pct_reconstruction_b200 import Context
    params = dict(c1_params, SCATTER_MODE="DETERMINISTIC")
    cfg = Config(**params)
    tr = P.simulate_tracks(P.water_cylinder_phantom(6.0), 40000, seed=82)
    hist = {k: v.numpy() for k, v in P.reconstruction_histories(cfg, tr).items()}
    x = (0.95 + 0.1 * np.random.default_rng(4).random(cfg.NUM_VOXELS)).astype(np.float32)
    images = []
    for window in (False, True, False):
        with Context(cfg) as ctx:
            ctx.set_reconstruction_histories(hist)
            ctx.x_host_2_GPU(x)
            ctx.set_l2_window(window)
            ctx.DROP_full_tx_iteration(1)
            if window:
                ctx.set_l2_window(False)
                ctx.set_l2_window(True)  # toggling rebuilds the captured iteration
            ctx.DROP_full_tx_iteration(2)
            images.append(ctx.x_GPU_2_host())
    assert np.abs(images[0] - x).max() > 0
    np.testing.assert_array_equal(images[1], images[0])
    np.testing.assert_array_equal(images[2], images[0])
