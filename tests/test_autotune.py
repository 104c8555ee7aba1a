"""Schedule autotuner (pct_autotune / pct_autotune_schedule).

The autotuner times DROP iterations of the loaded histories for several path-kernel chunkings,
path-kernel CTA sizes (histories per CTA) and path-order windows, and keeps the fastest of each.
These reorder launches and work only: the image it leaves behind is the one it found, and later
iterations give exactly what an untuned context gives (deterministic scatter, bit for bit).
"""
import numpy as np
import pytest

from pct_reconstruction_b200 import Config
from pct_reconstruction_b200 import phantoms as P
from pct_reconstruction_b200.engine import PCTError


def test_config_accepts_only_the_implemented_lanes_per_history():
    assert Config(THREADS_PER_HISTORY=32).THREADS_PER_HISTORY == 32
    with pytest.raises(PCTError):
        Config(THREADS_PER_HISTORY=8)


def test_config_accepts_only_the_implemented_schedules():
    assert Config(PATH_CTA_THREADS=64).PATH_CTA_THREADS == 64
    assert Config(PATH_ORDER_WINDOW=4096).PATH_ORDER_WINDOW == 4096
    assert Config().PATH_CTA_THREADS == 128 and Config().PATH_ORDER_WINDOW == 0
    with pytest.raises(PCTError):
        Config(PATH_CTA_THREADS=96)
    with pytest.raises(PCTError):
        Config(PATH_ORDER_WINDOW=-1)


@pytest.mark.gpu
def test_every_schedule_gives_the_same_image(c1_params):
    from pct_reconstruction_b200 import Context
    base = dict(c1_params, SCATTER_MODE="DETERMINISTIC")
    cfg = Config(**base)
    tr = P.simulate_tracks(P.water_cylinder_phantom(6.0), 40000, seed=85)
    hist = {k: v.numpy() for k, v in P.reconstruction_histories(cfg, tr).items()}
    x = (0.95 + 0.1 * np.random.default_rng(7).random(cfg.NUM_VOXELS)).astype(np.float32)
    images = []
    for cta, window in ((128, 0), (64, 0), (256, 0), (128, 4096), (64, 1000)):
        with Context(Config(**base, PATH_CTA_THREADS=cta, PATH_ORDER_WINDOW=window)) as ctx:
            ctx.set_reconstruction_histories(hist)
            ctx.x_host_2_GPU(x)
            ctx.DROP_full_tx_iteration(1)
            images.append(ctx.x_GPU_2_host())
    for im in images[1:]:
        np.testing.assert_array_equal(im, images[0])


@pytest.mark.gpu
def test_autotune_keeps_the_image_and_the_results(c1_params):
    from pct_reconstruction_b200 import Context
    cfg = Config(**dict(c1_params, SCATTER_MODE="DETERMINISTIC"))
    tr = P.simulate_tracks(P.water_cylinder_phantom(6.0), 60000, seed=84)
    hist = {k: v.numpy() for k, v in P.reconstruction_histories(cfg, tr).items()}
    x = (0.95 + 0.1 * np.random.default_rng(6).random(cfg.NUM_VOXELS)).astype(np.float32)
    with Context(cfg) as ref:
        ref.set_reconstruction_histories(hist)
        ref.x_host_2_GPU(x)
        ref.DROP_full_tx_iteration(1)
        ref.DROP_full_tx_iteration(2)
        expected = ref.x_GPU_2_host()
    with Context(cfg) as ctx:
        ctx.set_reconstruction_histories(hist)
        ctx.x_host_2_GPU(x)
        chosen = ctx.autotune_schedule()
        assert chosen["PATH_CHUNK_BLOCKS"] in (0, 4, 8, 16, 32, 64, 128)
        assert chosen["PATH_CTA_THREADS"] in (64, 128, 256)
        assert chosen["PATH_ORDER_WINDOW"] in (0, 4096, 16384)
        np.testing.assert_array_equal(ctx.x_GPU_2_host(), x)
        ctx.DROP_full_tx_iteration(1)
        ctx.DROP_full_tx_iteration(2)
        np.testing.assert_array_equal(ctx.x_GPU_2_host(), expected)
