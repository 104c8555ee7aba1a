"""Deterministic scatter (SCATTER_MODE = DETERMINISTIC).

The reference accumulates x_update with float atomics, so its image depends on the order in which
the additions land.  The deterministic mode accumulates each block's updates as 64-bit fixed-point
sums (scale 2^40): integer addition is associative, so repeated runs give bit-identical images.
Against the oracle's history-order float sums the images agree at the DROP tolerance.
"""
import numpy as np
import pytest

from oracle import Oracle
from pct_reconstruction_b200 import Config
from pct_reconstruction_b200 import phantoms as P
from pct_reconstruction_b200.engine import PCTError

IMAGE_REL_RMSE = 1e-6
IMAGE_ATOL = 1e-5


def test_config_rejects_deterministic_robustb():
    with pytest.raises(PCTError):
        Config(SCATTER_MODE="DETERMINISTIC", PROJECTION_ALGORITHM="ROBUSTB")
    assert Config(SCATTER_MODE="DETERMINISTIC").SCATTER_MODE == 1


@pytest.fixture(scope="module")
def scan(c1_params):
    cfg = Config(**c1_params)
    tr = P.simulate_tracks(P.water_cylinder_phantom(6.0), 40000, seed=81)
    hist = {k: v.numpy() for k, v in P.reconstruction_histories(cfg, tr).items()}
    x = (0.95 + 0.1 * np.random.default_rng(3).random(cfg.NUM_VOXELS)).astype(np.float32)
    return hist, x


def run(params, hist, x, iterations=2, reuse=False):
    from pct_reconstruction_b200 import Context
    with Context(Config(**params)) as ctx:
        ctx.set_reconstruction_histories(hist)
        ctx.x_host_2_GPU(x)
        ctx.set_path_reuse(reuse)
        for it in range(iterations):
            ctx.DROP_full_tx_iteration(it + 1)
        return ctx.x_GPU_2_host()


def close(g, o):
    rel = float(np.sqrt(np.mean((g.astype(np.float64) - o) ** 2)) / np.sqrt(np.mean(o.astype(np.float64) ** 2)))
    assert rel < IMAGE_REL_RMSE, rel
    np.testing.assert_allclose(g, o, rtol=0, atol=IMAGE_ATOL)


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ["DROP", "ROBUSTA"])
def test_deterministic_runs_are_bit_identical_and_match_oracle(c1_params, scan, algo):
    hist, x = scan
    p = dict(c1_params, SCATTER_MODE="DETERMINISTIC", PROJECTION_ALGORITHM=algo)
    a = run(p, hist, x)
    b = run(p, hist, x)
    c = run(p, hist, x, reuse=True)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(a, c)  # stored paths: the same sums, the same image
    o, _ = Oracle(Config(**p).struct).drop_iteration(hist, x, iterations=2)
    assert (o != x).sum() > 1000
    close(a, o)


@pytest.mark.gpu
def test_deterministic_needs_path_storage(c1_params, scan):
    from pct_reconstruction_b200 import Context
    hist, x = scan
    with Context(Config(**dict(c1_params, SCATTER_MODE="DETERMINISTIC"))) as ctx:
        ctx.set_reconstruction_histories(hist)
        ctx.set_path_storage_limit(-1)
        with pytest.raises(PCTError) as ei:
            ctx.DROP_full_tx_iteration(1)
        assert ei.value.status == 5


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ["DROP", "ROBUSTA"])
def test_captured_chain_matches_kernel_by_kernel(c1_params, scan, algo):
    """The captured iteration launches each DROP-block kernel and image update as a programmatic
    dependent of the kernel before it; the profiled iteration launches them one by one with
    events in between.  In deterministic mode both must give the same image bit for bit."""
    from pct_reconstruction_b200 import Context
    hist, x = scan
    p = dict(c1_params, SCATTER_MODE="DETERMINISTIC", PROJECTION_ALGORITHM=algo, PATH_CHUNK_BLOCKS=4)
    imgs = []
    for profiled in (False, True):
        with Context(Config(**p)) as ctx:
            ctx.set_reconstruction_histories(hist)
            ctx.x_host_2_GPU(x)
            for it in range(3):
                if profiled:
                    ctx.profile_drop_iteration()
                else:
                    ctx.DROP_full_tx_iteration(it + 1)
            imgs.append(ctx.x_GPU_2_host())
    assert (imgs[0] != x).sum() > 1000
    np.testing.assert_array_equal(imgs[0], imgs[1])
