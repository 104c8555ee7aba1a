"""Edge cases of the DROP stage, engine against the oracle through the C ABI (needs a GPU).

* no reconstruction histories: an iteration is refused (PCT_ERR_STATE) and the image is untouched;
* a single history, and histories whose MLP list is shorter than MIN_MLP_LENGTH (no update);
* a DROP block larger than the scan (one partial block), and a ragged last block, both with
  HISTORIES_PER_BLOCK 0 (every history) and with the reference's launch arithmetic (640);
each at the DROP tolerance of the main parity tests.
"""
import numpy as np
import pytest

from oracle import Oracle
from pct_reconstruction_b200 import Config, PCTError
from pct_reconstruction_b200 import phantoms as P

pytestmark = pytest.mark.gpu

IMAGE_REL_RMSE = 1e-6
IMAGE_ATOL = 1e-5


def scan(cfg, n, seed):
    tr = P.simulate_tracks(P.water_cylinder_phantom(6.0), n, seed=seed)
    return {k: v.numpy() for k, v in P.reconstruction_histories(cfg, tr).items()}


def take(hist, idx):
    return {k: np.ascontiguousarray(v[idx]) for k, v in hist.items()}


def engine_iteration(cfg, hist, x):
    from pct_reconstruction_b200 import Context
    with Context(cfg) as ctx:
        ctx.set_reconstruction_histories(hist)
        ctx.x_host_2_GPU(x)
        ctx.DROP_full_tx_iteration(1)
        return ctx.x_GPU_2_host()


def check(cfg, hist, x):
    g = engine_iteration(cfg, hist, x)
    o, _ = Oracle(cfg.struct).drop_iteration(hist, x)
    d = g.astype(np.float64) - o
    rms = float(np.sqrt(np.mean(d ** 2)) / np.sqrt(np.mean(o.astype(np.float64) ** 2)))
    assert rms < IMAGE_REL_RMSE
    np.testing.assert_allclose(g, o, rtol=0, atol=IMAGE_ATOL)
    return g


@pytest.fixture(scope="module")
def base(c1_params):
    cfg = Config(**dict(c1_params, HISTORIES_PER_BLOCK=0))
    hist = scan(cfg, 8000, seed=61)
    x = (0.9 + 0.2 * np.random.default_rng(8).random(cfg.NUM_VOXELS)).astype(np.float32)
    return cfg, hist, x


def test_no_histories_is_refused_and_keeps_the_image(base):
    from pct_reconstruction_b200 import Context
    cfg, hist, x = base
    with Context(cfg) as ctx:
        ctx.set_reconstruction_histories(take(hist, slice(0, 0)))
        ctx.x_host_2_GPU(x)
        with pytest.raises(PCTError):
            ctx.DROP_full_tx_iteration(1)
        np.testing.assert_array_equal(ctx.x_GPU_2_host(), x)


def test_single_history(base):
    cfg, hist, x = base
    counts = Oracle(cfg.struct).mlp_paths(take(hist, slice(0, 200)), x)[0]
    i = int(np.argmax(counts))  # a history long enough (>= MIN_MLP_LENGTH) to update the image
    assert counts[i] >= cfg.MIN_MLP_LENGTH
    g = check(cfg, take(hist, slice(i, i + 1)), x)
    assert np.count_nonzero(g != x) > 0


def test_paths_shorter_than_min_mlp_length_do_not_update(base, c1_params):
    _, hist, x = base
    cfg = Config(**dict(c1_params, HISTORIES_PER_BLOCK=0, MIN_MLP_LENGTH=100000))
    g = engine_iteration(cfg, take(hist, slice(0, 500)), x)
    np.testing.assert_array_equal(g, x)


@pytest.mark.parametrize("block,hpb", [(20000, 0), (20000, 640), (3000, 0), (3000, 640)])
def test_partial_and_ragged_blocks(base, c1_params, block, hpb):
    _, hist, x = base
    cfg = Config(**dict(c1_params, DROP_BLOCK_SIZE=block, HISTORIES_PER_BLOCK=hpb))
    n = len(hist["WEPL"])
    assert n < 20000 and n % 3000 != 0  # one partial block, or a ragged last block
    check(cfg, hist, x)
