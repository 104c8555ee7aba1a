"""Batches: several scans with different grids run as one graph per DROP iteration (GPU).

With SCATTER_MODE DETERMINISTIC each scan's image after batched iterations must equal, bit for
bit, the image of the same scan iterated on its own; with float atomics they agree at the DROP
tolerance.  A context that gets new histories makes the batch rebuild its graph.
"""
import numpy as np
import pytest

from pct_reconstruction_b200 import Batch, Config
from pct_reconstruction_b200 import phantoms as P

pytestmark = pytest.mark.gpu

SCANS = [
    # (grid parameters, phantom, tracks)
    (dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=6.4, SSD_V_SIZE=5.0,
          DROP_BLOCK_SIZE=3200, HISTORIES_PER_BLOCK=640, MLP_U_STEP=0.1), "water", 40000),
    (dict(VOXEL_WIDTH=0.2, VOXEL_HEIGHT=0.2, VOXEL_THICKNESS=0.5, RECON_CYL_RADIUS=6.4, SSD_V_SIZE=5.0,
          DROP_BLOCK_SIZE=5000, HISTORIES_PER_BLOCK=0), "ellipsoids", 30000),
    (dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=10.0, SSD_V_SIZE=9.0,
          DROP_BLOCK_SIZE=60000, HISTORIES_PER_BLOCK=480), "head", 60000),
]


def make_scan(i, params, kind, n):
    cfg = Config(**params)
    ph = {"water": P.water_cylinder_phantom(6.0), "head": P.head_phantom(),
          "ellipsoids": P.random_ellipsoid_phantom(i + 5, extent=(5.5, 5.5, 1.8))}[kind]
    tr = P.simulate_tracks(ph, n, seed=90 + i, continuous_angles=(kind != "water"),
                           t_extent=(20.0 if kind == "head" else 14.0), v_extent=(7.0 if kind == "head" else 3.5))
    hist = {k: v.numpy() for k, v in P.reconstruction_histories(cfg, tr).items()}
    x0 = (0.9 * P.truth_image(cfg, ph).numpy() + 0.1).astype(np.float32)
    return params, hist, x0


@pytest.fixture(scope="module")
def scans():
    return [make_scan(i, p, kind, n) for i, (p, kind, n) in enumerate(SCANS)]


def contexts(scans, mode):
    from pct_reconstruction_b200 import Context
    out = []
    for params, hist, x0 in scans:
        c = Context(Config(**dict(params, SCATTER_MODE=mode)))
        c.set_reconstruction_histories(hist)
        c.x_host_2_GPU(x0)
        out.append(c)
    return out


@pytest.mark.parametrize("mode", ["DETERMINISTIC", "ATOMIC"])
def test_batched_scans_equal_separate_runs(scans, mode):
    iters = 2
    sep = contexts(scans, mode)
    for c in sep:
        for it in range(iters):
            c.DROP_full_tx_iteration(it + 1)
    expect = [c.x_GPU_2_host() for c in sep]
    for c in sep:
        c.close()
    bat = contexts(scans, mode)
    with Batch(bat) as b:
        for it in range(iters):
            b.DROP_iteration(it + 1)
        b.synchronize()
        got = [c.x_GPU_2_host() for c in bat]
    for c in bat:
        c.close()
    for e, g, (params, hist, x0) in zip(expect, got, scans):
        assert (g != x0).sum() > 100
        if mode == "DETERMINISTIC":
            np.testing.assert_array_equal(g, e)
        else:
            np.testing.assert_allclose(g, e, rtol=1e-5, atol=1e-6)


def test_batch_rebuilds_after_new_histories(scans):
    ctxs = contexts(scans, "DETERMINISTIC")
    try:
        with Batch(ctxs) as b:
            b.DROP_iteration(1)
            b.synchronize()
            params, hist, x0 = scans[0]
            half = {k: v[: len(v) // 2] for k, v in hist.items()}
            ctxs[0].set_reconstruction_histories(half)  # new history count: its captured graph is released
            ctxs[0].x_host_2_GPU(x0)
            b.DROP_iteration(2)
            b.synchronize()
            got = ctxs[0].x_GPU_2_host()
        from pct_reconstruction_b200 import Context
        with Context(Config(**dict(params, SCATTER_MODE="DETERMINISTIC"))) as ref:
            ref.set_reconstruction_histories(half)
            ref.x_host_2_GPU(x0)
            ref.DROP_full_tx_iteration(1)
            np.testing.assert_array_equal(got, ref.x_GPU_2_host())
    finally:
        for c in ctxs:
            c.close()
