"""Parity against fixtures produced by the reference's own device code on a B200.

tests/golden/ref_*.npz were made by tests/golden/make_reference_fixtures.py, which runs the
reference's unmodified B.cu (compiled for sm_100a, oracle/build_reference.py) through
oracle/ref_harness.cu at the reference's built-in configuration (B.h defaults).  The CPU tests pin
the oracle; the GPU tests compare the engine through the C ABI.

Voxel lists: identical except for counted floating-point boundary ties (the oracle squares with
the correctly rounded product where the reference calls CUDA's powf; the reference's own build
also contracts multiply-adds into FMAs, which the engine's exact mode does not).
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import Oracle
from pct_reconstruction_b200 import Config

GOLDEN = Path(__file__).resolve().parent / "golden"
HIST = ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit", "xy_entry_angle", "xz_entry_angle",
        "xy_exit_angle", "xz_exit_angle", "WEPL", "first_MLP_voxel")
TIE_FRACTION = 2e-3


def load(name):
    p = GOLDEN / name
    if not p.exists():
        pytest.fail(f"missing fixture {p}: run tests/golden/make_reference_fixtures.py on a machine with a B200")
    return dict(np.load(p))


def default_image(nv):
    i = np.arange(nv, dtype=np.uint64)
    return (0.5 + ((i * np.uint64(2654435761)) % np.uint64(1000)).astype(np.float64) / 1000.0).astype(np.float32)


def csr_rows(counts, voxels):
    off = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
    return [voxels[off[i]:off[i + 1]] for i in range(len(counts))]


def count_list_ties(counts, rows, ref_counts, ref_rows):
    ties = 0
    for c, r, rc, rr in zip(counts, rows, ref_counts, ref_rows):
        if c != rc or not np.array_equal(r[:c], rr):
            ties += 1
    return ties


def drop_reference_image(f, nv):
    """x after the reference's DROP iteration: x_0 with the changed voxels (delta-coded indices)."""
    ref = default_image(nv)
    changed = np.cumsum(f["changed_delta"].astype(np.int64)) - 1
    ref[changed] = f["values"]
    return ref


def image_close(g, o, rel=1e-6, atol=1e-5):
    g64, o64 = g.astype(np.float64), o.astype(np.float64)
    r = float(np.sqrt(np.mean((g64 - o64) ** 2)) / np.sqrt(np.mean(o64 ** 2)))
    assert r < rel, r
    np.testing.assert_allclose(g, o, rtol=0, atol=atol)
    return r


# ---------------------------------------------------------------- oracle (CPU) ------------

def test_oracle_mlp_matches_reference_device_code():
    f = load("ref_mlp.npz")
    cfg = Config()
    hist = {k: f[k] for k in HIST}
    x0 = default_image(cfg.NUM_VOXELS)
    counts, vox, chord, adx, flags = Oracle(cfg.struct).mlp_paths(hist, x0)
    ref_rows = csr_rows(f["counts"], f["voxels"])
    rows = [vox[i, :counts[i]] for i in range(len(counts))]
    ties = count_list_ties(counts, rows, f["counts"], ref_rows)
    print(f"oracle vs reference MLP: {ties} tie histories of {len(counts)}")
    assert ties <= TIE_FRACTION * len(counts)
    np.testing.assert_allclose(chord, f["chord"], rtol=1e-6)
    same = np.array([c == rc and np.array_equal(r, rr) for c, r, rc, rr in zip(counts, rows, f["counts"], ref_rows)])
    np.testing.assert_allclose(adx[same], f["a_dot_x"][same], rtol=1e-13)


def test_oracle_drop_matches_reference_device_code():
    f = load("ref_drop.npz")
    cfg = Config(DROP_BLOCK_SIZE=int(f["drop_block_size"]))
    hist = {k: f[k] for k in HIST}
    x0 = default_image(cfg.NUM_VOXELS)
    ref = drop_reference_image(f, cfg.NUM_VOXELS)
    x1, _ = Oracle(cfg.struct).drop_iteration(hist, x0)
    r = image_close(x1, ref)
    print(f"oracle vs reference DROP: rel RMSE {r:.2e}")


# ---------------------------------------------------------------- engine (GPU) ------------

@pytest.mark.gpu
def test_engine_mlp_matches_reference_device_code():
    from pct_reconstruction_b200 import Context
    f = load("ref_mlp.npz")
    cfg = Config()
    hist = {k: f[k] for k in HIST}
    x0 = default_image(cfg.NUM_VOXELS)
    with Context(cfg) as ctx:
        ctx.set_reconstruction_histories(hist)
        ctx.x_host_2_GPU(x0)
        counts, vox, chord, adx = ctx.mlp_paths()
    ref_rows = csr_rows(f["counts"], f["voxels"])
    rows = [vox[i, :counts[i]] for i in range(len(counts))]
    ties = count_list_ties(counts, rows, f["counts"], ref_rows)
    print(f"engine vs reference MLP: {ties} tie histories of {len(counts)}")
    assert ties <= TIE_FRACTION * len(counts)
    np.testing.assert_allclose(chord, f["chord"], rtol=0, atol=0)  # same CUDA sinf/cosf, same operations


@pytest.mark.gpu
def test_engine_drop_matches_reference_device_code():
    from pct_reconstruction_b200 import Context
    f = load("ref_drop.npz")
    cfg = Config(DROP_BLOCK_SIZE=int(f["drop_block_size"]))
    hist = {k: f[k] for k in HIST}
    x0 = default_image(cfg.NUM_VOXELS)
    ref = drop_reference_image(f, cfg.NUM_VOXELS)
    with Context(cfg) as ctx:
        ctx.set_reconstruction_histories(hist)
        ctx.x_host_2_GPU(x0)
        ctx.DROP_full_tx_iteration(1)
        g = ctx.x_GPU_2_host()
    r = image_close(g, ref)
    print(f"engine vs reference DROP: rel RMSE {r:.2e}")
