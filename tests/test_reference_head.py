"""Parity at the head-size grid against the reference's own device code.

The reference's parameters are compile-time macros, so oracle/build_reference.py also compiles its
unmodified B.cu against a copy of B.h with the head grid: 200 x 200 x 32 voxels of 0.1 x 0.1 x 0.25
cm (R = 10 cm), MLP_U_STEP = VOXEL_WIDTH / 2 = 0.05 cm, DROP blocks of 60000, HISTORIES_PER_BLOCK
480.  tests/golden/make_reference_fixtures.py ran that build on a B200:
  * ref_mlp_head.npz: find_MLP_path_GPU_tabulated (B.cu:9104-9262) on 2000 head-phantom histories
    (inputs stored): voxel lists, effective chord lengths, sums of x over the paths;
  * ref_drop_head.npz: one DROP iteration (calculate_x_update_GPU's MLP + DROP_block_update_GPU +
    image_update_GPU, B.cu:9321-9419) over 120000 histories in two blocks of 60000, from a fixed
    non-uniform image.  The inputs are regenerated from their seed on cuda:0 and checked against
    the stored SHA-256; the image is stored as every 7th voxel and the SHA-256 of all of it.
Voxel lists must be identical except for counted floating-point boundary ties; images within
1e-6 relative RMSE (float atomics: the reference's accumulation order is not fixed).
"""
from pathlib import Path
import sys

import numpy as np
import pytest

from oracle import Oracle
from pct_reconstruction_b200 import Config

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
from fixture_inputs import HEAD, HIST, default_image, head_histories, sha256_of  # noqa: E402

TIE_FRACTION = 2e-3
IMAGE_REL_RMSE = 1e-6


def load(name):
    p = GOLDEN / name
    if not p.exists():
        pytest.fail(f"missing fixture {p}: run tests/golden/make_reference_fixtures.py on a machine with a B200")
    return dict(np.load(p))


def reference_lists(f):
    voxels = np.cumsum(f["voxels_delta"].astype(np.int64)).astype(np.uint32)
    off = np.concatenate([[0], np.cumsum(f["counts"].astype(np.int64))])
    return [voxels[off[i]:off[i + 1]] for i in range(len(f["counts"]))]


def list_ties(counts, vox, f):
    """Histories whose voxel list differs from the reference's, with the first few listed."""
    ref = reference_lists(f)
    bad = [i for i in range(len(counts))
           if counts[i] != f["counts"][i] or not np.array_equal(vox[i, :counts[i]], ref[i])]
    for i in bad[:5]:
        c = int(min(counts[i], f["counts"][i]))
        k = int(np.argmax(vox[i, :c] != ref[i][:c])) if np.any(vox[i, :c] != ref[i][:c]) else c
        print(f"  history {i}: lengths {int(counts[i])} / {int(f['counts'][i])}, first difference at entry {k}")
    return bad


def test_oracle_mlp_matches_reference_head_grid():
    f = load("ref_mlp_head.npz")
    cfg = Config(**HEAD)
    hist = {k: f[k] for k in HIST}
    counts, vox, chord, adx, flags = Oracle(cfg.struct).mlp_paths(hist, default_image(cfg.NUM_VOXELS))
    bad = list_ties(counts, vox, f)
    print(f"oracle vs reference MLP (head grid): {len(bad)} tie histories of {len(counts)}, "
          f"{int(f['counts'].sum())} path entries")
    assert len(bad) <= TIE_FRACTION * len(counts)
    np.testing.assert_allclose(chord, f["chord"], rtol=1e-6)
    same = np.ones(len(counts), bool)
    same[bad] = False
    np.testing.assert_allclose(adx[same], f["a_dot_x"][same], rtol=1e-13)


@pytest.mark.gpu
def test_engine_mlp_matches_reference_head_grid():
    from pct_reconstruction_b200 import Context
    f = load("ref_mlp_head.npz")
    cfg = Config(**HEAD)
    hist = {k: f[k] for k in HIST}
    with Context(cfg) as ctx:
        ctx.set_reconstruction_histories(hist)
        ctx.x_host_2_GPU(default_image(cfg.NUM_VOXELS))
        counts, vox, chord, adx = ctx.mlp_paths()
        c = ctx.counters()
    bad = list_ties(counts, vox, f)
    print(f"engine vs reference MLP (head grid): {len(bad)} tie histories of {len(counts)}")
    assert len(bad) <= TIE_FRACTION * len(counts)
    np.testing.assert_allclose(chord, f["chord"], rtol=0, atol=0)  # same CUDA sinf/cosf, same operations
    same = np.ones(len(counts), bool)
    same[bad] = False
    np.testing.assert_allclose(adx[same], f["a_dot_x"][same], rtol=1e-13)
    assert c["voxel_oob"] == 0 and c["path_overflow"] == 0 and c["table_range"] == 0


@pytest.mark.gpu
def test_engine_drop_matches_reference_head_grid():
    import hashlib

    from pct_reconstruction_b200 import Context
    f = load("ref_drop_head.npz")
    cfg = Config(**HEAD)
    hist = head_histories(cfg, int(f["histories"]), seed=int(f["seed"]))
    if not np.array_equal(sha256_of(hist), f["inputs_sha256"]):
        pytest.fail("the fixture's inputs could not be regenerated bit for bit on this machine "
                    "(tests/golden/fixture_inputs.py head_histories); the comparison would be meaningless")
    x0 = default_image(cfg.NUM_VOXELS)
    with Context(cfg) as ctx:
        ctx.set_reconstruction_histories(hist)
        ctx.x_host_2_GPU(x0)
        ctx.DROP_full_tx_iteration(1)
        g = ctx.x_GPU_2_host()
    step = int(f["sample_step"])
    gs, ref = g[::step].astype(np.float64), f["out_x_sample"].astype(np.float64)
    rel = float(np.sqrt(np.mean((gs - ref) ** 2)) / np.sqrt(np.mean(ref ** 2)))
    identical = float(np.mean(g[::step] == f["out_x_sample"]))
    whole = hashlib.sha256(g.tobytes()).digest() == bytes(f["out_x_sha256"])
    print(f"engine vs reference DROP (head grid, 2 blocks of 60000): rel RMSE {rel:.2e} on every {step}th voxel, "
          f"{identical:.4f} of them bit-identical, whole image identical: {whole}; "
          f"voxels changed: engine {int((g != x0).sum())}, reference {int(f['changed'])}")
    assert rel < IMAGE_REL_RMSE
    np.testing.assert_allclose(g[::step], f["out_x_sample"], rtol=0, atol=1e-5)
