"""Total variation superiorization against the reference's own host code.

tests/golden/ref_tvs_head.npz (tests/golden/make_reference_fixtures.py, head-grid harness build)
holds what the reference's calculate_total_variation (B.cu:10163-10184) and
generate_perturbation_array (B.cu:10246-10307) return for two 200 x 200 x 32 images: the head
phantom's RSP (piecewise constant: most gradients are zero, which the direction skips) and a
hash-noise image (every gradient non-zero).  The reference's draw of L is seeded from the wall
clock (randi, B.cu:11478), so the deterministic parts are pinned: the oracle's reference-arithmetic
mode (float accumulation in the reference's loop order) against the fixture on the CPU, bit for
bit, and the engine's TV (the same float terms, accumulated in double) on the GPU.
"""
from pathlib import Path
import hashlib
import sys

import numpy as np
import pytest

from oracle import TVS_ENGINE, TVS_REFERENCE, TvsOracle
from pct_reconstruction_b200 import Config

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
from fixture_inputs import HEAD, default_image  # noqa: E402


def load():
    p = GOLDEN / "ref_tvs_head.npz"
    if not p.exists():
        pytest.fail(f"missing fixture {p}: run tests/golden/make_reference_fixtures.py on a machine with a B200")
    return dict(np.load(p))


def images(cfg):
    from pct_reconstruction_b200 import phantoms as P
    return {"phantom": P.truth_image(cfg, P.head_phantom()).numpy(), "hash": default_image(cfg.NUM_VOXELS)}


@pytest.mark.parametrize("name", ["phantom", "hash"])
def test_oracle_tv_and_direction_match_reference(name):
    f = load()
    cfg = Config(**HEAD)
    x = images(cfg)[name]
    assert hashlib.sha256(x.tobytes()).digest() == bytes(f[f"{name}_x_sha256"])
    o = TvsOracle(cfg.struct, TVS_REFERENCE)
    tv = o.total_variation(x)
    ref_tv = float(f[f"{name}_TV"][0])
    _, v, _ = o.direction(x)
    step = int(f["sample_step"])
    same = float(np.mean(v[::step] == f[f"{name}_v_sample"]))
    whole = hashlib.sha256(v.astype(np.float32).tobytes()).digest() == bytes(f[f"{name}_v_sha256"])
    print(f"{name}: TV oracle {tv!r} reference {ref_tv!r}; direction bit-identical on {same:.4%} of the sample, "
          f"whole direction identical: {whole}")
    # the same float operations in the same order: bit for bit
    assert np.float32(tv) == np.float32(ref_tv)
    np.testing.assert_array_equal(v[::step].astype(np.float32), f[f"{name}_v_sample"])
    assert whole


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["phantom", "hash"])
def test_engine_tv_matches_reference(name):
    from pct_reconstruction_b200 import Context
    f = load()
    cfg = Config(**HEAD)
    x = images(cfg)[name]
    with Context(cfg) as ctx:
        ctx.x_host_2_GPU(x)
        tv = ctx.total_variation()
    ref_tv = float(f[f"{name}_TV"][0])
    terms_in_double = TvsOracle(cfg.struct, TVS_ENGINE).total_variation(x)
    print(f"{name}: TV engine (double sums) {tv!r}; the reference's float terms summed in double "
          f"{terms_in_double!r}; the reference's own float accumulator {ref_tv!r}")
    # the engine adds the reference's float terms in double: equal to the same terms summed in
    # double in any order up to double rounding
    assert tv == pytest.approx(terms_in_double, rel=1e-12)
    # the reference adds 1.27M float terms into one float accumulator, whose rounding drifts by up
    # to ~1e-3 of the total on these images
    assert tv == pytest.approx(ref_tv, rel=2e-3)
