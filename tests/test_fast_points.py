"""The exact mode's guarded fast MLP points (EXACT_FAST_POINTS = 1) against the reference's order.

oracle/pct_oracle_fastcheck.c restates the engine's fast evaluation of an MLP point (refined
reciprocals, fused multiply-adds, a first-order forward error bound; mlp_point_fast in
csrc/pct_mlp.cuh) next to the reference's operations in the reference's order
(find_MLP_path_GPU_tabulated, B.cu:9180-9235).  Over every point of every history: a point whose
voxel the bound proves must have the reference-order voxel (0 exceptions), and the bound must prove
nearly all points (the others are recomputed in the reference's order).  The GPU test compares the
engine's voxel lists with EXACT_FAST_POINTS = 1 and 0 directly.
"""
import numpy as np
import pytest

from oracle import Oracle
from pct_reconstruction_b200 import Config
from pct_reconstruction_b200 import phantoms as P

HEAD = dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=10.0, SSD_V_SIZE=9.0,
            DROP_BLOCK_SIZE=60000, HISTORIES_PER_BLOCK=480)
WATER = dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=6.4, SSD_V_SIZE=5.0,
             DROP_BLOCK_SIZE=3200, HISTORIES_PER_BLOCK=0, MLP_U_STEP=0.1)


def histories(params, phantom, n, seed, **kw):
    cfg = Config(**params)
    tr = P.simulate_tracks(phantom, int(n * 1.5), seed=seed, **kw)
    h = {k: v.numpy()[:n] for k, v in P.reconstruction_histories(cfg, tr).items()}
    return cfg, h


@pytest.mark.parametrize("case", ["head", "water", "builtin"])
def test_fast_points_never_disagree_with_reference_order(case):
    if case == "head":
        cfg, h = histories(HEAD, P.head_phantom(), 20000, 5, continuous_angles=True, t_extent=20.0, v_extent=7.0)
    elif case == "water":
        cfg, h = histories(WATER, P.water_cylinder_phantom(6.0), 20000, 6)
    else:
        cfg, h = histories({}, P.water_cylinder_phantom(7.0), 10000, 7, continuous_angles=True, t_extent=16.0,
                           v_extent=7.0)
    points, accepted, mismatched = Oracle(cfg.struct).fast_point_check(h)
    print(f"{case}: {points} MLP points, {accepted} proven by the bound ({accepted / points:.5%}), "
          f"{mismatched} proven points with a voxel other than the reference-order one")
    assert points > 1_000_000
    assert mismatched == 0
    assert accepted >= 0.99 * points


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["head", "water"])
def test_engine_fast_points_lists_equal_reference_order(case):
    import torch
    from pct_reconstruction_b200 import Context
    if case == "head":
        cfg, h = histories(HEAD, P.head_phantom(), 200000, 8, continuous_angles=True, t_extent=20.0, v_extent=7.0)
        params = HEAD
    else:
        cfg, h = histories(WATER, P.water_cylinder_phantom(6.0), 200000, 9)
        params = WATER
    n = len(h["WEPL"])
    outs = []
    for fast in (1, 0):
        with Context(Config(**params, EXACT_FAST_POINTS=fast)) as ctx:
            ctx.set_reconstruction_histories(h)
            ctx.x_host_2_GPU(np.ones(cfg.NUM_VOXELS, np.float32))
            cnt = torch.zeros(n, dtype=torch.int32, device="cuda")
            vox = torch.zeros(n * 512, dtype=torch.int32, device="cuda")
            adx = torch.zeros(n, dtype=torch.float64, device="cuda")
            ctx.mlp_paths_device(0, n, 512, cnt, vox, None, adx)
            torch.cuda.synchronize()
            outs.append((cnt.cpu().numpy(), vox.view(n, 512).cpu().numpy(), adx.cpu().numpy()))
    (c1, v1, a1), (c0, v0, a0) = outs
    assert c1.max() <= 512
    np.testing.assert_array_equal(c1, c0)
    np.testing.assert_array_equal(v1, v0)
    np.testing.assert_array_equal(a1, a0)


def test_voxel_guard_is_sound_and_rejects_faces():
    """The fast point's voxel guard (guarded_indices in csrc/pct_mlp.cuh, restated in the oracle) on
    positions of the head grid: an accepted position with error bound err gets the reference's index
    (int(|pos - zero| / size), calculate_voxel_GPU B.cu:11091), and so does every position within err
    of it; a position within err of a voxel face is rejected."""
    cfg = Config(**HEAD)
    o = Oracle(cfg.struct)
    zero = np.array([-cfg.RECON_CYL_RADIUS, cfg.RECON_CYL_RADIUS, cfg.RECON_CYL_HEIGHT / 2])
    size = np.array([cfg.VOXEL_WIDTH, cfg.VOXEL_HEIGHT, cfg.VOXEL_THICKNESS])
    extent = np.array([cfg.COLUMNS, cfg.ROWS, cfg.SLICES]) * size
    sign = np.array([1.0, -1.0, -1.0])  # x grows from X_ZERO, y and z fall from Y/Z_ZERO (B.h:846-921)
    rng = np.random.default_rng(11)

    def reference_index(pos):
        return (np.abs(pos - zero) / size).astype(np.int64)

    for err in (0.0, 1e-9, 1e-4, 1e-2):
        n = 60000
        pos = zero + sign * rng.uniform(0.0, 1.0, (n, 3)) * extent
        # a third of the positions at a voxel face of one axis, offset by a multiple of err
        near = np.arange(0, n, 3)
        axis = rng.integers(0, 3, len(near))
        k = rng.integers(1, 30, len(near))
        frac = rng.choice([0.0, 0.25, 0.5, 0.99, -0.25, -0.5, -0.99, 1.01, -1.01, 2.0, -2.0], len(near))
        pos[near, axis] = zero[axis] + sign[axis] * (k * size[axis] + frac * err)
        ok, idx = o.guarded_indices(pos[:, 0], pos[:, 1], pos[:, 2], err)
        ref = reference_index(pos)
        assert np.array_equal(idx[ok], ref[ok]), err
        for a in range(3):
            for s in (-1.0, 1.0):
                moved = pos[ok].copy()
                moved[:, a] += s * err
                assert np.array_equal(reference_index(moved), ref[ok]), (err, a, s)
        inside = np.zeros(n, bool)
        inside[near] = np.abs(frac) < 1.0
        assert not ok[inside].any(), err
        print(f"err {err:g} cm: {ok.mean():.4%} of positions proven; all {int(inside.sum())} within err of a face rejected")
