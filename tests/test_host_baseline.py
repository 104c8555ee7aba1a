"""The reference's host MLP + DROP restated in the oracle (the timed CPU baseline), on the CPU.

oracle_host_drop_iteration follows O.cu: calculate_MLP (O.cu:4017-4211, the explicit FP64 MLP with
pow/log per step, no lookup tables), the chord length from atanf of the chord slopes
(O.cu:6634-6636) through the float overload of EffectiveChordLength (O.cu:3745-3767), and
DROP_blocks / DROP_update (O.cu:7680-7711) with double accumulators.  It is the reference arm of
the throughput comparison, so it is pinned here:
  * its chord function against the tabulated path's chord (pinned bit-exactly against the
    reference's device code elsewhere) where both formulas apply, and at the known answer
    (0, 0) -> VOXEL_WIDTH;
  * its MLP voxel lists against the tabulated MLP's (the tables quantise u_2 to 5e-5 cm, so a
    few lists differ at voxel-boundary ties);
  * one history's DROP update against the O.cu formula worked by hand;
  * thread-count independence of the OpenMP port.
The host code is not the parity oracle: O.cu passes atanf angles in (-pi/2, pi/2) to a chord
formula written for angles in [0, pi/2), so its chord (and update) differs from the device
path's for histories with a negative slope.  test_host_chord_sign_quirk records that.
"""
import numpy as np
import pytest

from oracle import Oracle
from pct_reconstruction_b200 import Config
from pct_reconstruction_b200 import phantoms as P

C1 = dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=6.4, SSD_V_SIZE=5.0,
          DROP_BLOCK_SIZE=3200, HISTORIES_PER_BLOCK=0, MLP_U_STEP=0.1)


@pytest.fixture(scope="module")
def c1_histories():
    cfg = Config(**C1)
    tr = P.simulate_tracks(P.water_cylinder_phantom(6.0), 6000, seed=41)
    return cfg, {k: v.numpy() for k, v in P.reconstruction_histories(cfg, tr).items()}


def test_host_chord_matches_device_chord_formula():
    o = Oracle(Config(**C1).struct)
    assert o.host_effective_chord_length(0.0, 0.0) == np.float32(0.1)
    for t in (0.05, 0.2, 0.7, 1.2, 1.5):
        for v in (0.0, 0.1, 0.3):
            h, d = o.host_effective_chord_length(t, v), o.effective_chord_length(t, v)
            assert abs(h - d) <= 4e-7 * d, (t, v, h, d)


def test_host_chord_sign_quirk():
    # eff_angle_t = a - int(a / (pi/2)) * (pi/2) keeps a negative atanf angle negative
    # (O.cu:3751), so the host chord of a line with slope -s is not that of slope +s
    o = Oracle(Config(**C1).struct)
    assert o.host_effective_chord_length(-0.3, 0.0) != o.host_effective_chord_length(0.3, 0.0)


def test_host_mlp_lists_match_tabulated_mlp(c1_histories):
    cfg, h = c1_histories
    o = Oracle(cfg.struct)
    hc, hv, _ = o.host_mlp_paths(h)
    tc, tv, _, _, _ = o.mlp_paths(h, np.ones(cfg.NUM_VOXELS, np.float32))
    same = np.array([hc[i] == tc[i] and np.array_equal(hv[i, :hc[i]], tv[i, :tc[i]]) for i in range(len(hc))])
    print(f"host vs tabulated MLP: {int((~same).sum())} of {len(hc)} lists differ (table quantisation ties), "
          f"length difference at most {int(np.abs(hc.astype(int) - tc.astype(int)).max())}")
    assert same.mean() > 0.99
    assert np.abs(hc.astype(int) - tc.astype(int)).max() <= 2


def test_host_drop_single_history_known_answer():
    # One history along +x (zero angles, zero slopes): atanf(0) = 0, so L = (float)VOXEL_WIDTH; the
    # path is a run of columns of one row; with x = c everywhere, DROP_blocks gives
    # upd = L * lambda * (w - L * m * c) / (L^2 * m) and DROP_update adds (float)upd once per voxel.
    cfg = Config(**dict(C1, DROP_BLOCK_SIZE=1))
    o = Oracle(cfg.struct)
    row = int(abs(0.55 - cfg.RECON_CYL_RADIUS) / cfg.VOXEL_HEIGHT)
    sl = int(abs(0.375 - cfg.RECON_CYL_HEIGHT / 2) / cfg.VOXEL_THICKNESS)
    col_in = int(abs(-3.05 + cfg.RECON_CYL_RADIUS) / cfg.VOXEL_WIDTH)
    h = {k: np.array([v], np.float32) for k, v in dict(
        x_entry=-3.05, y_entry=0.55, z_entry=0.375, x_exit=3.075, y_exit=0.55, z_exit=0.375, xy_entry_angle=0.0,
        xz_entry_angle=0.0, xy_exit_angle=0.0, xz_exit_angle=0.0, WEPL=7.0).items()}
    h["first_MLP_voxel"] = np.array([col_in + row * cfg.COLUMNS + sl * cfg.COLUMNS * cfg.ROWS], np.uint32)
    c = np.float32(0.5)
    x = np.full(cfg.NUM_VOXELS, c, np.float32)
    x1, visited = o.host_drop_iteration(h, x)
    changed = np.nonzero(x1 != x)[0]
    m = len(changed)
    assert visited == m and 55 <= m <= 62
    assert np.all(changed // cfg.COLUMNS % cfg.ROWS == row) and np.all(changed // (cfg.COLUMNS * cfg.ROWS) == sl)
    cols = changed % cfg.COLUMNS
    assert cols[0] == col_in and np.array_equal(cols, np.arange(col_in, col_in + m))
    L = float(np.float32(cfg.VOXEL_WIDTH))
    lam = float(np.float32(cfg.LAMBDA))
    upd = L * lam * ((float(np.float32(7.0)) - L * (m * float(c))) / (L ** 2 * m))
    np.testing.assert_array_equal(x1[changed], np.float32(c) + np.float32(upd))


def test_host_drop_independent_of_thread_count(c1_histories):
    cfg, h = c1_histories
    o = Oracle(cfg.struct)
    x0 = (0.9 * P.truth_image(cfg, P.water_cylinder_phantom(6.0)) + 0.1).numpy()
    x1, v1 = o.host_drop_iteration(h, x0, threads=1)
    x8, v8 = o.host_drop_iteration(h, x0, threads=8)
    assert v1 == v8
    # double accumulators: the order of the atomic additions changes the sums only in the last bits
    np.testing.assert_allclose(x8, x1, rtol=0, atol=1e-7)


@pytest.mark.parametrize("params", [
    {},
    dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=10.0, SSD_V_SIZE=9.0,
         T_BIN_SIZE=0.1, V_BIN_SIZE=0.25, ANGULAR_BIN_SIZE=4.0, DROP_BLOCK_SIZE=60000, HISTORIES_PER_BLOCK=480,
         ITERATIONS=12, LAMBDA=0.0001),
    dict(C1, ITERATIONS=6, LAMBDA=0.0001),
    dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, RECON_CYL_RADIUS=6.45, SSD_V_SIZE=4.75),
])
def test_oracle_configuration_matches_engine_configuration(params):
    # the CPU baseline derives its configuration without the engine library (oracle/refconfig.py);
    # every field the oracle reads must equal the engine's derivation of the same parameters
    from oracle.refconfig import reference_config
    r, e = reference_config(**params), Config(**params)
    for k in ("COLUMNS", "ROWS", "SLICES", "NUM_VOXELS", "VOXEL_WIDTH", "VOXEL_HEIGHT", "VOXEL_THICKNESS",
              "RECON_CYL_RADIUS", "RECON_CYL_HEIGHT", "MLP_U_STEP", "MIN_MLP_LENGTH", "LAMBDA", "DROP_BLOCK_SIZE",
              "HISTORIES_PER_BLOCK", "PROJECTION_ALGORITHM", "PSI_SIGN", "ETA", "IDENTIFY_X_N_AIR",
              "X_N_AIR_THRESHOLD"):
        assert getattr(r, k) == getattr(e, k), k
