"""Pins the CPU oracle (CPU only).

The reference ships no tests or golden vectors, so the oracle is pinned by known answers derived
by hand from the reference's formulas (this file) and by fixtures produced by the reference's own
device functions on a B200 (tests/test_oracle_reference_fixtures.py).
"""
from fractions import Fraction

import numpy as np
import pytest

from oracle import Oracle
from pct_reconstruction_b200 import Config


def nearest_float32(fr: Fraction) -> float:
    """Correctly rounded float32 of an exact rational (ties to even)."""
    f = np.float32(float(fr))
    cands = [np.nextafter(f, np.float32(-np.inf)), f, np.nextafter(f, np.float32(np.inf))]
    best = min(cands, key=lambda c: (abs(Fraction(float(c)) - fr), int(np.array(c).view(np.uint32)) & 1))
    return float(best)


def test_a_coefficients_use_float_powers_of_ten(c1_params):
    # B.h:749-754: A_i = c_i * pow((float)10, (float)e_i) -> float-rounded power of ten.
    o = Oracle(Config(**c1_params).struct)
    expect = [c * nearest_float32(Fraction(1, 10 ** -e)) for c, e in
              ((7.457, -6), (4.548, -7), (-5.777, -8), (1.301, -8), (-9.228, -10), (2.687, -11))]
    assert o.a_coefficients() == expect


def test_chord_length_axis_aligned_is_voxel_width(c1_params):
    # EffectiveChordLength (B.cu:8873) at angles (0, 0): both factors are exactly 1.
    cfg = Config(**c1_params)
    o = Oracle(cfg.struct)
    assert o.effective_chord_length(0.0, 0.0) == cfg.VOXEL_WIDTH


def straight_history(cfg, x_in, x_out, y, z, xz=0.0):
    col = lambda x: int(abs(x + cfg.RECON_CYL_RADIUS) / cfg.VOXEL_WIDTH)
    row = int(abs(y - cfg.RECON_CYL_RADIUS) / cfg.VOXEL_HEIGHT)
    sl = int(abs(z - cfg.RECON_CYL_HEIGHT / 2) / cfg.VOXEL_THICKNESS)
    first = col(x_in) + row * cfg.COLUMNS + sl * cfg.COLUMNS * cfg.ROWS
    h = {k: np.array([v], np.float32) for k, v in dict(
        x_entry=x_in, y_entry=y, z_entry=z, x_exit=x_out, y_exit=y, z_exit=z,
        xy_entry_angle=0.0, xz_entry_angle=xz, xy_exit_angle=0.0, xz_exit_angle=xz, WEPL=0.0).items()}
    h["first_MLP_voxel"] = np.array([first], np.uint32)
    return h, row, sl


def test_zero_scatter_mlp_is_the_straight_row(c1_params):
    # A history along +x with t_in = t_out and zero angles: every MLP point has t_1 = t_in, so the
    # voxel list is the run of columns of one row.  u_2 = 6.125 cm at a 0.1 cm step gives 60 loop
    # iterations (depth 6.025 ... 0.125) at positions x_in + k*0.1 -> columns 34..93.
    cfg = Config(**c1_params)
    o = Oracle(cfg.struct)
    h, row, sl = straight_history(cfg, -3.05, 3.075, 0.55, 0.375)
    x = np.ones(cfg.NUM_VOXELS, np.float32)
    counts, vox, chord, adx, flags = o.mlp_paths(h, x)
    base = row * cfg.COLUMNS + sl * cfg.COLUMNS * cfg.ROWS
    expect = [base + c for c in range(33, 94)]
    assert counts[0] == 61
    assert list(vox[0, :61]) == expect
    assert chord[0] == cfg.VOXEL_WIDTH
    assert adx[0] == 61.0
    assert flags.tolist() == [0, 0, 0]


def test_drop_single_history_update(c1_params):
    # One history, uniform x = c: upd = L*((w - L*n*c)/(L^2*n))*lambda (rounded to float), added
    # once to each of the n distinct path voxels (B.cu:9356-9357, 9522-9536, 9398-9419).
    p = dict(c1_params, DROP_BLOCK_SIZE=1, HISTORIES_PER_BLOCK=0)
    cfg = Config(**p)
    o = Oracle(cfg.struct)
    h, row, sl = straight_history(cfg, -3.05, 3.075, 0.55, 0.375)
    c, n, L = 0.5, 61, cfg.VOXEL_WIDTH
    w = 7.0
    h["WEPL"][:] = w
    x = np.full(cfg.NUM_VOXELS, c, np.float32)
    x1, flags = o.drop_iteration(h, x)
    lam = float(np.float32(cfg.LAMBDA))
    aia = float(np.float32(L) * np.float32(L)) * n
    upd = np.float32(L * ((float(np.float32(w)) - (n * c) * L) / aia) * lam)
    changed = np.nonzero(x1 != x)[0]
    assert len(changed) == n
    np.testing.assert_array_equal(x1[changed], np.float32(c) + upd)


def test_drop_zero_residual_is_a_fixed_point(c1_params):
    # WEPL equal to L * sum(x) over the path leaves the image unchanged.
    p = dict(c1_params, DROP_BLOCK_SIZE=1, HISTORIES_PER_BLOCK=0)
    cfg = Config(**p)
    o = Oracle(cfg.struct)
    h, _, _ = straight_history(cfg, -3.05, 3.075, 0.55, 0.375)
    h["WEPL"][:] = np.float32(61 * 0.5 * cfg.VOXEL_WIDTH)
    x = np.full(cfg.NUM_VOXELS, 0.5, np.float32)
    x1, _ = o.drop_iteration(h, x)
    assert np.abs(x1 - x).max() < 1e-7


def test_histories_per_block_launch_arithmetic(c1_params):
    # calculate_x_update_GPU<<<floor(B/HPB), HPB>>> covers floor(B/HPB)*HPB histories of a block
    # (B.cu:9558): with B = 5 and HPB = 2 the 5th history of each block is skipped.
    p = dict(c1_params, DROP_BLOCK_SIZE=5, HISTORIES_PER_BLOCK=2)
    cfg = Config(**p)
    o = Oracle(cfg.struct)
    hs = [straight_history(cfg, -3.05, 3.075, 0.55 + 0.2 * k, 0.375)[0] for k in range(5)]
    h = {k: np.concatenate([d[k] for d in hs]) for k in hs[0]}
    h["WEPL"][:] = 9.0
    x = np.full(cfg.NUM_VOXELS, 0.5, np.float32)
    x1, _ = o.drop_iteration(h, x)
    rows_changed = {int(v) // cfg.COLUMNS % cfg.ROWS for v in np.nonzero(x1 != x)[0]}
    expect_rows = {int(abs(0.55 + 0.2 * k - cfg.RECON_CYL_RADIUS) / cfg.VOXEL_HEIGHT) for k in range(4)}
    assert rows_changed == expect_rows
