"""Statistics, cuts, sinogram, filter and backprojection against the reference's own device code.

Fixture tests/golden/ref_stats_fbp.npz (tests/golden/make_reference_fixtures.py) holds binned
history vectors and bin sums and what the reference's kernels made of them at its built-in
configuration (256x256x32, 560x36x120 bins): calculate_means_GPU, sum_squared_deviations_GPU +
calculate_standard_deviations_GPU, statistical_cuts_GPU, construct_sinogram_GPU, filter_GPU and
backprojection_GPU2 (B.cu:5608-6479).  Each stage is checked on the reference's own inputs to that
stage, so a difference is that stage's:
  * means, sinogram (per-bin divisions), filter and backprojection (one thread per output, fixed
    loop order) are deterministic in the reference and must match bit for bit on the GPU;
  * the standard deviations and sinogram sums accumulate with float atomics in the reference, so
    they match within the accumulation-order tolerance;
  * the cut survivors must match exactly (ties at the cut boundaries counted, none expected).
The CPU oracle is held to the same stages, with glibc math in the backprojection (last-bit
tolerance).
"""
import hashlib
from pathlib import Path

import numpy as np
import pytest

from oracle import GEOM, PreOracle
from pct_reconstruction_b200 import Config

F = np.load(Path(__file__).resolve().parent / "golden" / "ref_stats_fbp.npz")
NZ = F["bins_nonzero"]
SUM_RTOL = 2e-6  # float atomics in the reference vs a fixed order


def full(values, nb, dtype=np.float32):
    a = np.zeros(nb, dtype)
    a[NZ] = values
    return a


def geometry():
    n = len(F["in_WEPL"])
    g = {k: np.zeros(n, np.float32) for k in GEOM}
    for k in ("xy_entry_angle", "xz_entry_angle", "xy_exit_angle", "xz_exit_angle"):
        g[k] = F["in_" + k]
    return g


def ref_kept():
    return F["out_failed_cuts"] == 0


def test_oracle_statistics_and_cuts_match_reference():
    cfg = Config()
    nb = cfg.NUM_BINS
    keep, counts, means, sds, sino = PreOracle(cfg.struct).statistics_and_cuts(
        F["in_bin_num"], F["in_WEPL"], geometry(), full(F["in_bin_counts"], nb, np.int32),
        [full(F["in_sum_WEPL"], nb), full(F["in_sum_ut"], nb), full(F["in_sum_uv"], nb)])
    for k, m in zip(("mean_WEPL", "mean_rel_ut_angle", "mean_rel_uv_angle"), means):
        np.testing.assert_array_equal(m[NZ], F["out_" + k], err_msg=k)
    for k, s in zip(("stddev_WEPL", "stddev_rel_ut_angle", "stddev_rel_uv_angle"), sds):
        np.testing.assert_allclose(s[NZ], F["out_" + k], rtol=SUM_RTOL, atol=1e-9, err_msg=k)
    ties = int(np.sum(keep.astype(bool) != ref_kept()))
    print(f"oracle vs reference cut survivors: {ties} differ of {len(keep)}")
    assert ties <= 1e-3 * len(keep)
    np.testing.assert_array_equal(counts[NZ], F["out_bin_counts"])
    np.testing.assert_allclose(sino[NZ], F["out_sinogram_sums"], rtol=SUM_RTOL, atol=1e-5)


def test_oracle_filter_and_backprojection_match_reference():
    cfg = Config()
    o = PreOracle(cfg.struct)
    nb = cfg.NUM_BINS
    sino, filt = o.sinogram_filter(full(F["out_bin_counts"], nb, np.int32), full(F["out_sinogram_sums"], nb))
    np.testing.assert_array_equal(sino[NZ], F["out_sinogram"])
    np.testing.assert_allclose(filt[F["filtered_nonzero"]], F["out_sinogram_filtered"], rtol=1e-6, atol=1e-9)
    ref_filt = np.zeros(nb, np.float32)
    ref_filt[F["filtered_nonzero"]] = F["out_sinogram_filtered"]
    fbp = o.backprojection(ref_filt)
    sample = fbp[::int(F["FBP_sample_step"])]
    np.testing.assert_allclose(sample, F["out_FBP_sample"], rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
def test_engine_statistics_and_cuts_match_reference():
    from pct_reconstruction_b200 import Context
    cfg = Config()
    nb = cfg.NUM_BINS
    g = geometry()
    n = len(F["in_WEPL"])
    with Context(cfg) as ctx:
        ctx.set_history_vectors({**g, "WEPL": F["in_WEPL"]})
        ctx.set_array("bin_num_vector", F["in_bin_num"])
        ctx.set_array("bin_counts", full(F["in_bin_counts"], nb, np.int32))
        ctx.set_array("mean_WEPL", full(F["in_sum_WEPL"], nb))
        ctx.set_array("mean_rel_ut_angle", full(F["in_sum_ut"], nb))
        ctx.set_array("mean_rel_uv_angle", full(F["in_sum_uv"], nb))
        ctx.stage("calculate_means")
        for k in ("mean_WEPL", "mean_rel_ut_angle", "mean_rel_uv_angle"):
            np.testing.assert_array_equal(ctx.get_array(k)[NZ], F["out_" + k], err_msg=k)
        ctx.stage("sum_squared_deviations")
        ctx.stage("calculate_standard_deviations")
        for k in ("stddev_WEPL", "stddev_rel_ut_angle", "stddev_rel_uv_angle"):
            np.testing.assert_allclose(ctx.get_array(k)[NZ], F["out_" + k], rtol=SUM_RTOL, atol=1e-9, err_msg=k)
            ctx.set_array(k, full(F["out_" + k], nb))  # the cuts below see the reference's own deviations
        assert not ctx.get_array("bin_counts").any()  # calculate_standard_deviations_GPU clears the counts
        ctx.stage("statistical_cuts")
        kept_wepl = ctx.get_array("WEPL_vector")
        np.testing.assert_array_equal(ctx.get_array("bin_counts")[NZ], F["out_bin_counts"])
        np.testing.assert_allclose(ctx.get_array("sinogram")[NZ], F["out_sinogram_sums"], rtol=SUM_RTOL, atol=1e-5)
    np.testing.assert_array_equal(kept_wepl, F["in_WEPL"][ref_kept()])  # same survivors, in order
    assert len(kept_wepl) < n


@pytest.mark.gpu
def test_engine_sinogram_filter_backprojection_bit_identical():
    from pct_reconstruction_b200 import Context
    cfg = Config()
    nb = cfg.NUM_BINS
    with Context(cfg) as ctx:
        ctx.set_array("bin_counts", full(F["out_bin_counts"], nb, np.int32))
        ctx.set_array("sinogram", full(F["out_sinogram_sums"], nb))
        ctx.stage("construct_sinogram")
        np.testing.assert_array_equal(ctx.get_array("sinogram")[NZ], F["out_sinogram"])
        ctx.stage("FBP")
        filt = ctx.get_array("sinogram_filtered")
        fbp = ctx.get_array("FBP_image")
    nzf = np.nonzero(filt)[0]
    np.testing.assert_array_equal(nzf, F["filtered_nonzero"])
    np.testing.assert_array_equal(filt[nzf], F["out_sinogram_filtered"])
    np.testing.assert_array_equal(fbp[::int(F["FBP_sample_step"])], F["out_FBP_sample"])
    assert hashlib.sha256(fbp.tobytes()).digest() == F["out_FBP_sha256"].tobytes()


# ---------------------------------------------------------------- FBP hull, median, edges --

E = np.load(Path(__file__).resolve().parent / "golden" / "ref_edges.npz")


def edge_counts():
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    from make_reference_fixtures import edge_counts as make
    cfg = Config()
    c = make(cfg.COLUMNS, cfg.ROWS, cfg.SLICES)
    assert hashlib.sha256(c.tobytes()).digest() == E["counts_sha256"].tobytes()
    return c


def unpack(bits, n):
    return np.unpackbits(bits)[:n]


def expected_msc(cfg, counts):
    """The reference runs MSC_edge_detection_GPU(MSC_counts) in place (B.cu:6911): a voxel is 0 when
    its 3x3 max difference or its own count exceeds MSC_DIFF_THRESH, or outside the ring.  In place,
    a block can read neighbours another block already overwrote, so the fixture runs the
    out-of-place variant MSC_edge_detection_GPU(counts, output) (B.cu:6958), whose condition lacks
    the own-count term; adding that term gives the race-free in-place result."""
    return unpack(E["out_MSC_hull"], cfg.NUM_VOXELS) & (counts <= cfg.MSC_DIFF_THRESH).astype(np.uint8)


def test_oracle_edge_detection_matches_reference():
    cfg = Config()
    counts = edge_counts()
    o = PreOracle(cfg.struct)
    np.testing.assert_array_equal(o.edge_detection(1, counts.copy()).astype(np.uint8), expected_msc(cfg, counts))
    np.testing.assert_array_equal(o.edge_detection(2, counts.copy()).astype(np.uint8),
                                  unpack(E["out_SM_hull"], cfg.NUM_VOXELS))


@pytest.mark.gpu
def test_engine_fbp_median_and_hull_bit_identical():
    from pct_reconstruction_b200 import Context
    cfg = Config(ENDPOINTS_HULL="FBP_HULL")
    nb, nv = cfg.NUM_BINS, cfg.NUM_VOXELS
    with Context(cfg) as ctx:
        ctx.set_array("bin_counts", full(F["out_bin_counts"], nb, np.int32))
        ctx.set_array("sinogram", full(F["out_sinogram_sums"], nb))
        ctx.stage("construct_sinogram")
        ctx.stage("FBP")
        med = ctx.get_array("FBP_median_filtered")
        hull = ctx.get_array("FBP_hull")
    np.testing.assert_array_equal(med[::int(F["FBP_sample_step"])], F["out_FBP_median_sample"])
    assert hashlib.sha256(med.tobytes()).digest() == F["out_FBP_median_sha256"].tobytes()
    np.testing.assert_array_equal(hull, unpack(F["out_FBP_hull"], nv))


@pytest.mark.gpu
def test_engine_edge_detection_bit_identical():
    from pct_reconstruction_b200 import Context
    cfg = Config(MSC_ON=1, SM_ON=1)
    nv = cfg.NUM_VOXELS
    counts = edge_counts()
    with Context(cfg) as ctx:
        ctx.set_array("MSC_counts", counts)
        ctx.set_array("SM_counts", counts)
        ctx.stage("hull_detection_finish")
        msc, sm = ctx.get_array("MSC_counts"), ctx.get_array("SM_counts")
    np.testing.assert_array_equal(msc.astype(np.uint8), expected_msc(cfg, counts))
    np.testing.assert_array_equal(sm.astype(np.uint8), unpack(E["out_SM_hull"], nv))
