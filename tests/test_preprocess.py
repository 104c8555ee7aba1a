"""Preprocessing stages: tracker data -> reconstruction histories and the initial image.

CPU tests pin the oracle (oracle/pct_oracle_pre.c) against the reference-device fixtures
(intersections, binning, MLP endpoints) and against hand-checkable properties; GPU tests compare
the engine through the C ABI with the fixtures and with the oracle on the same inputs.

Integer results (missed flags, bin numbers, survivors, hull voxels, first MLP voxels) must agree
except at floating-point boundary ties, which are counted: the CPU oracle's glibc float
functions (atan2f, tanf, powf) can differ from CUDA's in the last bit.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import GEOM, TRACKER, PreOracle
from pct_reconstruction_b200 import Config
from pct_reconstruction_b200 import phantoms as P

GOLDEN = Path(__file__).resolve().parent / "golden"
TIE_FRACTION = 2e-3


def load(name):
    return dict(np.load(GOLDEN / name))


def survivor_keys(geom, wepl):
    """One hashable key per history (bit patterns of entry x/y, entry angle and WEPL)."""
    cols = [np.asarray(geom[k], np.float32).view(np.uint32) for k in ("x_entry", "y_entry", "xy_entry_angle")]
    cols.append(np.asarray(wepl, np.float32).view(np.uint32))
    return set(zip(*[c.tolist() for c in cols]))


def mismatch_fraction(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.mean(a != b)) if a.size else 0.0


# ---------------------------------------------------------------- oracle vs reference -----

def test_oracle_intersections_and_binning_match_reference():
    f = load("ref_intersections_binning.npz")
    cfg = Config()
    o = PreOracle(cfg.struct)
    geom, missed = o.intersections({k: f[k] for k in TRACKER}, f["gantry_angle"].astype(np.float32), True)
    ref_missed = f["missed_recon_volume"]
    assert mismatch_fraction(missed, ref_missed) <= TIE_FRACTION
    hit = (missed == 0) & (ref_missed == 0)
    assert hit.sum() > 1000
    for k in GEOM:
        np.testing.assert_allclose(geom[k][hit], f["out_" + k][hit], rtol=2e-6, atol=2e-6)
    bin_num, counts, sums = o.binning({k: f["out_" + k] for k in GEOM}, f["WEPL"], ref_missed)
    ties = int((bin_num != f["bin_num"]).sum())
    print(f"oracle vs reference bins: {ties} tie histories of {len(bin_num)}")
    assert ties <= TIE_FRACTION * len(bin_num)
    nz = f["bins_nonzero"]
    assert mismatch_fraction(counts[nz], f["bin_counts_nonzero"]) <= TIE_FRACTION
    assert counts.sum() == f["bin_counts_nonzero"].sum() or ties > 0


def test_oracle_endpoints_match_reference():
    f = load("ref_endpoints.npz")
    cfg = Config()
    hull = P.hull_image(cfg, P.water_cylinder_phantom(float(f["hull_radius"]))).numpy().astype(np.uint8)
    geom, fv = PreOracle(cfg.struct).collect_endpoints(hull, {k: f[k] for k in GEOM})
    ties = int((fv != f["out_first_MLP_voxel"]).sum())
    print(f"oracle vs reference endpoints: {ties} tie histories of {len(fv)}")
    assert ties <= TIE_FRACTION * len(fv)
    same = fv == f["out_first_MLP_voxel"]
    for k in ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit"):
        np.testing.assert_allclose(geom[k][same], f["out_" + k][same], rtol=1e-6, atol=1e-6)


# ---------------------------------------------------------------- oracle properties -------

def test_oracle_median_filter_matches_numpy():
    cfg = Config(COLUMNS=20, ROWS=18, SLICES=3, VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, RECON_CYL_RADIUS=1.0)
    rng = np.random.default_rng(1)
    img = rng.random(cfg.NUM_VOXELS).astype(np.float32)
    out = PreOracle(cfg.struct).median_filter(img, 2)
    vol = img.reshape(cfg.SLICES, cfg.ROWS, cfg.COLUMNS)
    ref = np.zeros_like(vol)
    for s in range(cfg.SLICES):
        for r in range(2, cfg.ROWS - 2):
            for c in range(2, cfg.COLUMNS - 2):
                ref[s, r, c] = np.sort(vol[s, r - 2:r + 3, c - 2:c + 3].ravel())[12]
    np.testing.assert_array_equal(out, ref.ravel())


def test_oracle_hull_walk_carves_straight_row():
    # One SC history along +x through a grid: every voxel of its row between the entry and exit
    # voxels (exclusive of the exit voxel) is carved.
    cfg = Config(COLUMNS=40, ROWS=40, SLICES=4, VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25,
                 RECON_CYL_RADIUS=2.0, SSD_V_SIZE=2.0, SC_LOWER_THRESHOLD=-1.0, SC_UPPER_THRESHOLD=1.0)
    o = PreOracle(cfg.struct)
    hull = o.initialize_hull()
    geom = {k: np.zeros(1, np.float32) for k in GEOM}
    geom["x_entry"][:] = -1.55
    geom["x_exit"][:] = 1.55
    geom["y_entry"][:] = geom["y_exit"][:] = 0.05
    geom["z_entry"][:] = geom["z_exit"][:] = 0.1
    carved, bounded = o.hull_walks(0, geom, np.zeros(1, np.float32), np.zeros(1, np.uint8), hull)
    assert bounded == 0
    row = int(abs(0.05 - 2.0) / 0.1)
    sl = int(abs(0.1 - 0.5) / 0.25)
    changed = np.nonzero(carved != hull)[0]
    cols = sorted(int(v) % 40 for v in changed)
    assert all(int(v) // 40 % 40 == row and int(v) // 1600 == sl for v in changed)
    assert cols == list(range(int((-1.55 + 2.0) / 0.1), int((1.55 + 2.0) / 0.1)))


# ---------------------------------------------------------------- engine (GPU) -------------

@pytest.mark.gpu
def test_engine_intersections_binning_match_reference():
    from pct_reconstruction_b200 import Context
    f = load("ref_intersections_binning.npz")
    cfg = Config()
    tracker = {k: f[k] for k in TRACKER}
    tracker["WEPL"] = f["WEPL"]
    tracker["gantry_angle"] = f["gantry_angle"].astype(np.float32)
    with Context(cfg) as ctx:
        ctx.load_tracker_data(tracker, integer_angles=True)
        ctx.stage("recon_volume_intersections")
        missed = ctx.get_array("missed_recon_volume")
        geom = {k: ctx.get_array(k) for k in GEOM}
        ctx.stage("binning")
        bin_num = ctx.get_array("bin_num")
        counts = ctx.get_array("bin_counts")
        n_vec = len(ctx.get_array("WEPL_vector"))
    ties = int((missed != f["missed_recon_volume"]).sum())
    print(f"engine vs reference missed flags: {ties} ties of {len(missed)}")
    assert ties <= TIE_FRACTION * len(missed)
    hit = (missed == 0) & (f["missed_recon_volume"] == 0)
    exact = np.ones(len(missed), bool)
    for k in GEOM:
        exact &= geom[k] == f["out_" + k]
        np.testing.assert_allclose(geom[k][hit], f["out_" + k][hit], rtol=2e-6, atol=2e-6)
    print(f"engine vs reference intersections: {int(exact[hit].sum())} of {int(hit.sum())} bit-identical")
    assert exact[hit].mean() > 0.99
    # missed histories get bin numbers from the reference's uninitialised intercepts (B.cu:4944-4950
    # leave u_entry/t_entry unset when the line misses the cylinder); only hits are comparable
    bties = int((bin_num[hit] != f["bin_num"][hit]).sum())
    print(f"engine vs reference bins: {bties} ties of {int(hit.sum())} hits")
    assert bties <= TIE_FRACTION * hit.sum()
    nz = f["bins_nonzero"]
    assert mismatch_fraction(counts[nz], f["bin_counts_nonzero"]) <= TIE_FRACTION
    assert n_vec == int((missed == 0).sum())


@pytest.mark.gpu
def test_engine_endpoints_match_reference():
    from pct_reconstruction_b200 import Context
    f = load("ref_endpoints.npz")
    cfg = Config()
    hull = P.hull_image(cfg, P.water_cylinder_phantom(float(f["hull_radius"]))).numpy().astype(np.uint8)
    hist = {k: f[k] for k in GEOM}
    hist["WEPL"] = f["WEPL"]
    with Context(cfg) as ctx:
        ctx.set_history_vectors(hist)
        ctx.set_array("hull", hull)
        ctx.stage("reconstruction_cuts")
        n = ctx.reconstruction_histories
        fv_kept = ctx.get_array("first_MLP_voxel_vector")
        kept = {k: ctx.get_array(k + "_vector") for k in ("x_entry", "y_exit")}
    ref_fv = f["out_first_MLP_voxel"]
    ref_keep = ref_fv != cfg.NUM_VOXELS
    print(f"engine vs reference endpoints: {n} kept, reference {int(ref_keep.sum())}")
    assert abs(n - int(ref_keep.sum())) <= TIE_FRACTION * len(ref_fv)
    if n == int(ref_keep.sum()):
        assert mismatch_fraction(fv_kept, ref_fv[ref_keep]) <= TIE_FRACTION
        np.testing.assert_allclose(kept["x_entry"], f["out_x_entry"][ref_keep], rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(kept["y_exit"], f["out_y_exit"][ref_keep], rtol=1e-6, atol=1e-6)


@pytest.fixture(scope="module")
def c1_scan(c1_params):
    cfg = Config(**dict(c1_params, SC_ON=1, MSC_ON=1, SM_ON=1, SC_LOWER_THRESHOLD=-10.0, SC_UPPER_THRESHOLD=0.0,
                        MSC_DIFF_THRESH=50))
    tr = P.simulate_tracks(P.water_cylinder_phantom(6.0), 60000, seed=31, continuous_angles=False,
                           angle_interval_deg=4.0, t_extent=16.0, v_extent=3.5)
    td = {k: v.numpy() for k, v in P.tracker_data(tr).items()}
    return cfg, td


@pytest.mark.gpu
def test_engine_statistics_fbp_hulls_match_oracle(c1_scan):
    from pct_reconstruction_b200 import Context
    cfg, td = c1_scan
    o = PreOracle(cfg.struct)
    with Context(cfg) as ctx:
        ctx.load_tracker_data(td, integer_angles=True)
        for st in ("recon_volume_intersections", "binning"):
            ctx.stage(st)
        raw = {k: ctx.get_array(k) for k in GEOM}
        missed = ctx.get_array("missed_recon_volume")
        vec = {k: ctx.get_array(k + "_vector") for k in GEOM}
        wepl_vec, bin_vec = ctx.get_array("WEPL_vector"), ctx.get_array("bin_num_vector")
        counts, mw = ctx.get_array("bin_counts"), ctx.get_array("mean_WEPL")
        mu, mv = ctx.get_array("mean_rel_ut_angle"), ctx.get_array("mean_rel_uv_angle")
        ctx.stage("hull_detection")
        g_sc, g_msc, g_sm = ctx.get_array("SC_hull"), ctx.get_array("MSC_counts"), ctx.get_array("SM_counts")
        for st in ("calculate_means", "sum_squared_deviations", "calculate_standard_deviations", "statistical_cuts"):
            ctx.stage(st)
        n_cut = len(ctx.get_array("WEPL_vector"))
        survivors = survivor_keys({k: ctx.get_array(k + "_vector") for k in GEOM}, ctx.get_array("WEPL_vector"))
        g_sino_sums = ctx.get_array("sinogram")
        g_counts2 = ctx.get_array("bin_counts")
        ctx.stage("construct_sinogram")
        ctx.stage("FBP")
        g_filtered, g_fbp, g_med = ctx.get_array("sinogram_filtered"), ctx.get_array("FBP_image"), ctx.get_array(
            "FBP_median_filtered")
        ctx.stage("hull_detection_finish")
        g_msc_hull, g_sm_hull = ctx.get_array("MSC_counts"), ctx.get_array("SM_counts")
    # statistics and cuts from the engine's own binned vectors and sums
    keep, o_counts2, _, _, o_sino_sums = o.statistics_and_cuts(bin_vec, wepl_vec, vec, counts, [mw, mu, mv])
    # survivors as sets: the histories the engine kept vs those the oracle keeps (its standard
    # deviations sum in a fixed order where the engine's use float atomics, so a history within
    # rounding of k*sigma may flip; each such tie is listed)
    kept = keep.astype(bool)
    o_survivors = survivor_keys({k: v[kept] for k, v in vec.items()}, wepl_vec[kept])
    only_engine, only_oracle = survivors - o_survivors, o_survivors - survivors
    print(f"cuts: engine {n_cut} survivors, oracle {int(kept.sum())}; kept only by the engine "
          f"{len(only_engine)}, only by the oracle {len(only_oracle)}")
    for t in list(only_engine)[:5] + list(only_oracle)[:5]:
        print("  tie history (x_entry, y_entry, xy_entry_angle, WEPL bits):", t)
    assert len(survivors) == n_cut
    assert len(only_engine) + len(only_oracle) <= TIE_FRACTION * len(keep)
    # sinogram/filter/backprojection/median from the engine's sums (isolates float-order effects)
    o_sino, o_filtered = o.sinogram_filter(g_counts2, g_sino_sums)
    np.testing.assert_allclose(g_filtered, o_filtered, rtol=2e-5, atol=1e-4)
    o_fbp = o.backprojection(g_filtered)
    np.testing.assert_allclose(g_fbp, o_fbp, rtol=2e-5, atol=1e-4)
    np.testing.assert_array_equal(g_med, o.median_filter(g_fbp, cfg.FBP_MED_FILTER_RADIUS))
    # hull walks from the engine's intersections
    base = o.initialize_hull()
    o_sc, b0 = o.hull_walks(0, raw, ctx_wepl := td["WEPL"], missed, base)
    o_msc, b1 = o.hull_walks(1, raw, ctx_wepl, missed, base)
    o_sm, b2 = o.hull_walks(2, raw, ctx_wepl, missed, base)
    # integer images that do not depend on the walk order: exact (the engine and the oracle run
    # the same uncontracted double arithmetic); the reference itself pins both in
    # tests/test_reference_walks.py
    for name, g, o_img in (("SC", g_sc.astype(np.int32), o_sc), ("MSC", g_msc, o_msc), ("SM", g_sm, o_sm)):
        diff = np.nonzero(g != o_img)[0]
        print(f"{name} hull walks: {len(diff)} voxels differ from the oracle {diff[:10].tolist()}")
        assert len(diff) == 0
    assert b0 == 0 and b1 == 0 and b2 == 0
    np.testing.assert_array_equal(g_msc_hull, o.edge_detection(1, g_msc))
    np.testing.assert_array_equal(g_sm_hull, o.edge_detection(2, g_sm))


@pytest.mark.gpu
def test_full_preprocessing_then_drop(c1_scan):
    from pct_reconstruction_b200 import Context
    cfg, td = c1_scan
    with Context(cfg) as ctx:
        n = ctx.preprocessing(td, integer_angles=True)
        x0 = ctx.x_GPU_2_host()
        hull = ctx.get_array("hull")
        fbp_median = ctx.get_array("FBP_median_filtered")
        assert n > 1000 and hull.sum() > 1000
        # X_0 = HYBRID (initial_iterate_generate_hybrid, B.cu:8582-8591): the (median-filtered) FBP
        # image where the hull is set, 0 elsewhere -- element by element
        np.testing.assert_array_equal(x0, np.where(hull != 0, fbp_median, np.float32(0)))
        assert np.abs(x0[hull == 1]).max() > 0
        ctx.DROP_full_tx_iteration(1)
        x1 = ctx.x_GPU_2_host()
        assert np.isfinite(x1).all() and (x1 != x0).sum() > 1000
        assert ctx.counters()["wait_expired"] == 0
