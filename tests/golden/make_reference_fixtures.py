"""Generate golden fixtures from the reference's own device code (run on a machine with a B200).

The reference ships no tests or golden vectors.  This script feeds seeded synthetic inputs to the
reference's unmodified B.cu compiled for sm_100a and linked with a harness (oracle/build_reference.py,
oracle/ref_harness.cu), and stores inputs and the reference's outputs as compressed .npz fixtures.
B.cu's parameters are compile-time, so each fixture uses one of the two harness builds:
  * oracle/_ref/ref_harness, the reference's built-in configuration (B.h defaults: 256 x 256 x 32
    voxels of 0.0625 x 0.0625 x 0.25 cm, R = 8 cm, MLP_U_STEP 0.03125 cm, HISTORIES_PER_BLOCK 640):
    ref_mlp, ref_drop, ref_intersections_binning, ref_endpoints, ref_stats_fbp, ref_edges and
    ref_hull_walks;
  * oracle/_ref/head/ref_harness, the head-size grid from a patched copy of B.h (200 x 200 x 32
    voxels of 0.1 x 0.1 x 0.25 cm, R = 10 cm, MLP_U_STEP 0.05 cm, HISTORIES_PER_BLOCK 480):
    ref_hull_walks_head, ref_mlp_head, ref_drop_head and ref_tvs_head;
  * oracle/_ref/scurve/ref_harness, the built-in configuration with S_CURVE_ON set to ON:
    ref_s_curve (the five S-curve functions and s_curve_scale_GPU) and ref_drop_scurve (the
    ref_drop iteration with the S-curve attenuation).
Inputs too large to store are regenerated from their seed on cuda:0 (tests/golden/fixture_inputs.py)
and the fixture keeps their SHA-256.

  python tests/golden/make_reference_fixtures.py --out <dir> [--only name,name,...]
"""
from __future__ import annotations

import argparse
import hashlib
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))
from fixture_inputs import GEOM6, HEAD, HIST, default_image, head_histories, head_tracker_data, sha256_of  # noqa: E402
from pct_reconstruction_b200 import Config  # noqa: E402
from pct_reconstruction_b200 import phantoms as P  # noqa: E402

HARNESS = ROOT / "oracle" / "_ref" / "ref_harness"
HARNESS_HEAD = ROOT / "oracle" / "_ref" / "head" / "ref_harness"
HARNESS_SCURVE = ROOT / "oracle" / "_ref" / "scurve" / "ref_harness"
GOLDEN = Path(__file__).resolve().parent
# path lengths of the s_curve_scale_GPU pairs (every j < n of each): MIN_MLP_LENGTH, odd and even
# lengths around the sigmoid's midpoint, and the longest list the reference's MLP writes
S_CURVE_LENGTHS = (30, 31, 41, 100, 257, 1280)
GEOM = ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit", "xy_entry_angle", "xz_entry_angle",
        "xy_exit_angle", "xz_exit_angle")
# WEPL windows of the hull-walk fixtures (cm): SC carves [-10, -0.05], MSC counts [-10, 0.1], SM
# counts WEPL >= 2; different windows so that each hull sees its own set of walks
WALK_WINDOWS = np.array([-10.0, -0.05, -10.0, 0.1, 2.0], np.float64)


def edge_counts(C, R, S):
    """Seeded synthetic hit-count image for the edge-detection fixture: a plateau inside 0.42*C
    falling off outside, +2% per slice, integer noise in [0, 12)."""
    yy, xx = np.mgrid[0:R, 0:C]
    r2 = ((xx - C / 2 + 0.5) ** 2 + (yy - R / 2 + 0.5) ** 2) / (0.42 * C) ** 2
    rng = np.random.default_rng(17)
    counts = np.stack([np.where(r2 < 1.0, 300 - 40 * r2, 300 * np.exp(-6 * (r2 - 1.0))) * (1 + 0.02 * k)
                       for k in range(S)])
    return (counts + rng.integers(0, 12, counts.shape)).astype(np.int32).ravel()


def run(cmd, d, arrays, harness=HARNESS):
    for k, v in arrays.items():
        np.ascontiguousarray(v).tofile(Path(d) / f"{k}.bin")
    subprocess.run([str(harness), cmd, str(d)], check=True)


def out(d, name, dtype):
    return np.fromfile(Path(d) / f"out_{name}.bin", dtype=dtype)


def sparse(a):
    """Nonzero entries of an integer image: delta-coded indices and values."""
    nz = np.nonzero(a)[0]
    delta = np.diff(np.concatenate([[-1], nz]))
    return delta.astype(np.uint32), a[nz].astype(np.int32)


def walks_fixture(harness, geom, wepl, missed, extra, path):
    """The hull walks of SC_GPU/MSC_GPU/SM_GPU (bounded harness walk) on stored geometry."""
    with tempfile.TemporaryDirectory() as d:
        run("walks", d, {**{k: geom[k] for k in GEOM6}, "WEPL": wepl, "missed_recon_volume": missed,
                         "walk_params": WALK_WINDOWS}, harness)
        carved = out(d, "SC_carved", np.uint8)
        msc_d, msc_v = sparse(out(d, "MSC_counts", np.int32))
        sm_d, sm_v = sparse(out(d, "SM_counts", np.int32))
        status, steps = out(d, "status", np.int32), out(d, "steps", np.int32)
    print(path.name, "walk status counts (ended / below zero / step bound):", np.bincount(status, minlength=3))
    np.savez_compressed(path, **extra, walk_windows=WALK_WINDOWS, num_voxels=np.int64(len(carved)),
                        out_SC_carved=np.packbits(carved), out_MSC_delta=msc_d, out_MSC_values=msc_v,
                        out_SM_delta=sm_d, out_SM_values=sm_v, out_status=status.astype(np.uint8),
                        out_steps=steps.astype(np.uint16))


def make_hull_walks(dst):
    """Built-in configuration, on the reference's own intersections of ref_intersections_binning."""
    f = np.load(Path(__file__).resolve().parent / "ref_intersections_binning.npz")
    geom = {k: f["out_" + k] for k in GEOM6}
    walks_fixture(HARNESS, geom, f["WEPL"], f["missed_recon_volume"], {"source": np.array("ref_intersections_binning")},
                  dst / "ref_hull_walks.npz")


def make_hull_walks_head(dst):
    """Head grid: the reference's intersections (integer gantry angles) of 16000 simulated
    head-phantom protons, then its walks."""
    td = head_tracker_data(16000, seed=515)
    with tempfile.TemporaryDirectory() as d:
        run("intersections", d, td, HARNESS_HEAD)
        geom = {k: out(d, k, np.float32) for k in GEOM6}
        missed = out(d, "missed_recon_volume", np.uint8)
    hit = missed == 0
    geom = {k: v[hit] for k, v in geom.items()}
    walks_fixture(HARNESS_HEAD, geom, td["WEPL"][hit], np.zeros(int(hit.sum()), np.uint8),
                  {**{"in_" + k: v for k, v in geom.items()}, "in_WEPL": td["WEPL"][hit]},
                  dst / "ref_hull_walks_head.npz")


def check_bounds(cfg, hist):
    """The reference's MLP and DROP kernels index the image with unchecked voxel numbers.  The
    engine's voxel lists are the reference's, and the engine counts every entry outside the
    (one-slice padded) image, so it runs first: the reference's kernels are only run on inputs
    where that count is 0."""
    from pct_reconstruction_b200 import Context
    with Context(cfg) as ctx:
        ctx.set_reconstruction_histories(hist)
        ctx.x_host_2_GPU(default_image(cfg.NUM_VOXELS))
        import torch
        counts = torch.zeros(len(hist["WEPL"]), dtype=torch.int32, device="cuda")
        ctx.mlp_paths_device(0, len(hist["WEPL"]), 0, counts, None, None, None)
        ctx.synchronize()
        c = ctx.counters()
    if c["voxel_oob"] or c["path_overflow"] or c["table_range"]:
        raise SystemExit(f"inputs would index outside the reference's arrays: {c}")


def make_mlp_head(dst):
    """Head grid: MLP voxel lists, chords and sums of x of 2000 histories (inputs stored)."""
    cfg = Config(**HEAD)
    hist = head_histories(cfg, 2000, seed=616)
    check_bounds(cfg, hist)
    x0 = default_image(cfg.NUM_VOXELS)
    with tempfile.TemporaryDirectory() as d:
        run("mlp", d, {**hist, "x": x0}, HARNESS_HEAD)
        counts, voxels = out(d, "counts", np.uint32), out(d, "voxels", np.uint32)
        np.savez_compressed(dst / "ref_mlp_head.npz", **hist, counts=counts,
                            voxels_delta=np.diff(np.concatenate([[0], voxels.astype(np.int64)])).astype(np.int32),
                            chord=out(d, "chord", np.float64), a_dot_x=out(d, "a_dot_x", np.float64))


def make_drop_head(dst):
    """Head grid: one DROP iteration over 120000 histories in two blocks of 60000 (each block's
    ⌊60000/480⌋ x 480 = 60000 histories are all processed), from default_image; the inputs are
    regenerated from their seed, the image kept as every 7th voxel plus the SHA-256 of all."""
    cfg = Config(**HEAD)
    n = 120000
    hist = head_histories(cfg, n, seed=717)
    check_bounds(cfg, hist)
    x0 = default_image(cfg.NUM_VOXELS)
    with tempfile.TemporaryDirectory() as d:
        run("drop", d, {**hist, "x": x0, "drop_params": np.array([cfg.DROP_BLOCK_SIZE], np.int32)}, HARNESS_HEAD)
        x1 = out(d, "x", np.float32)
    np.savez_compressed(dst / "ref_drop_head.npz", seed=np.int64(717), histories=np.int64(n),
                        inputs_sha256=sha256_of(hist), sample_step=np.int64(7), out_x_sample=x1[::7],
                        out_x_sha256=np.frombuffer(hashlib.sha256(x1.tobytes()).digest(), np.uint8),
                        changed=np.int64(int((x1 != x0).sum())))


def tvs_images(cfg):
    """Two head-grid images for the TVS fixture: the head phantom's RSP (piecewise constant, so
    most gradients are zero) and default_image (every gradient non-zero)."""
    return {"phantom": P.truth_image(cfg, P.head_phantom()).numpy(), "hash": default_image(cfg.NUM_VOXELS)}


def make_tvs_head(dst):
    """Head grid: the reference's calculate_total_variation and generate_perturbation_array (host
    code) on two images; the direction is kept as every 5th voxel plus the SHA-256 of all."""
    cfg = Config(**HEAD)
    out_arrays = {}
    for name, x in tvs_images(cfg).items():
        with tempfile.TemporaryDirectory() as d:
            run("tvs", d, {"x": x}, HARNESS_HEAD)
            out_arrays[f"{name}_x_sha256"] = np.frombuffer(hashlib.sha256(x.tobytes()).digest(), np.uint8)
            out_arrays[f"{name}_TV"] = out(d, "TV", np.float32)
            v = out(d, "v", np.float32)
            out_arrays[f"{name}_v_sample"] = v[::5]
            out_arrays[f"{name}_v_sha256"] = np.frombuffer(hashlib.sha256(v.tobytes()).digest(), np.uint8)
    np.savez_compressed(dst / "ref_tvs_head.npz", sample_step=np.int64(5), **out_arrays)


def make_builtin(dst):
    """The built-in configuration's fixtures (MLP, DROP, intersections, binning, endpoints,
    statistics and FBP, edge detection)."""
    cfg = Config()  # the reference's built-in configuration
    nv = cfg.NUM_VOXELS
    phantom = P.water_cylinder_phantom(7.0)
    tracks = P.simulate_tracks(phantom, 20000, seed=2024, continuous_angles=True, t_extent=16.0, v_extent=7.0)
    hist = {k: v.numpy() for k, v in P.reconstruction_histories(cfg, tracks).items()}
    hist["first_MLP_voxel"] = hist["first_MLP_voxel"].view(np.uint32)
    x0 = default_image(nv)

    with tempfile.TemporaryDirectory() as d:
        # MLP voxel lists
        n_mlp = 2000
        sub = {k: v[:n_mlp] for k, v in hist.items()}
        run("mlp", d, {**sub, "x": x0})
        np.savez_compressed(dst / "ref_mlp.npz", **sub, counts=out(d, "counts", np.uint32),
                            voxels=out(d, "voxels", np.uint32), chord=out(d, "chord", np.float64),
                            a_dot_x=out(d, "a_dot_x", np.float64))
    with tempfile.TemporaryDirectory() as d:
        # one DROP iteration, blocks of 2000 (each covers floor(2000/640)*640 = 1920 histories)
        n_drop = 6000
        sub = {k: v[:n_drop] for k, v in hist.items()}
        run("drop", d, {**sub, "x": x0, "drop_params": np.array([2000], np.int32)})
        x1 = out(d, "x", np.float32)
        changed = np.nonzero(x1 != x0)[0]
        delta = np.diff(np.concatenate([[-1], changed]))  # changed voxel indices, delta-coded
        np.savez_compressed(dst / "ref_drop.npz", **sub, drop_block_size=np.int32(2000),
                            changed_delta=delta.astype(np.uint16 if delta.max() < 65536 else np.uint32),
                            values=x1[changed])
    # recon-volume intersections and binning from tracker hits (integer gantry angles)
    tracks_d = P.simulate_tracks(phantom, 20000, seed=77, continuous_angles=False, angle_interval_deg=4.0,
                                 t_extent=16.0, v_extent=7.0)
    td = {k: v.numpy() for k, v in P.tracker_data(tracks_d).items()}
    td["gantry_angle"] = np.rint(td["gantry_angle"]).astype(np.int32)
    with tempfile.TemporaryDirectory() as d:
        run("binning", d, td)
        res = {k: out(d, k, np.float32) for k in ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit",
                                                 "xy_entry_angle", "xz_entry_angle", "xy_exit_angle",
                                                 "xz_exit_angle")}
        missed = out(d, "missed_recon_volume", np.uint8)
        bin_num = out(d, "bin_num", np.int32)
        bin_counts = out(d, "bin_counts", np.int32)
        sum_wepl = out(d, "sum_WEPL", np.float32)
        nz = np.nonzero(bin_counts)[0].astype(np.int32)
        np.savez_compressed(dst / "ref_intersections_binning.npz", **td,
                            **{"out_" + k: v for k, v in res.items()}, missed_recon_volume=missed,
                            bin_num=bin_num, bins_nonzero=nz, bin_counts_nonzero=bin_counts[nz],
                            sum_WEPL_nonzero=sum_wepl[nz])
        # MLP endpoints against the phantom's hull, from the intersections of the histories that
        # hit the reconstruction volume
        keep = np.nonzero(missed == 0)[0][:8000]
        ep_in = {k: res[k][keep] for k in res}
        ep_in["WEPL"] = td["WEPL"][keep]
        ep_in["first_MLP_voxel"] = np.zeros(len(keep), np.uint32)
        hull = P.hull_image(cfg, phantom).numpy().astype(np.uint8)
    with tempfile.TemporaryDirectory() as d:
        run("endpoints", d, {**ep_in, "hull": hull})
        ep_out = {k: out(d, k, np.float32) for k in ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit")}
        np.savez_compressed(dst / "ref_endpoints.npz", **ep_in, hull_radius=np.float64(7.0),
                            out_first_MLP_voxel=out(d, "first_MLP_voxel", np.uint32),
                            **{"out_" + k: v for k, v in ep_out.items()})
    # statistics, cuts, sinogram, filter and backprojection: histories concentrated on a few
    # thousand bins (narrow t/v extent, 90 discrete angles) so that bins hold several histories
    tracks_s = P.simulate_tracks(phantom, 80000, seed=91, continuous_angles=False, angle_interval_deg=4.0,
                                 t_extent=2.0, v_extent=1.0)
    ts = {k: v.numpy() for k, v in P.tracker_data(tracks_s).items()}
    ts["gantry_angle"] = np.rint(ts["gantry_angle"]).astype(np.int32)
    geom_names = ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit", "xy_entry_angle",
                  "xz_entry_angle", "xy_exit_angle", "xz_exit_angle")
    with tempfile.TemporaryDirectory() as d:
        run("binning", d, ts)
        g = {k: out(d, k, np.float32) for k in geom_names}
        missed = out(d, "missed_recon_volume", np.uint8)
        bin_num = out(d, "bin_num", np.int32)
        sums = {k: out(d, k, np.float32) for k in ("sum_WEPL", "sum_ut", "sum_uv")}
        bin_counts = out(d, "bin_counts", np.int32)
    keep = np.nonzero((missed == 0) & (bin_num >= 0))[0]  # binning()'s host compaction (B.cu:5429-5450)
    vec = {k: g[k][keep] for k in ("xy_entry_angle", "xz_entry_angle", "xy_exit_angle", "xz_exit_angle")}
    vec["WEPL"] = ts["WEPL"][keep]
    vec["bin_num"] = bin_num[keep]
    with tempfile.TemporaryDirectory() as d:
        run("stats_fbp", d, {**vec, "bin_counts": bin_counts, **sums})
        nz = np.nonzero(bin_counts)[0].astype(np.int32)
        res = {k: out(d, k, np.float32)[nz] for k in ("mean_WEPL", "mean_rel_ut_angle", "mean_rel_uv_angle",
                                                     "stddev_WEPL", "stddev_rel_ut_angle", "stddev_rel_uv_angle",
                                                     "sinogram_sums", "sinogram")}
        failed = out(d, "failed_cuts", np.uint8)
        counts_full = out(d, "bin_counts", np.int32)
        sums_full = out(d, "sinogram_sums", np.float32)
        counts_after = counts_full[nz]
        fbp_in_run = out(d, "FBP_image", np.float32)
    # the FBP stages again, alone, on the stored counts and sums: the fixture's FBP outputs must be a
    # function of what the fixture stores, not of the float-atomic order inside the run above
    fbp_runs = []
    for _ in range(2):
        with tempfile.TemporaryDirectory() as d:
            run("fbp", d, {"bin_counts": counts_full, "sinogram_sums": sums_full})
            fbp_runs.append({k: out(d, k, t) for k, t in (("sinogram", np.float32), ("sinogram_filtered", np.float32),
                                                          ("FBP_image", np.float32), ("FBP_median", np.float32),
                                                          ("FBP_hull", np.uint8))})
    for k in fbp_runs[0]:
        assert fbp_runs[0][k].tobytes() == fbp_runs[1][k].tobytes(), f"reference {k} not reproducible"
    assert fbp_runs[0]["sinogram"][nz].tobytes() == res["sinogram"].tobytes()
    print("FBP voxels differing between the chained run and the stand-alone run:",
          int(np.sum(fbp_in_run.view(np.uint32) != fbp_runs[0]["FBP_image"].view(np.uint32))))
    filt = fbp_runs[0]["sinogram_filtered"]
    fnz = np.nonzero(filt)[0].astype(np.int32)
    fbp = fbp_runs[0]["FBP_image"]
    fbp_med = fbp_runs[0]["FBP_median"]
    fbp_hull = fbp_runs[0]["FBP_hull"]
    import hashlib
    sample = np.arange(0, len(fbp), 13, dtype=np.int64)
    np.savez_compressed(dst / "ref_stats_fbp.npz", **{"in_" + k: v for k, v in vec.items()},
                        bins_nonzero=nz, in_bin_counts=bin_counts[nz],
                        **{"in_" + k: v[nz] for k, v in sums.items()},
                        **{"out_" + k: v for k, v in res.items()}, out_failed_cuts=failed,
                        out_bin_counts=counts_after, filtered_nonzero=fnz, out_sinogram_filtered=filt[fnz],
                        out_FBP_sha256=np.frombuffer(hashlib.sha256(fbp.tobytes()).digest(), np.uint8),
                        FBP_sample_step=np.int64(13), out_FBP_sample=fbp[sample],
                        out_FBP_median_sha256=np.frombuffer(hashlib.sha256(fbp_med.tobytes()).digest(), np.uint8),
                        out_FBP_median_sample=fbp_med[sample], out_FBP_hull=np.packbits(fbp_hull))
    # MSC / SM edge detection on a smooth synthetic counts image (the walks that fill the counts are
    # not run: on some inputs they never terminate)
    counts = edge_counts(cfg.COLUMNS, cfg.ROWS, cfg.SLICES)
    with tempfile.TemporaryDirectory() as d:
        run("edges", d, {"counts": counts})
        import hashlib
        np.savez_compressed(dst / "ref_edges.npz",
                            counts_sha256=np.frombuffer(hashlib.sha256(counts.tobytes()).digest(), np.uint8),
                            out_MSC_hull=np.packbits(out(d, "MSC_hull", np.int32).astype(np.uint8)),
                            out_SM_hull=np.packbits(out(d, "SM_hull", np.int32).astype(np.uint8)),
                            out_SM_thresholds=out(d, "SM_thresholds", np.int32))


def make_s_curve(dst):
    """The reference's S-curve functions for k < 1312 (rows in the S_CURVES order SIGMOID, TANH,
    ATAN, ERF, LIN_OVER_ROOT) and s_curve_scale_GPU(j, n) for every j < n of S_CURVE_LENGTHS."""
    count = 1312
    n = np.concatenate([np.full(m, m, np.uint32) for m in S_CURVE_LENGTHS])
    j = np.concatenate([np.arange(m, dtype=np.uint32) for m in S_CURVE_LENGTHS])
    with tempfile.TemporaryDirectory() as d:
        run("scurve", d, {"scurve_params": np.array([count], np.int32), "scurve_j": j, "scurve_n": n}, HARNESS_SCURVE)
        curves = out(d, "curves", np.float32).reshape(5, count)
        scale = out(d, "scale", np.float32)
    np.savez_compressed(dst / "ref_s_curve.npz", curves=curves, j=j, n=n, scale=scale)


def make_drop_scurve(dst):
    """ref_drop's DROP iteration (its stored 6000 histories, blocks of 2000, from default_image)
    through the S_CURVE_ON build; the changed voxels as in ref_drop."""
    f = dict(np.load(GOLDEN / "ref_drop.npz"))
    hist = {k: f[k] for k in HIST}
    x0 = default_image(Config().NUM_VOXELS)
    with tempfile.TemporaryDirectory() as d:
        run("drop", d, {**hist, "x": x0, "drop_params": np.array([int(f["drop_block_size"])], np.int32)},
            HARNESS_SCURVE)
        x1 = out(d, "x", np.float32)
    changed = np.nonzero(x1 != x0)[0]
    delta = np.diff(np.concatenate([[-1], changed]))
    np.savez_compressed(dst / "ref_drop_scurve.npz", drop_block_size=f["drop_block_size"],
                        inputs_sha256=sha256_of(hist),
                        changed_delta=delta.astype(np.uint16 if delta.max() < 65536 else np.uint32),
                        values=x1[changed])


MAKERS = {"builtin": make_builtin, "hull_walks": make_hull_walks, "hull_walks_head": make_hull_walks_head,
          "mlp_head": make_mlp_head, "drop_head": make_drop_head, "tvs_head": make_tvs_head,
          "s_curve": make_s_curve, "drop_scurve": make_drop_scurve}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--only", default=",".join(MAKERS), help="comma-separated subset of " + ",".join(MAKERS))
    args = ap.parse_args()
    dst = Path(args.out)
    dst.mkdir(parents=True, exist_ok=True)
    for name in args.only.split(","):
        MAKERS[name](dst)
    for f in sorted(dst.glob("ref_*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
