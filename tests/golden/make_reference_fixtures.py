"""Generate golden fixtures from the reference's own device code (run on a machine with a B200).

The reference ships no tests or golden vectors.  This script feeds seeded synthetic inputs to
oracle/_ref/ref_harness -- the reference's unmodified B.cu compiled for sm_100a and linked with a
harness (oracle/build_reference.py, oracle/ref_harness.cu) -- and stores inputs and the
reference's outputs as compressed .npz fixtures.  It works at the reference's built-in
configuration (B.h defaults: 256 x 256 x 32 voxels of 0.0625 x 0.0625 x 0.25 cm, R = 8 cm,
MLP_U_STEP 0.03125 cm, HISTORIES_PER_BLOCK 640), because B.cu's parameters are compile-time.

  python tests/golden/make_reference_fixtures.py --out <dir>
"""
from __future__ import annotations

import argparse
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from pct_reconstruction_b200 import Config  # noqa: E402
from pct_reconstruction_b200 import phantoms as P  # noqa: E402

HARNESS = ROOT / "oracle" / "_ref" / "ref_harness"
HIST = ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit", "xy_entry_angle", "xz_entry_angle",
        "xy_exit_angle", "xz_exit_angle", "WEPL", "first_MLP_voxel")


def default_image(nv: int) -> np.ndarray:
    """Deterministic non-uniform image used as x_0 by the MLP and DROP fixtures."""
    i = np.arange(nv, dtype=np.uint64)
    return (0.5 + ((i * np.uint64(2654435761)) % np.uint64(1000)).astype(np.float64) / 1000.0).astype(np.float32)


def edge_counts(C, R, S):
    """Seeded synthetic hit-count image for the edge-detection fixture: a plateau inside 0.42*C
    falling off outside, +2% per slice, integer noise in [0, 12)."""
    yy, xx = np.mgrid[0:R, 0:C]
    r2 = ((xx - C / 2 + 0.5) ** 2 + (yy - R / 2 + 0.5) ** 2) / (0.42 * C) ** 2
    rng = np.random.default_rng(17)
    counts = np.stack([np.where(r2 < 1.0, 300 - 40 * r2, 300 * np.exp(-6 * (r2 - 1.0))) * (1 + 0.02 * k)
                       for k in range(S)])
    return (counts + rng.integers(0, 12, counts.shape)).astype(np.int32).ravel()


def run(cmd, d, arrays):
    for k, v in arrays.items():
        np.ascontiguousarray(v).tofile(Path(d) / f"{k}.bin")
    subprocess.run([str(HARNESS), cmd, str(d)], check=True)


def out(d, name, dtype):
    return np.fromfile(Path(d) / f"out_{name}.bin", dtype=dtype)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    args = ap.parse_args()
    dst = Path(args.out)
    dst.mkdir(parents=True, exist_ok=True)
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
    for f in sorted(dst.glob("ref_*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
