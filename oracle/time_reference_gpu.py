"""Time the reference's own GPU DROP iteration next to the engine's on the same inputs (needs a B200).

MEASUREMENT INFRASTRUCTURE: runs oracle/_ref/ref_harness (the reference's unmodified B.cu compiled
for sm_100a, built by oracle/build_reference.py) with its `time_drop` command, and the engine through
its C ABI, on the same seeded histories at the reference's built-in configuration (B.h: 256 x 256 x
32 voxels of 0.0625 x 0.0625 x 0.25 cm, R = 8 cm, MLP_U_STEP 0.03125 cm, DROP_BLOCK_SIZE 204800,
HISTORIES_PER_BLOCK 640) -- B.cu's parameters are compile-time, so this is the configuration its
code can be run at.  Both are timed with CUDA events per DROP iteration, histories resident on the
device.  Prints one JSON line: both throughputs, their ratio, and the relative RMSE between the two
images after the timed iterations (float atomics: the scatter order differs).

  python oracle/time_reference_gpu.py [--histories 10000000] [--iterations 3]
"""
from __future__ import annotations

import argparse
import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
from pct_reconstruction_b200 import Config, Context  # noqa: E402
from pct_reconstruction_b200 import phantoms as P  # noqa: E402

HARNESS = ROOT / "oracle" / "_ref" / "ref_harness"
HIST = ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit", "xy_entry_angle", "xz_entry_angle",
        "xy_exit_angle", "xz_exit_angle", "WEPL", "first_MLP_voxel")


def histories(cfg, n, seed):
    parts, have, k = [], 0, 0
    while have < n:
        tr = P.simulate_tracks(P.water_cylinder_phantom(7.0), min(4_000_000, int((n - have) * 1.5) + 1000),
                               seed=seed + k, device="cuda", continuous_angles=True, t_extent=16.0, v_extent=7.0)
        h = P.reconstruction_histories(cfg, tr)
        parts.append(h)
        have += len(h["WEPL"])
        k += 1
    return {key: torch.cat([p[key] for p in parts])[:n].contiguous() for key in parts[0]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--histories", type=int, default=10_000_000)
    ap.add_argument("--iterations", type=int, default=3)
    args = ap.parse_args()
    if not HARNESS.exists():
        print(json.dumps({"unavailable": f"{HARNESS} not built (oracle/build_reference.py)"}))
        return
    cfg = Config()  # the reference's built-in configuration
    hist = histories(cfg, args.histories, seed=4242)
    n = len(hist["WEPL"])
    x0 = (0.9 * P.truth_image(cfg, P.water_cylinder_phantom(7.0), device="cuda") + 0.1).cpu().numpy()

    # the engine first: its voxel indices are the reference's bit for bit, so its bounds counters say
    # whether the reference's kernels (which do not check) would index outside their arrays
    ctx = Context(cfg)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_reconstruction_histories(hist)
    ctx.x_host_2_GPU(x0)
    ms = []
    for it in range(args.iterations):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx.DROP_full_tx_iteration(it + 1)
        b.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    x = ctx.x_GPU_2_host().astype(np.float64)
    counters = ctx.counters()
    ctx.close()
    if counters["voxel_oob"] or counters["path_overflow"] or counters["table_range"]:
        print(json.dumps({"unavailable": f"inputs would index outside the reference's arrays: {counters}"}))
        return

    with tempfile.TemporaryDirectory() as d:
        for k in HIST:
            a = hist[k].cpu().numpy()
            if k == "first_MLP_voxel":
                a = a.view(np.uint32)
            np.ascontiguousarray(a).tofile(Path(d) / f"{k}.bin")
        x0.astype(np.float32).tofile(Path(d) / "x.bin")
        np.array([cfg.DROP_BLOCK_SIZE, args.iterations], np.int32).tofile(Path(d) / "drop_params.bin")
        subprocess.run([str(HARNESS), "time_drop", d], check=True)
        ref_ms = np.fromfile(Path(d) / "out_ms.bin", np.float32)
        ref_x = np.fromfile(Path(d) / "out_x.bin", np.float32)

    # the engine's other modes on the same inputs: mixed-precision path kernel, and precomputed-path
    # DROP (paths computed by the first iteration and kept; not an MLP+DROP iteration)
    modes = {}
    for name, over, reuse in (("mixed_precision", {"PRECISION": "MIXED"}, False), ("precomputed_paths", {}, True)):
        c2 = Context(Config(**over))
        c2.set_stream(stream.cuda_stream)
        c2.set_reconstruction_histories(hist)
        c2.x_host_2_GPU(x0)
        c2.set_path_reuse(reuse)
        c2.DROP_full_tx_iteration(1)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for it in range(2):
            c2.DROP_full_tx_iteration(it + 2)
        b.record(stream)
        torch.cuda.synchronize()
        m = a.elapsed_time(b) / 2
        modes[name] = {"ms_per_iteration": m, "histories_per_s": n / (m / 1000.0)}
        c2.close()

    ref_best, eng_best = float(np.min(ref_ms)), float(np.min(ms[1:] if len(ms) > 1 else ms))
    rmse = float(np.sqrt(np.mean((x - ref_x) ** 2)) / np.sqrt(np.mean(ref_x.astype(np.float64) ** 2)))
    print(json.dumps({
        "config": f"reference built-in: {cfg.COLUMNS}x{cfg.ROWS}x{cfg.SLICES} voxels, MLP step {cfg.MLP_U_STEP} cm, "
                  f"DROP blocks {cfg.DROP_BLOCK_SIZE}, HISTORIES_PER_BLOCK {cfg.HISTORIES_PER_BLOCK}",
        "histories": n, "iterations": args.iterations,
        "reference_gpu_ms_per_iteration": [float(v) for v in ref_ms],
        "engine_ms_per_iteration": ms,
        "reference_gpu_histories_per_s": n / (ref_best / 1000.0),
        "engine_histories_per_s": n / (eng_best / 1000.0),
        "speedup": ref_best / eng_best,
        "image_rel_rmse_engine_vs_reference": rmse,
        "engine_other_modes": {k: dict(v, speedup_vs_reference_gpu=ref_best / v["ms_per_iteration"])
                               for k, v in modes.items()}}))


if __name__ == "__main__":
    main()
