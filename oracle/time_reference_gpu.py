"""Time the reference's own GPU DROP iteration next to the engine's on the same inputs (needs a B200).

MEASUREMENT INFRASTRUCTURE: runs a harness build of the reference's unmodified B.cu
(oracle/build_reference.py) with its `time_drop` command -- per DROP block a kernel that does what
calculate_x_update_GPU (B.cu:9321) does (find_MLP_path_GPU_tabulated + DROP_block_update_GPU), then
image_update_GPU (B.cu:9398) -- and the engine through its C ABI, on the same seeded histories.
B.cu's parameters are compile-time, so each configuration has its own harness build:

  --config head     the head-size workload of bench.py: 200 x 200 x 32 voxels of 0.1 x 0.1 x 0.25 cm,
                    MLP_U_STEP 0.05 cm, DROP blocks of 60000, HISTORIES_PER_BLOCK 480, head phantom
                    with continuous angles (default 50M histories); harness oracle/_ref/head/ref_harness
  --config builtin  the reference's B.h values: 256 x 256 x 32 voxels of 0.0625 x 0.0625 x 0.25 cm,
                    MLP_U_STEP 0.03125 cm, DROP blocks of 204800, HISTORIES_PER_BLOCK 640, water
                    cylinder (default 10M histories); harness oracle/_ref/ref_harness
  --config small    the small workload of bench.py: 128 x 128 x 16 voxels of 0.1 x 0.1 x 0.25 cm,
                    MLP_U_STEP 0.1 cm, DROP blocks of 3200, HISTORIES_PER_BLOCK 640, water cylinder with
                    four inserts, 90 angles (default 2M histories); harness oracle/_ref/small/ref_harness

Both are timed with CUDA events per DROP iteration, histories resident on the device.  The engine
runs first: its voxel indices are the reference's bit for bit and it counts every index outside
the padded image, so the reference's kernels (which do not check) only run when that count is 0.
Prints one JSON line: both throughputs, their ratio, and the relative RMSE between the two images
after the timed iterations (float atomics: the scatter order differs).

  python oracle/time_reference_gpu.py [--config head|builtin|small] [--histories N] [--iterations 3]
"""
from __future__ import annotations

import argparse
import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
HARNESS = {"builtin": ROOT / "oracle" / "_ref" / "ref_harness", "head": ROOT / "oracle" / "_ref" / "head" / "ref_harness",
           "small": ROOT / "oracle" / "_ref" / "small" / "ref_harness"}
HIST = ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit", "xy_entry_angle", "xz_entry_angle",
        "xy_exit_angle", "xz_exit_angle", "WEPL", "first_MLP_voxel")
# B.h values of the head harness build (the patched macros; everything else at B.h's value)
HEAD_PARAMS = dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, RECON_CYL_RADIUS=10.0, DROP_BLOCK_SIZE=60000,
                   HISTORIES_PER_BLOCK=480)
SMALL_PARAMS = dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, RECON_CYL_RADIUS=6.4, SSD_V_SIZE=5.0, DROP_BLOCK_SIZE=3200,
                    HISTORIES_PER_BLOCK=640, MLP_U_STEP=0.1)


def reference_gpu_iterations(config: str, hist: dict, x0: np.ndarray, drop_block_size: int, iterations: int):
    """The reference's DROP iterations on `hist` (host or CUDA arrays) from image x0: milliseconds
    per iteration (CUDA events inside the harness) and the final image."""
    exe = HARNESS[config]
    if not exe.exists():
        raise FileNotFoundError(f"{exe} not built (oracle/build_reference.py)")
    with tempfile.TemporaryDirectory() as d:
        for k in HIST:
            a = hist[k]
            a = a.cpu().numpy() if hasattr(a, "cpu") else np.asarray(a)
            if k == "first_MLP_voxel":
                a = a.view(np.uint32)
            np.ascontiguousarray(a).tofile(Path(d) / f"{k}.bin")
        np.ascontiguousarray(x0, np.float32).tofile(Path(d) / "x.bin")
        np.array([drop_block_size, iterations], np.int32).tofile(Path(d) / "drop_params.bin")
        subprocess.run([str(exe), "time_drop", d], check=True)
        return np.fromfile(Path(d) / "out_ms.bin", np.float32), np.fromfile(Path(d) / "out_x.bin", np.float32)


def builtin_histories(cfg, n, seed):
    import torch
    from pct_reconstruction_b200 import phantoms as P
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
    import torch
    sys.path.insert(0, str(ROOT))
    from pct_reconstruction_b200 import Config, Context
    from pct_reconstruction_b200 import phantoms as P
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", choices=["head", "builtin", "small"], default="head")
    ap.add_argument("--histories", type=int, default=None)
    ap.add_argument("--iterations", type=int, default=3)
    args = ap.parse_args()
    if not HARNESS[args.config].exists():
        print(json.dumps({"unavailable": f"{HARNESS[args.config]} not built (oracle/build_reference.py)"}))
        return
    import bench
    if args.config in ("head", "small"):
        from pct_reconstruction_b200 import replicas
        workload = "head" if args.config == "head" else "water"
        n_req = args.histories or (50_000_000 if args.config == "head" else 2_000_000)
        cfg = Config(**bench.workload_params(workload))
        params = HEAD_PARAMS if args.config == "head" else SMALL_PARAMS
        assert all(getattr(cfg, k) == v for k, v in params.items() if k not in ("RECON_CYL_RADIUS", "SSD_V_SIZE"))
        hist, x0_t = bench.generate(cfg, workload, n_req, seed=replicas.replica_seed(1, 0), device="cuda")
        x0 = x0_t.cpu().numpy()
        desc = f"{args.config} bench workload (bench.py generate, the same seed as its timed scan)"
    else:
        cfg = Config()
        hist = builtin_histories(cfg, args.histories or 10_000_000, seed=4242)
        x0 = (0.9 * P.truth_image(cfg, P.water_cylinder_phantom(7.0), device="cuda") + 0.1).cpu().numpy()
        desc = "water cylinder r = 7 cm, continuous angles"
    n = len(hist["WEPL"])

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

    ref_ms, ref_x = reference_gpu_iterations(args.config, hist, x0, cfg.DROP_BLOCK_SIZE, args.iterations)

    # the engine's other modes on the same inputs: mixed-precision path kernel, and precomputed-path
    # DROP (paths computed by the first iteration and kept; not an MLP+DROP iteration)
    modes = {}
    base = dict(bench.workload_params({"head": "head", "small": "water"}[args.config])) if args.config != "builtin" else {}
    for name, over, reuse in (("mixed_precision", {"PRECISION": "MIXED"}, False), ("precomputed_paths", {}, True)):
        c2 = Context(Config(**base, **over))
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
        "config": f"{args.config}: {cfg.COLUMNS}x{cfg.ROWS}x{cfg.SLICES} voxels, MLP step {cfg.MLP_U_STEP} cm, "
                  f"DROP blocks {cfg.DROP_BLOCK_SIZE}, HISTORIES_PER_BLOCK {cfg.HISTORIES_PER_BLOCK}; {desc}",
        "histories": n, "iterations": args.iterations, "engine_bounds_counters": counters,
        "inputs_fingerprint": bench.inputs_fingerprint(hist) if args.config != "builtin" else None,
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
