#!/usr/bin/env python3
"""MLP + DROP throughput on B200: histories per second per DROP iteration.

Workload (default): head-size plain pipeline -- 200x200x32 voxels of 1x1x2.5 mm, ellipsoidal
head phantom, continuous stage angles, 50M reconstruction histories, DROP blocks of 60000
histories (HISTORIES_PER_BLOCK 480, so every history of a block is processed), MLP step
VOXEL_WIDTH/2, lambda 1e-4, exact (FP64, reference-rounding) MLP.  A step is one DROP iteration
over all histories: the MLP path kernel (in chunks of DROP blocks, on a low-priority stream, chunk
size, histories per CTA and order window chosen by pct_autotune_schedule), and per DROP block the gather/update/scatter kernel and the image
update, all replayed from one CUDA graph.  Inputs (2.4 GB of history arrays) are larger than L2, so
no flush is needed between steps.  The line also carries e2e (host buffers, uploads overlapped with
the previous step), the roofline object, the CPU baseline and, under `secondary`, precomputed-path
DROP, mixed precision, the L2 window, the learned start and the preprocessing stages.

  python bench.py [--gpus N --steps K --warmup W]       # this engine
  python bench.py --impl reference ...                   # the reference's host MLP+DROP (CPU)
  python bench.py --workload water|batch|learned|precision|preprocessing   # other configurations

With N > 1 (torchrun) every rank reconstructs its own scan: the path has no data-parallel split
inside a DROP block that pays off at these block sizes, so ranks are independent replicas and
`value` is the total histories of all ranks divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import ctypes as C

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "MLP+DROP histories/s/iter on 1 B200"
# FP64 operations (add, subtract, multiply, divide; each one rounding) of one MLP point of the
# exact walk, counted from find_MLP_path_GPU_tabulated (B.cu:9180-9244): Sigma_2 moments 9, its
# determinant 3 (plus a float powf), its inverse 3 divisions, the first term 11 and its determinant
# 3, each of the t and v solves 16, the rotation back 6, the three voxel indices 6, and the depth
# and position recurrences 2 -- 75 in all.  The per-history setup (about 1% of a path's work) is
# not counted.
FP64_OPS_PER_MLP_POINT = 75
UNIT = "histories/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--histories", type=int, default=50_000_000)
    ap.add_argument("--workload", choices=["head", "water", "batch", "learned", "precision", "preprocessing"],
                    default="head",
                    help="batch: 32 scans of different grids as one graph per iteration; learned: time to 1%% "
                         "RMSE from the learned vs the FBP start (neither is the headline)")
    ap.add_argument("--scans", type=int, default=32, help="batch workload: number of scans")
    ap.add_argument("--batch-block", type=int, default=3200,
                    help="batch workload: DROP_BLOCK_SIZE of every scan (HISTORIES_PER_BLOCK 640)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU-baseline sample time")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the secondary measurements (precomputed-path DROP, mixed precision)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default schedule (for profiling runs with a fixed launch shape)")
    return ap.parse_args()


def workload_params(name):
    if name == "head":
        return dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=10.0, SSD_V_SIZE=9.0,
                    T_BIN_SIZE=0.1, V_BIN_SIZE=0.25, ANGULAR_BIN_SIZE=4.0, DROP_BLOCK_SIZE=60000,
                    HISTORIES_PER_BLOCK=480, ITERATIONS=12, LAMBDA=0.0001)
    return dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=6.4, SSD_V_SIZE=5.0,
                T_BIN_SIZE=0.1, V_BIN_SIZE=0.25, ANGULAR_BIN_SIZE=4.0, DROP_BLOCK_SIZE=3200,
                HISTORIES_PER_BLOCK=640, ITERATIONS=6, LAMBDA=0.0001, MLP_U_STEP=0.1)


def workload_desc(name, n):
    if name == "head":
        return (f"head-size plain pipeline: 200x200x32 voxels (1x1x2.5 mm), head phantom, continuous angles, "
                f"{n} reconstruction histories, DROP blocks of 60000, MLP step 0.5 mm, one DROP iteration per step")
    return (f"small plain pipeline: 128x128x16 voxels (1x1x2.5 mm), water cylinder with 4 inserts, 90 angles, "
            f"{n} reconstruction histories, DROP blocks of 3200, MLP step 1 mm, one DROP iteration per step")


def generate(cfg, name, n, seed, device):
    """Seeded synthetic reconstruction histories (simulated MCS tracks through the phantom)."""
    import torch
    from pct_reconstruction_b200 import phantoms as P
    ph = P.head_phantom() if name == "head" else P.water_cylinder_phantom(6.0)
    kw = dict(continuous_angles=(name == "head"), t_extent=(20.0 if name == "head" else 18.0),
              v_extent=(7.0 if name == "head" else 4.0))
    parts, have, k = [], 0, 0
    while have < n:
        m = min(8_000_000, int((n - have) * 1.4) + 1000)
        tr = P.simulate_tracks(ph, m, seed=seed * 1000 + k, device=device, **kw)
        h = P.reconstruction_histories(cfg, tr)
        parts.append(h)
        have += len(h["WEPL"])
        k += 1
    out = {key: torch.cat([p[key] for p in parts])[:n].contiguous() for key in parts[0]}
    x0 = P.truth_image(cfg, ph, device=device)
    # start from a smoothed, biased version of the truth so the iteration has work to do
    x0 = (0.9 * x0 + 0.1).contiguous()
    return out, x0


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"pct_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.idx)], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if not self.proc or not self.path.exists():
            return None
        sm, mx, reasons, watts = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [s.strip() for s in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            try:
                watts.append(float(f[3]))
            except ValueError:
                pass
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_mhz_min": min(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "power_w_median": statistics.median(watts) if watts else None, "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


def profiled_traffic_per_history(kernel_name):
    """DRAM bytes per history of `kernel_name` from the committed ncu summary, if any."""
    p = ROOT / "profiles" / f"{kernel_name}.json"
    if not p.exists():
        return None
    try:
        return float(json.loads(p.read_text())["dram_bytes_per_history"])
    except Exception:
        return None


def profiled_fp64_pipe_pct(kernel_name):
    """FP64-pipe utilisation (%) of `kernel_name` from the committed ncu summary, if any."""
    p = ROOT / "profiles" / f"{kernel_name}.json"
    try:
        return float(json.loads(p.read_text())["fp64_pipe_pct"])
    except Exception:
        return None


def cpu_baseline(cfg, hist_cpu, x0_cpu, target_s, threads):
    """The reference's host MLP+DROP (O.cu restated in oracle/) on a bounded sample."""
    from oracle import Oracle
    o = Oracle(cfg.struct)
    n_all = len(hist_cpu["WEPL"])
    probe = min(n_all, 20000)
    sample = {k: v[:probe] for k, v in hist_cpu.items()}
    t0 = time.perf_counter()
    o.host_drop_iteration(sample, x0_cpu, threads=threads)
    dt = time.perf_counter() - t0
    m = int(min(n_all, max(probe, probe * target_s / max(dt, 1e-3))))
    sample = {k: v[:m] for k, v in hist_cpu.items()}
    t0 = time.perf_counter()
    o.host_drop_iteration(sample, x0_cpu, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": m / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"first {m} histories of the workload, one DROP iteration (blocks of {cfg.DROP_BLOCK_SIZE}), "
                      f"{dt:.1f} s on {threads} threads"}


def inputs_fingerprint(hist) -> str:
    """A cheap fingerprint of history arrays (device-side sums of the 32-bit patterns, plain and
    position-weighted), to recognise the exact inputs of an earlier run."""
    import torch
    parts = []
    for k in sorted(hist):
        a = hist[k].contiguous().view(torch.int32).to(torch.int64)
        w = torch.arange(a.numel(), device=a.device, dtype=torch.int64) % 1021 + 1
        parts.append(f"{int(a.sum().item()) & 0xffffffffffff:x}.{int((a * w).sum().item()) & 0xffffffffffff:x}")
    return "-".join(parts)


# Fingerprint of the head workload's 50M histories (generate(..., seed=replica_seed(1, 0)) on a
# B200), on which the engine's bounds counters (voxel_oob, path_overflow, table_range) were all 0:
# every voxel index of every MLP path lies inside the one-slice padded image.  The reference's
# kernels do not check their indices, so the reference-GPU leg runs only on these inputs.
HEAD_WORKLOAD_FINGERPRINT = (
    "28abac62b798.93e47478d9ea-1d1ab265a347.17db4b4b2e4e-734140462d67.9e60890e9cf8-6ce71adf1dbc.286c2244c73c-f08b6e154457.9fdf113e9635-9a3cca0b2aee.6ea1529ba306-a3fbc4cdbe86.c637599982c5-82d18ff25eb6.9c1b2e039e2d-3b749eebf269.41891022113a-3739cae27a5e.626ac77496d1-ef554cfbb541.30df2aee8dd1-ec7f0c9cd749.c132eac12a94")


def reference_gpu_leg(cfg, args):
    """The reference's own device code (B.cu compiled against a copy of B.h with the head grid,
    oracle/build_reference.py) timed on the full head workload: one DROP iteration per step as
    calculate_x_update_GPU + image_update_GPU do it (oracle/time_reference_gpu.py), CUDA events
    inside the harness, histories resident on the device."""
    import torch
    from oracle.time_reference_gpu import HARNESS, reference_gpu_iterations
    from pct_reconstruction_b200 import replicas
    if args.workload != "head" or not torch.cuda.is_available():
        return None
    if not HARNESS["head"].exists():
        return {"unavailable": f"{HARNESS['head'].relative_to(ROOT)} not built (oracle/build_reference.py)"}
    hist, x0 = generate(cfg, "head", args.histories, seed=replicas.replica_seed(1, 0), device="cuda")
    fp = inputs_fingerprint(hist)
    if fp != HEAD_WORKLOAD_FINGERPRINT:
        return {"skipped": "the regenerated inputs are not the ones whose voxel indices the engine's bounds counters "
                           "cleared (the reference's kernels do not check theirs)", "inputs_fingerprint": fp}
    n = len(hist["WEPL"])
    iters = 3
    ms, _ = reference_gpu_iterations("head", hist, x0.cpu().numpy(), cfg.DROP_BLOCK_SIZE, iters)
    best = float(np.min(ms))
    return {"value": n / (best / 1000.0), "unit": UNIT, "histories": n, "ms_per_iteration": [float(m) for m in ms],
            "what": "the reference's find_MLP_path_GPU_tabulated + DROP_block_update_GPU per DROP block and "
                    "image_update_GPU (B.cu:9321-9419), unmodified B.cu compiled for sm_100a with the head grid's "
                    "B.h values; CUDA events per iteration, best of 3"}


def run_reference(args):
    """--impl reference: the reference's host MLP+DROP (O.cu:4017, 7680-7711 restated in the
    oracle; O.cu does not compile on Linux) on all host cores, a bounded sample of whole DROP blocks
    per step.  The configuration is derived from B.h's values by oracle/refconfig.py, without the
    engine library.  The line adds, under reference_gpu, the reference's own device code timed on
    the full workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch
    from oracle import Oracle
    from oracle.refconfig import reference_config
    cfg = reference_config(**workload_params(args.workload))
    threads = os.cpu_count() or 1
    blocks = 4 if args.workload == "head" else 32
    sample_n = blocks * cfg.DROP_BLOCK_SIZE
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    hist, x0 = generate(cfg, args.workload, sample_n, seed=7, device=dev)
    hist = {k: v.cpu().numpy() for k, v in hist.items()}
    x0 = x0.cpu().numpy()
    o = Oracle(cfg.struct)
    for _ in range(args.warmup):
        o.host_drop_iteration(hist, x0, threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.host_drop_iteration(hist, x0, threads=threads)
        times.append(time.perf_counter() - t0)
    ms = 1000 * statistics.mean(times)
    value = sample_n / (ms / 1000)
    sample = (f"{sample_n} histories of the workload per step: {blocks} whole DROP blocks of {cfg.DROP_BLOCK_SIZE}, "
              f"one DROP iteration (O.cu's host MLP + DROP restated in oracle/), {threads} host threads")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": workload_desc(args.workload, args.histories), "sample": sample},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_gpu": reference_gpu_leg(cfg, args)}
    print(json.dumps(line), flush=True)


def secondary_measurements(cfg, ctx, hist, x0, stream, args):
    """Modes beside the headline, each timed over 3 iterations with CUDA events: precomputed-path
    DROP (paths computed by one iteration and kept; later iterations run the DROP blocks only --
    not an MLP+DROP iteration, so never the headline), the mixed-precision modes (with their
    accuracy against the exact path: voxel-list mismatches, MLP point deviation, image RMSE after 2
    iterations from the same start) and the exact mode with S_CURVE_ON."""
    import torch
    from pct_reconstruction_b200 import Config, Context
    n = len(hist["WEPL"])
    out = {}

    def timed(c, k=3):
        s0, e0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s0.record(stream)
        for i in range(k):
            c.DROP_full_tx_iteration(i + 1)
        e0.record(stream)
        torch.cuda.synchronize()
        return s0.elapsed_time(e0) / k

    ctx.set_reconstruction_histories(hist)
    ctx.x_host_2_GPU(x0)
    ctx.DROP_full_tx_iteration(1)
    ms_plain = timed(ctx)
    ctx.set_l2_window(True)
    ctx.DROP_full_tx_iteration(1)
    ms_window = timed(ctx)
    ctx.set_l2_window(False)
    out["l2_window"] = {"ms_per_iteration": ms_window, "ms_per_iteration_without": ms_plain,
                        "note": "image and accumulator in persisting L2 lines (pct_set_l2_window)"}
    ctx.x_host_2_GPU(x0)
    ctx.set_path_reuse(True)
    ctx.DROP_full_tx_iteration(1)
    ms = timed(ctx)
    ctx.set_path_reuse(False)
    out["precomputed_path_drop"] = {"ms_per_iteration": ms, "histories_per_s": n / (ms / 1000.0),
                                    "note": "MLP paths computed once and kept in HBM; DROP blocks only"}
    ctx.x_host_2_GPU(x0)
    for i in range(2):
        ctx.DROP_full_tx_iteration(i + 1)
    x_exact = ctx.x_GPU_2_host().astype(np.float64)
    m = Context(Config(**dict(workload_params(args.workload), PRECISION="MIXED")))
    try:
        m.set_stream(stream.cuda_stream)
        m.set_reconstruction_histories(hist)
        m.x_host_2_GPU(x0)
        for i in range(2):
            m.DROP_full_tx_iteration(i + 1)
        x_mixed = m.x_GPU_2_host().astype(np.float64)
        rmse = float(np.sqrt(np.mean((x_mixed - x_exact) ** 2)) / np.sqrt(np.mean(x_exact ** 2)))
        ms_m = timed(m)
        k = min(n, 1_000_000)
        dt, dv, mism, ill = m.mlp_precision(0, k)
        dev_mm = np.maximum(dt, dv) * 10.0
        prof = m.profile_drop_iteration()
        out["mixed_precision"] = {
            "ms_per_iteration": ms_m, "histories_per_s": n / (ms_m / 1000.0),
            "path_kernel_ms": prof["path"]["ms"],
            "image_rel_rmse_vs_exact_2_iterations": rmse,
            "sample_histories": k,
            "histories_with_differing_voxel_steps": float(np.mean(mism > 0)),
            "point_deviation_mm": {"p99": float(np.quantile(dev_mm, 0.99)), "p99.9": float(np.quantile(dev_mm, 0.999)),
                                   "max": float(dev_mm.max())},
            "histories_with_ill_conditioned_reference_steps": float(np.mean(ill > 0)),
            "note": "deviation over steps where the reference's Sigma_2 is well conditioned"}
    finally:
        m.close()
    # the mixed mode with the compensated per-voxel accumulation (a returning atomic and a second
    # reduction per path entry)
    mc = Context(Config(**dict(workload_params(args.workload), PRECISION="MIXED_COMPENSATED")))
    try:
        mc.set_stream(stream.cuda_stream)
        mc.set_reconstruction_histories(hist)
        mc.x_host_2_GPU(x0)
        for i in range(2):
            mc.DROP_full_tx_iteration(i + 1)
        x_mc = mc.x_GPU_2_host().astype(np.float64)
        rmse_mc = float(np.sqrt(np.mean((x_mc - x_exact) ** 2)) / np.sqrt(np.mean(x_exact ** 2)))
        ms_mc = timed(mc)
        out["mixed_compensated"] = {"ms_per_iteration": ms_mc, "histories_per_s": n / (ms_mc / 1000.0),
                                    "image_rel_rmse_vs_exact_2_iterations": rmse_mc}
    finally:
        mc.close()
    # the exact mode with the S-curve attenuation of the reference's S_CURVE_ON build (sigmoid,
    # dual-sided): a table read and three FP64 multiplies more per path entry in the block kernel
    block_ms_plain = ctx.profile_drop_iteration()["block"]["ms"]
    sc = Context(Config(**dict(workload_params(args.workload), S_CURVE_ON=1)))
    try:
        sc.set_stream(stream.cuda_stream)
        sc.set_reconstruction_histories(hist)
        sc.x_host_2_GPU(x0)
        sc.DROP_full_tx_iteration(1)
        ms_sc = timed(sc)
        out["s_curve"] = {"ms_per_iteration": ms_sc, "histories_per_s": n / (ms_sc / 1000.0),
                          "block_kernels_ms": sc.profile_drop_iteration()["block"]["ms"],
                          "block_kernels_ms_without": block_ms_plain,
                          "note": "S_CURVE_ON (sigmoid, dual-sided), against the exact iteration without it"}
    finally:
        sc.close()
    return out


WEIGHTS = ROOT / "pct_reconstruction_b200" / "weights" / "unet_200x200x32.bin"


PREPROCESSING_STAGES = ("recon_volume_intersections", "binning", "hull_detection", "hull_detection_finish",
                        "calculate_means", "sum_squared_deviations", "calculate_standard_deviations",
                        "statistical_cuts", "construct_sinogram", "FBP", "hull_selection", "define_initial_iterate",
                        "reconstruction_cuts")


def preprocessing_measurement(protons=20_000_000):
    """Per-stage wall time (device-synchronised) of preprocessing() for one head-phantom scan of
    `protons` simulated protons at the head grid (MSC and SM hulls, FBP), tracker data resident on
    the device; the second of two passes on one context, so first-use allocations are excluded."""
    import torch
    from pct_reconstruction_b200 import Config, Context
    from pct_reconstruction_b200 import learned as L
    from pct_reconstruction_b200 import phantoms as P
    dev = torch.device("cuda", 0)
    cfg = Config(**L.scan_config((200, 200, 32), 60000, 12))
    tr = P.simulate_tracks(P.head_phantom(), protons, seed=5, device=dev, continuous_angles=True,
                           t_extent=20.0, v_extent=7.0)
    td = P.tracker_data(tr)
    del tr
    out = {}
    with Context(cfg) as ctx:
        for rep in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.load_tracker_data(td)
            ctx.synchronize()
            times = {"load_tracker_data": (time.perf_counter() - t0) * 1e3}
            for st in PREPROCESSING_STAGES:
                t0 = time.perf_counter()
                ctx.stage(st)
                ctx.synchronize()
                times[st] = (time.perf_counter() - t0) * 1e3
        total = sum(times.values())
        out = {"protons": protons, "reconstruction_histories": ctx.reconstruction_histories,
               "total_ms": total, "protons_per_s": protons / (total / 1e3), "stage_ms": times}
    return out


def learned_start_measurement(n_scans=4, histories=20_000_000, tolerances=(0.01, 0.005)):
    """Time to tolerance, learned vs FBP start, on held-out random-ellipsoid phantoms at the head
    grid (200x200x32, 60000-history blocks, 12 iterations, 20M simulated protons per scan).  The
    reference image is the FBP-started DROP image after 12 iterations; per start: iterations and
    device-synchronised wall time until the relative RMSE inside the hull is within tolerance
    (the learned start includes the network call)."""
    import torch
    from pct_reconstruction_b200 import Config
    from pct_reconstruction_b200 import learned as L
    if not WEIGHTS.exists():
        return {"unavailable": f"no trained parameter file ({WEIGHTS.name})"}
    cfg = Config(**L.scan_config((200, 200, 32), 60000, 12))
    dev = torch.device("cuda", 0)
    rows, truths = [], []
    with L.UNet(cfg.COLUMNS, cfg.ROWS, cfg.SLICES) as net:
        net.load(WEIGHTS)
        for k in range(n_scans):
            ph, td = L.scan_phantom(cfg, 900_000 + k, histories, dev)  # training used seeds 1000 + i
            r = L.evaluate_scan(cfg, td, net, 12, 1.0)
            truths.append(L.evaluate_scan_truth(cfg, ph, td, net, 12))
            del td
            rows.append(r)

    def reach(r, tol, extra):
        k = next((i for i, e in enumerate(r["rel_rmse"]) if e <= tol), None)
        return (None, None) if k is None else (k, extra + float(sum(r["iteration_ms"][:k])))

    out = {"scans": n_scans, "histories_per_scan": histories, "reference": "FBP-started DROP image after 12 iterations",
           "start_rel_rmse": {"fbp": [r["fbp"]["rel_rmse"][0] for r in rows],
                              "learned": [r["learned"]["rel_rmse"][0] for r in rows]},
           "network_ms": statistics.median(r["learned"]["start_ms"] for r in rows),
           "drop_iteration_ms": statistics.median(t for r in rows for t in r["fbp"]["iteration_ms"]),
           "reconstruction_histories": [r["histories"] for r in rows]}
    for tol in tolerances:
        f = [reach(r["fbp"], tol, 0.0) for r in rows]
        g = [reach(r["learned"], tol, r["learned"]["start_ms"]) for r in rows]
        key = f"to_{tol * 100:g}pct"
        out[key] = {"fbp_iterations": [a for a, _ in f], "learned_iterations": [a for a, _ in g],
                    "fbp_ms": [b for _, b in f], "learned_ms": [b for _, b in g]}
        ok = [(a[1], b[1]) for a, b in zip(f, g) if a[1] is not None and b[1] is not None]
        out[key]["median_wall_time_ratio_fbp_over_learned"] = (
            statistics.median(a / b for a, b in ok) if ok else None)
    # against the phantom's true RSP (not the network's training target): time to the larger of
    # the two starts' best errors, which both reach, and both starts' error after 12 iterations
    out["truth"] = {
        "metric": "relative RMSE to the phantom's true RSP inside the hull",
        "common_level": [t["common_level"] for t in truths],
        "start_rel_rmse": {"fbp": [t["fbp"]["rel_rmse_to_truth"][0] for t in truths],
                           "learned": [t["learned"]["rel_rmse_to_truth"][0] for t in truths]},
        "final_rel_rmse_12_iterations": {"fbp": [t["fbp"]["final_rel_rmse_to_truth"] for t in truths],
                                         "learned": [t["learned"]["final_rel_rmse_to_truth"] for t in truths]},
        "iterations_to_level": {"fbp": [t["fbp"]["iterations_to_level"] for t in truths],
                                "learned": [t["learned"]["iterations_to_level"] for t in truths]},
        "ms_to_level": {"fbp": [t["fbp"]["ms_to_level"] for t in truths],
                        "learned": [t["learned"]["ms_to_level"] for t in truths]},
        "median_wall_time_ratio_fbp_over_learned": statistics.median(
            t["fbp"]["ms_to_level"] / max(t["learned"]["ms_to_level"], 1e-9) for t in truths)}
    return out


def batch_scans(n_scans, seed, device, block_size=3200):
    """Seeded batch workload: grids from 64x64x8 to 256x256x48 (1x1x2.5 mm voxels), random
    ellipsoid-union phantoms (RSP of the inserts uniform in [0.2, 1.8]), continuous angles, and
    history counts log-uniform in [0.5M, 8M]."""
    from pct_reconstruction_b200 import Config
    from pct_reconstruction_b200 import phantoms as P
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_scans):
        cols = int(rng.choice([64, 96, 128, 160, 200, 256]))
        slices = int(rng.integers(8, 49))
        R = cols * 0.05
        params = dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=R,
                      SSD_V_SIZE=slices * 0.25 + 1.0, T_BIN_SIZE=0.1, V_BIN_SIZE=0.25, ANGULAR_BIN_SIZE=4.0,
                      DROP_BLOCK_SIZE=block_size, HISTORIES_PER_BLOCK=640, LAMBDA=0.0001)
        cfg = Config(**params)
        ph = P.random_ellipsoid_phantom(seed * 100 + i, extent=(0.8 * R, 0.8 * R, 0.4 * cfg.RECON_CYL_HEIGHT))
        n = int(np.exp(rng.uniform(np.log(0.5e6), np.log(8e6))))
        parts, have, k = [], 0, 0
        while have < n:
            tr = P.simulate_tracks(ph, min(8_000_000, int((n - have) * 1.6) + 1000), seed=seed * 1000 + i * 10 + k,
                                   device=device, continuous_angles=True, t_extent=2.2 * R,
                                   v_extent=0.9 * cfg.RECON_CYL_HEIGHT)
            h = P.reconstruction_histories(cfg, tr)
            parts.append(h)
            have += len(h["WEPL"])
            k += 1
        import torch
        hist = {key: torch.cat([p_[key] for p_ in parts])[:n].contiguous() for key in parts[0]}
        x0 = (0.9 * P.truth_image(cfg, ph, device=device) + 0.1).contiguous()
        out.append((params, hist, x0))
    return out


def batch_main(args):
    """Batched scans: aggregate histories/s of one graph launch per iteration for all scans, next to
    the same scans iterated one at a time, and each scan's image RMSE against its one-at-a-time run."""
    import torch
    from pct_reconstruction_b200 import Batch, Config, Context
    dev = torch.device("cuda", 0)
    scans = batch_scans(args.scans, seed=3, device=dev, block_size=args.batch_block)
    total = sum(len(h["WEPL"]) for _, h, _ in scans)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    # one at a time: each scan's iteration alone, timed on its own stream
    alone_ms, alone_img, path_ms, chain_ms = [], [], [], []
    for params, hist, x0 in scans:
        c = Context(Config(**params))
        c.set_stream(stream.cuda_stream)
        c.set_reconstruction_histories(hist)
        c.x_host_2_GPU(x0)
        c.autotune()
        for i in range(args.warmup):
            c.DROP_full_tx_iteration(i + 1)
        c.x_host_2_GPU(x0)
        c.DROP_full_tx_iteration(1)  # the image after one iteration from x0
        torch.cuda.synchronize()
        alone_img.append(c.x_GPU_2_host())
        a, b = ev(), ev()
        a.record(stream)
        for i in range(args.steps):
            c.DROP_full_tx_iteration(i + 2)
        b.record(stream)
        torch.cuda.synchronize()
        alone_ms.append(a.elapsed_time(b) / args.steps)
        prof = c.profile_drop_iteration()  # each launch alone, serialised, with CUDA events
        path_ms.append(prof["path"]["ms"])
        chain_ms.append(prof["block"]["ms"] + prof["update"]["ms"])
        c.close()
    # batched: all scans, one graph per iteration
    ctxs, chosen = [], []
    for params, hist, x0 in scans:
        c = Context(Config(**params))
        c.set_reconstruction_histories(hist)
        c.x_host_2_GPU(x0)
        chosen.append(c.autotune_schedule())  # each scan's schedule, by measurement
        ctxs.append(c)
    b = Batch(ctxs)
    bstream = torch.cuda.ExternalStream(b.stream)
    for i in range(args.warmup):
        b.DROP_iteration(i + 1)
    b.synchronize()
    for c, (_, _, x0) in zip(ctxs, scans):
        c.x_host_2_GPU(x0)
    b.DROP_iteration(1)
    b.synchronize()
    rmse = []
    for c, ref in zip(ctxs, alone_img):
        g = c.x_GPU_2_host().astype(np.float64)
        rmse.append(float(np.sqrt(np.mean((g - ref) ** 2)) / np.sqrt(np.mean(ref.astype(np.float64) ** 2))))
    launches0 = sum(c.kernel_launches for c in ctxs)
    with ClockSampler(0) as clocks:
        a, e = ev(), ev()
        a.record(bstream)
        for i in range(args.steps):
            b.DROP_iteration(i + 2)
        e.record(bstream)
        b.synchronize()
        torch.cuda.synchronize()
    ms = a.elapsed_time(e) / args.steps
    launches = sum(c.kernel_launches for c in ctxs) - launches0
    b.close()
    for c in ctxs:
        c.close()
    grids = [f"{Config(**p).COLUMNS}x{Config(**p).ROWS}x{Config(**p).SLICES}:{len(h['WEPL'])}" for p, h, _ in scans]
    print(json.dumps({
        "metric": "batched MLP+DROP histories/s/iter on 1 B200 (all scans)", "value": total / (ms / 1000.0),
        "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{len(scans)} scans, random ellipsoid unions, continuous angles, "
                               f"{total} histories in all, DROP blocks of {args.batch_block}", "scans": grids},
        "one_at_a_time": {"ms_per_iteration_sum": float(sum(alone_ms)),
                          "histories_per_s": total / (sum(alone_ms) / 1000.0)},
        "speedup_vs_one_at_a_time": float(sum(alone_ms) / ms),
        # every kernel of every scan's iteration launched alone, back to back: the path kernels
        # (x-independent, FP64-bound) and the DROP block and image-update kernels (L2-bound); a path
        # CTA fills an SM's register file, so the two kinds share SMs only at kernel edges and a batch
        # iteration is not expected to be much shorter than their sum
        "path_kernels_ms_sum": float(sum(path_ms)), "block_and_update_kernels_ms_sum": float(sum(chain_ms)),
        "kernels_ms_sum": float(sum(path_ms) + sum(chain_ms)),
        "batch_over_kernel_sum": float(ms / (sum(path_ms) + sum(chain_ms))),
        "per_scan_image_rel_rmse_vs_one_at_a_time": {"max": max(rmse), "mean": float(np.mean(rmse))},
        "autotuned_schedules": chosen,
        "gpu_launches": launches, "clocks": clocks.summary()}), flush=True)


def precision_main(args):
    """--workload precision: the precision study on the small configuration's inputs (128x128x16,
    water cylinder with four inserts, 1 mm MLP step, blocks of 3200, 6 iterations) at 10M
    histories.  The FP64 reference is the exact mode (bit-identical voxel lists to the reference's
    FP64 device code); against it: the mixed-precision MLP's point deviation (mm, over the steps
    where the reference's Sigma_2 is well conditioned), histories whose voxel lists differ, and the
    relative RSP RMSE after 6 iterations for mixed/exact x atomic/deterministic scatter, with the
    atomic mode's own run-to-run RMSE as the floor."""
    import torch
    from pct_reconstruction_b200 import Config, Context
    from pct_reconstruction_b200 import replicas
    rank, _, world = replicas.world()
    if rank != 0:
        return
    dev = torch.device("cuda", 0)
    n_hist = args.histories if args.histories != 50_000_000 else 10_000_000
    base = workload_params("water")
    cfg0 = Config(**base)
    hist, x0 = generate(cfg0, "water", n_hist, seed=7, device=dev)
    n = len(hist["WEPL"])
    iters = cfg0.ITERATIONS
    images, times, kernel_ms = {}, {}, {}

    def run(precision, scatter, key):
        c = Config(**dict(base, PRECISION=precision, SCATTER_MODE=scatter))
        with Context(c) as ctx:
            ctx.set_reconstruction_histories(hist)
            ctx.x_host_2_GPU(x0)
            ctx.DROP_full_tx_iteration(1)  # builds the layout and the graph
            ctx.x_host_2_GPU(x0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for it in range(1, iters + 1):
                ctx.DROP_full_tx_iteration(it)
            ctx.synchronize()
            times[key] = (time.perf_counter() - t0) * 1e3 / iters
            images[key] = ctx.x_GPU_2_host().astype(np.float64)
            # one more iteration, each launch timed alone: the path kernels (MLP) and the DROP block
            # kernels (gather, update value, scatter) apart
            prof = ctx.profile_drop_iteration()
            kernel_ms[key] = {"path": prof["path"]["ms"], "drop_blocks": prof["block"]["ms"],
                              "image_updates": prof["update"]["ms"]}
            if precision == "MIXED" and scatter == "ATOMIC":
                dmax, mism_h, ill_h, steps_dev = 0.0, 0, 0, []
                for s0 in range(0, n, 2_000_000):
                    k = min(2_000_000, n - s0)
                    dt, dv, mm, ip = ctx.mlp_precision(s0, k)
                    d = np.maximum(dt, dv) * 10.0
                    dmax = max(dmax, float(d.max()))
                    mism_h += int((mm > 0).sum())
                    ill_h += int((ip > 0).sum())
                    steps_dev.append(d)
                d = np.concatenate(steps_dev)
                return {"max_point_deviation_mm": dmax, "p99_point_deviation_mm": float(np.quantile(d, 0.99)),
                        "p999_point_deviation_mm": float(np.quantile(d, 0.999)),
                        "histories_with_differing_voxel_lists": mism_h / n,
                        "histories_with_ill_conditioned_reference_steps": ill_h / n}
        return None

    with ClockSampler(0) as clocks:
        run("EXACT", "DETERMINISTIC", "exact_det")
        run("EXACT", "DETERMINISTIC", "exact_det_again")
        run("EXACT", "ATOMIC", "exact_atomic")
        run("EXACT", "ATOMIC", "exact_atomic_again")
        mlp = run("MIXED", "ATOMIC", "mixed_atomic")
        run("MIXED_COMPENSATED", "ATOMIC", "mixed_compensated_atomic")
        run("MIXED", "DETERMINISTIC", "mixed_det")
    ref = images["exact_det"]
    rel = lambda a: float(np.sqrt(np.mean((a - ref) ** 2)) / np.sqrt(np.mean(ref ** 2)))  # noqa: E731
    line = {"metric": "precision study: MLP path deviation and RSP RMSE against the FP64 (exact) mode",
            "value": rel(images["mixed_atomic"]), "unit": "relative RSP RMSE after 6 iterations (mixed, atomic)",
            "n_gpus": 1, "steps": iters, "warmup": 1, "ms_per_step": times["mixed_atomic"], "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64/f32", "data": "synthetic",
            "config": {"workload": f"small plain pipeline inputs: 128x128x16 voxels, water cylinder with 4 inserts, "
                                   f"{n} reconstruction histories, 1 mm MLP step, blocks of 3200, {iters} iterations"},
            "mlp": mlp,
            "rel_rmse_vs_exact_deterministic": {
                "exact_deterministic_rerun": rel(images["exact_det_again"]),
                "exact_atomic": rel(images["exact_atomic"]),
                "exact_atomic_rerun_vs_exact_atomic": float(
                    np.sqrt(np.mean((images["exact_atomic_again"] - images["exact_atomic"]) ** 2)) / np.sqrt(np.mean(ref ** 2))),
                "mixed_atomic": rel(images["mixed_atomic"]),
                "mixed_compensated_atomic": rel(images["mixed_compensated_atomic"]),
                "mixed_deterministic": rel(images["mixed_det"])},
            "ms_per_iteration": times, "kernel_ms_per_iteration": kernel_ms, "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)


def preprocessing_main(args):
    """--workload preprocessing: per-stage wall time of preprocessing() for one head-phantom scan
    (protons = --histories, default 20M) at the head grid; one line (rank 0)."""
    from pct_reconstruction_b200 import replicas
    rank, _, _ = replicas.world()
    if rank != 0:
        return
    protons = args.histories if args.histories != 50_000_000 else 20_000_000
    with ClockSampler(0) as clocks:
        r = preprocessing_measurement(protons)
    print(json.dumps({"metric": "preprocessing protons/s on 1 B200 (head grid, one scan)", "value": r["protons_per_s"],
                      "unit": "protons/s", "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": r["total_ms"],
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64/f32",
                      "data": "synthetic", "config": {"workload": f"head phantom, {protons} simulated protons, "
                                                                  "200x200x32, MSC and SM hulls, FBP"},
                      "preprocessing": r, "clocks": clocks.summary()}), flush=True)


def learned_main(args):
    """--workload learned: time to within 1% relative RMSE of the FBP-started 12-iteration image,
    learned start vs FBP start, median over held-out phantoms (one line, rank 0; replicas only)."""
    from pct_reconstruction_b200 import replicas
    rank, _, world = replicas.world()
    if rank != 0:
        return
    with ClockSampler(0) as clocks:
        r = learned_start_measurement(n_scans=max(args.steps, 1))
    if "unavailable" in r:
        print(json.dumps({"metric": "time to 1% RSP RMSE, learned vs FBP start", **r}), flush=True)
        return
    t = r["to_1pct"]
    learned_ms = statistics.median(x for x in t["learned_ms"] if x is not None)
    line = {"metric": "time to 1% RSP RMSE, learned start (DROP reference image: FBP start, 12 iterations)",
            "value": learned_ms, "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": 0,
            "ms_per_step": learned_ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16", "data": "synthetic",
            "config": {"workload": "learned DROP initializer: 200x200x32 voxels, random-ellipsoid phantoms, "
                                   "20M simulated protons per scan, 60000-history blocks, 12 iterations",
                       "fbp_start_ms_median": statistics.median(x for x in t["fbp_ms"] if x is not None)},
            "learned_start": r, "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "batch":
        batch_main(args)
        return
    if args.workload == "learned":
        learned_main(args)
        return
    if args.workload == "precision":
        precision_main(args)
        return
    if args.workload == "preprocessing":
        preprocessing_main(args)
        return
    import torch
    import torch.distributed as dist
    from pct_reconstruction_b200 import Config, Context

    from pct_reconstruction_b200 import replicas
    rank, local, world = replicas.world()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local)

    def barrier():
        if world > 1:
            dist.barrier()

    cfg = Config(**workload_params(args.workload))
    hist, x0 = generate(cfg, args.workload, args.histories, seed=replicas.replica_seed(1, rank), device=dev)
    n = len(hist["WEPL"])
    fingerprint = inputs_fingerprint(hist)
    ctx = Context(cfg, device=local)
    # A dedicated (non-default) stream shared by the engine and the timing events.
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    torch.cuda.synchronize()
    ctx.set_reconstruction_histories(hist)
    ctx.x_host_2_GPU(x0)
    # the schedule (path-kernel chunking, histories per CTA, order window) chosen by measurement
    # (setup, not timed)
    schedule = None if args.no_autotune else ctx.autotune_schedule()

    # ---- warm-up (also captures the iteration graph) ----
    for i in range(args.warmup):
        ctx.DROP_full_tx_iteration(i + 1)
    torch.cuda.synchronize()

    # ---- timed region: K DROP iterations, inputs resident in HBM ----
    launches0 = ctx.kernel_launches
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        barrier()
        torch.cuda.synchronize()
        start.record(stream)
        for i in range(args.steps):
            ctx.DROP_full_tx_iteration(args.warmup + i + 1)
        end.record(stream)
        torch.cuda.synchronize()
        barrier()
    gpu_launches = ctx.kernel_launches - launches0
    value, ms_step = replicas.aggregate_throughput(n, start.elapsed_time(end) / args.steps, device=dev)
    counters = ctx.counters()

    # ---- roofline of the dominant kernel: one more iteration launched kernel by kernel, with CUDA
    #      events around every launch on the context stream (recorded by the engine) ----
    counts = torch.zeros(n, dtype=torch.int32, device=dev)
    ctx.mlp_paths_device(0, n, 0, counts, None, None, None)
    torch.cuda.synchronize()
    cnt = counts.to(torch.int64)
    B, hpb = cfg.DROP_BLOCK_SIZE, cfg.HISTORIES_PER_BLOCK
    covered = torch.zeros(n, dtype=torch.bool, device=dev)
    for s0 in range(0, n, B):
        hp = min(B, n - s0)
        cov = (hp // hpb) * hpb if hpb > 0 else hp
        covered[s0:s0 + cov] = True
    c = cnt[covered]
    scat = c * (c >= cfg.MIN_MLP_LENGTH)
    n_cov, sum_n, sum_scat = int(covered.sum().item()), float(c.sum().item()), float(scat.sum().item())
    prof = ctx.profile_drop_iteration()
    torch.cuda.synchronize()
    two_phase = prof["path"]["launches"] > 0
    # algorithmic bytes: path kernel reads 48 B of history data and writes the voxel list (4 B per
    # entry) plus its length and chord (12 B); block kernel reads the list back, gathers x (4 B per
    # entry), scatters {x_update, S} (8 B per entry) and reads WEPL/offset/length/chord (24 B)
    path_bytes = 48.0 * n_cov + 4.0 * sum_n + 12.0 * n_cov
    block_bytes = 8.0 * sum_n + 8.0 * sum_scat + 24.0 * n_cov
    if not two_phase:  # fused kernel: inputs + gather + scatter
        block_bytes = 48.0 * n_cov + 4.0 * sum_n + 8.0 * sum_scat
    groups = {"path": path_bytes, "block": block_bytes}
    dom = max((g for g in groups if prof[g]["launches"] > 0), key=lambda g: prof[g]["ms"])
    avg_ms = prof[dom]["ms"] / prof[dom]["launches"]
    bytes_per_launch = groups[dom] / prof[dom]["launches"]
    peaks, peak_kind = measured_peaks()
    achieved = bytes_per_launch / (avg_ms / 1000.0) / 1e9
    kernel_name = {"path": "mlp_phase1_exact_kernel", "block": ("drop_phase2_kernel" if two_phase
                                                               else "drop_block_exact_kernel")}[dom]
    tph = profiled_traffic_per_history(kernel_name)
    hbm = {"achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
           "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)", "algorithmic_bytes_per_launch": bytes_per_launch}
    if dom == "path":
        # the path kernel is bound by FP64 issue: its algorithmic work is FP64_OPS_PER_MLP_POINT
        # operations per MLP point (loop trip), counted by pct_mlp_steps; the peak is this GPU's FP64
        # FMA issue rate measured now (pct_fp64_fma_rate), one operation per instruction, because
        # the exact mode keeps every multiply and add separately rounded (no contraction)
        trips = torch.zeros(n, dtype=torch.int32, device=dev)
        ctx.mlp_steps_device(0, n, trips)
        sum_trips = float(trips[covered].to(torch.int64).sum().item())
        rate = C.c_double(0.0)
        st = ctx.lib.pct_fp64_fma_rate(local, C.byref(rate))
        peak_tops = rate.value / 1e12 if st == 0 else None
        ops_per_launch = FP64_OPS_PER_MLP_POINT * sum_trips / prof[dom]["launches"]
        achieved_tops = ops_per_launch / (avg_ms / 1000.0) / 1e12
        roofline = {"bound": "fp64", "achieved": achieved_tops, "peak": peak_tops, "unit": "TFLOP/s",
                    "frac": (achieved_tops / peak_tops) if peak_tops else None,
                    "traffic": (tph * n_cov / prof[dom]["launches"] if tph else None),
                    "kernel": kernel_name,
                    "peak_source": "measured in this run: FP64 FMA instructions/s of all SMs (pct_fp64_fma_rate), one "
                                   "operation per instruction; MEASURED_PEAKS.json holds no FP64 figure",
                    "peak_fma_2flop_tflops": 2 * peak_tops if peak_tops else None,
                    "algorithmic_fp64_ops_per_launch": ops_per_launch,
                    "fp64_ops_per_mlp_point": FP64_OPS_PER_MLP_POINT,
                    "mlp_points_per_history": sum_trips / max(n_cov, 1),
                    "kernel_ms_avg": avg_ms, "launches": prof[dom]["launches"],
                    "mean_path_voxels": sum_n / max(n_cov, 1),
                    "iteration_breakdown_ms": {g: prof[g]["ms"] for g in prof},
                    "fp64_pipe_pct_profiled": profiled_fp64_pipe_pct(kernel_name),
                    "hbm": hbm}
    else:
        roofline = {"bound": "hbm", **hbm, "traffic": (tph * n_cov / prof[dom]["launches"] if tph else None),
                    "kernel": kernel_name, "kernel_ms_avg": avg_ms, "launches": prof[dom]["launches"],
                    "mean_path_voxels": sum_n / max(n_cov, 1),
                    "iteration_breakdown_ms": {g: prof[g]["ms"] for g in prof}}

    # ---- e2e: same metric through the C ABI with host buffers (H2D of the histories and D2H of
    #      the image inside the timed region) ----
    e2e = None
    if not args.no_e2e:
        host = {k: v.cpu().pin_memory() for k, v in hist.items()}
        x_host = np.empty(cfg.NUM_VOXELS, np.float32)
        h2d = sum(v.numel() * v.element_size() for v in host.values())
        d2h = x_host.nbytes
        ctx.set_reconstruction_histories(host)
        ctx.DROP_full_tx_iteration(1)
        ctx.x_GPU_2_host()
        k_e2e = max(1, args.steps)
        barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as e2e_clocks:
            s1, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s1.record(stream)
            # every step's histories go host -> device inside the timed region; step i+1's upload
            # runs on the copy stream while step i reconstructs (pct_stage_reconstruction_histories)
            ctx.stage_reconstruction_histories(host)
            for i in range(k_e2e):
                ctx.use_staged_histories()
                if i + 1 < k_e2e:
                    ctx.stage_reconstruction_histories(host)
                ctx.DROP_full_tx_iteration(i + 1)
                x_host = ctx.x_GPU_2_host()
            e1.record(stream)
            torch.cuda.synchronize()
        barrier()
        e2e_value, e2e_ms = replicas.aggregate_throughput(n, s1.elapsed_time(e1) / k_e2e, device=dev)
        e2e = {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": e2e_ms, "steps": k_e2e,
               "upload": "each step's 2.4 GB of histories from pinned host memory; step i+1's upload runs on a copy "
                         "stream during step i (the first step's does not overlap)",
               "clocks": e2e_clocks.summary()}

    # ---- secondary measurements (not the headline): precomputed-path DROP and mixed precision ----
    extras = None
    if world == 1 and not args.no_extras:
        extras = secondary_measurements(cfg, ctx, hist, x0, stream, args)
        extras["learned_start"] = learned_start_measurement(n_scans=2)
        extras["preprocessing"] = preprocessing_measurement()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        hist_cpu = {k: v[:12_000_000].cpu().numpy() for k, v in hist.items()}
        cpu = cpu_baseline(cfg, hist_cpu, x0.cpu().numpy(), args.cpu_seconds, os.cpu_count() or 1)
        # the sequential reference's own setting: one host thread, on a shorter sample
        one = cpu_baseline(cfg, hist_cpu, x0.cpu().numpy(), args.cpu_seconds / 2, 1)
        cpu["single_core"] = {"value": one["value"], "cores": 1, "sample": one["sample"]}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": workload_desc(args.workload, n), "histories_per_rank": n,
                           "grid": f"{cfg.COLUMNS}x{cfg.ROWS}x{cfg.SLICES}", "drop_block_size": B,
                           "histories_per_block": hpb, "mlp_u_step_cm": cfg.MLP_U_STEP, "precision": "exact",
                           "l2": "inputs (history arrays) larger than L2; no flush",
                           "parallelism": f"replicas x{world}",
                           "mode": "two-phase (stored paths)" if two_phase else "single-pass",
                           "schedule": schedule or "defaults", "inputs_fingerprint": fingerprint},
                "e2e": e2e, "gpu_launches": gpu_launches, "roofline": roofline, "cpu_baseline": cpu,
                "clocks": clocks.summary(), "counters": counters, "secondary": extras}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
