"""Train the learned DROP initializer on pairs made by the plain pipeline, then evaluate it.

    python -m pct_reconstruction_b200.train_initializer --pairs 1000 --steps 12000 --eval 100 \\
        --out pct_reconstruction_b200/weights/unet_200x200x32.bin --summary summary.json
    python -m pct_reconstruction_b200.train_initializer --params <file> --eval 100   # evaluation only

Each training pair is one seeded random-ellipsoid phantom (RSP of the inserts uniform in
[0.2, 1.8]) scanned with `--histories` simulated protons at continuous gantry angles, preprocessed
by the engine (binning, cuts, FBP, MSC/SM hull, x_0 = FBP_median x hull) and reconstructed by
`--iterations` DROP iterations from x_0: the network learns (x_0, hull) -> that image.  Held-out
phantoms (other seeds) are then reconstructed from both starts, and the iterations and wall time
each start needs to come within `--tolerance` relative RMSE (inside the hull) of the FBP-started
image are reported.  Because that image is also the network's training target, each held-out
phantom is evaluated a second time against its true RSP (learned.evaluate_scan_truth): both
starts' error to the truth after every iteration, and the time each needs to reach the larger of
their two best errors (a level both reach).  Everything runs on one GPU through libpct_b200.so.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--grid", type=int, nargs=3, default=(200, 200, 32), metavar=("COLUMNS", "ROWS", "SLICES"))
    ap.add_argument("--pairs", type=int, default=1000)
    ap.add_argument("--histories", type=int, default=20_000_000, help="simulated protons per scan")
    ap.add_argument("--iterations", type=int, default=12)
    ap.add_argument("--block", type=int, default=60000, help="DROP_BLOCK_SIZE")
    ap.add_argument("--steps", type=int, default=12000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--eval", type=int, default=16, help="held-out phantoms")
    ap.add_argument("--tolerance", type=float, default=0.01)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None, help="parameter file to write")
    ap.add_argument("--params", default=None, help="evaluate this parameter file instead of training")
    ap.add_argument("--summary", default=None, help="JSON summary to write")
    args = ap.parse_args(argv)

    import torch
    from . import Config
    from . import learned as L
    dev = torch.device("cuda", 0)
    cfg = Config(**L.scan_config(tuple(args.grid), args.block, args.iterations))
    log = lambda m: print(m, flush=True)  # noqa: E731
    net = L.UNet(cfg.COLUMNS, cfg.ROWS, cfg.SLICES, seed=args.seed)
    losses, t_data, t_train = [float("nan")], 0.0, 0.0
    if args.params:
        net.load(args.params)
        args.pairs = args.steps = 0
    else:
        t0 = time.time()
        pairs = [L.make_pair(cfg, 1000 + k, args.histories, args.iterations, dev) for k in range(args.pairs)]
        torch.cuda.synchronize()
        t_data = time.time() - t0
        log(f"{len(pairs)} pairs in {t_data:.1f} s")
        t0 = time.time()
        losses = L.train(net, pairs, args.steps, lr=args.lr, seed=args.seed, log=log)
        torch.cuda.synchronize()
        t_train = time.time() - t0
        del pairs
    if args.out:
        net.save(args.out)
    evals, truths = [], []
    for k in range(args.eval):
        ph, td = L.scan_phantom(cfg, 900_000 + k, args.histories, dev)
        r = L.evaluate_scan(cfg, td, net, args.iterations, args.tolerance)
        t = L.evaluate_scan_truth(cfg, ph, td, net, args.iterations)
        del td
        evals.append(r)
        truths.append(t)
        log(f"held-out {k}: fbp {r['fbp']['iterations_to_tolerance']} it / {r['fbp']['ms_to_tolerance']} ms, "
            f"learned {r['learned']['iterations_to_tolerance']} it / {r['learned']['ms_to_tolerance']} ms, "
            f"start error fbp {r['fbp']['rel_rmse'][0]:.4f} learned {r['learned']['rel_rmse'][0]:.4f}; "
            f"to truth: level {t['common_level']:.4f}, fbp {t['fbp']['iterations_to_level']} it / "
            f"{t['fbp']['ms_to_level']:.1f} ms, learned {t['learned']['iterations_to_level']} it / "
            f"{t['learned']['ms_to_level']:.1f} ms, final fbp {t['fbp']['final_rel_rmse_to_truth']:.4f} "
            f"learned {t['learned']['final_rel_rmse_to_truth']:.4f}")
    summary = {
        "grid": list(args.grid), "pairs": args.pairs, "histories_per_scan": args.histories,
        "iterations": args.iterations, "steps": args.steps, "data_seconds": t_data, "train_seconds": t_train,
        "train_ms_per_step": 1e3 * t_train / max(args.steps, 1),
        "loss_first_100": float(np.mean(losses[:100])), "loss_last_100": float(np.mean(losses[-100:])),
        "tolerance": args.tolerance, "eval": evals, "eval_truth": truths,
    }
    if args.summary:
        with open(args.summary, "w") as f:
            json.dump(summary, f)
    net.close()
    return summary


if __name__ == "__main__":
    main()
