"""Seeded inputs shared by the fixture generator (make_reference_fixtures.py) and the tests.

Inputs too large to store in a fixture are regenerated from a seed on cuda:0 (a B200 with the same
torch build in both places), and the fixture keeps their SHA-256 so that a test can tell a
regeneration mismatch from a parity failure.
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

HIST = ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit", "xy_entry_angle", "xz_entry_angle",
        "xy_exit_angle", "xz_exit_angle", "WEPL", "first_MLP_voxel")
GEOM6 = ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit")

# The head-size grid of the reference harness built from a patched B.h (oracle/build_reference.py,
# configuration "head"): 200 x 200 x 32 voxels of 0.1 x 0.1 x 0.25 cm, R = 10 cm, SSD_V_SIZE 9 cm,
# MLP_U_STEP = VOXEL_WIDTH / 2, DROP blocks of 60000, HISTORIES_PER_BLOCK 480; every other
# parameter at its B.h value.
HEAD = dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, RECON_CYL_RADIUS=10.0, DROP_BLOCK_SIZE=60000, HISTORIES_PER_BLOCK=480)


def sha256_of(arrays: dict, names=HIST) -> np.ndarray:
    h = hashlib.sha256()
    for k in names:
        h.update(np.ascontiguousarray(arrays[k]).tobytes())
    return np.frombuffer(h.digest(), np.uint8)


def default_image(nv: int) -> np.ndarray:
    """Deterministic non-uniform image used as x_0 by the MLP and DROP fixtures."""
    i = np.arange(nv, dtype=np.uint64)
    return (0.5 + ((i * np.uint64(2654435761)) % np.uint64(1000)).astype(np.float64) / 1000.0).astype(np.float32)


def head_histories(cfg, n: int, seed: int, device="cuda") -> dict:
    """n reconstruction histories of the head phantom at the head grid (continuous angles), as
    numpy arrays (first_MLP_voxel as uint32)."""
    import torch
    from pct_reconstruction_b200 import phantoms as P
    parts, have, k = [], 0, 0
    while have < n:
        tr = P.simulate_tracks(P.head_phantom(), int((n - have) * 1.4) + 1000, seed=seed * 100 + k, device=device,
                               continuous_angles=True, t_extent=20.0, v_extent=7.0)
        h = P.reconstruction_histories(cfg, tr)
        parts.append(h)
        have += len(h["WEPL"])
        k += 1
    out = {key: torch.cat([p[key] for p in parts])[:n].cpu().numpy() for key in parts[0]}
    out["first_MLP_voxel"] = out["first_MLP_voxel"].view(np.uint32)
    return out


def head_tracker_data(n: int, seed: int, device="cuda") -> dict:
    """Tracker hits of n simulated head-phantom protons at 90 gantry angles 4 degrees apart (the
    integer-angle intersection path of the reference), numpy arrays; gantry_angle as int32."""
    from pct_reconstruction_b200 import phantoms as P
    tr = P.simulate_tracks(P.head_phantom(), n, seed=seed, device=device, continuous_angles=False,
                           angle_interval_deg=4.0, t_extent=20.0, v_extent=7.0)
    td = {k: v.cpu().numpy() for k, v in P.tracker_data(tr).items()}
    td["gantry_angle"] = np.rint(td["gantry_angle"]).astype(np.int32)
    return td
