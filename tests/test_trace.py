"""PCT_TRACE: one stderr line per DROP iteration from pct_drop_full_tx_iteration (GPU).

With PCT_TRACE set when the context is created, each iteration reports whether the path layout was
built or kept and the iteration graph captured or reused, with their host times.  The first
iteration after new histories builds both; a second iteration on the same histories keeps the layout
and reuses the graph; new histories of the same count rebuild the layout but keep the graph.
"""
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

SCRIPT = r"""
import numpy as np
from pct_reconstruction_b200 import Config, Context
from pct_reconstruction_b200 import phantoms as P
cfg = Config(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=6.4, SSD_V_SIZE=5.0,
             DROP_BLOCK_SIZE=1000, HISTORIES_PER_BLOCK=0, MLP_U_STEP=0.1)
tracks = P.simulate_tracks(P.water_cylinder_phantom(6.0), 6000, seed=3)
hist = {k: v.numpy() for k, v in P.reconstruction_histories(cfg, tracks).items()}
with Context(cfg, device=0) as ctx:
    ctx.set_reconstruction_histories(hist)
    ctx.x_host_2_GPU(np.full(cfg.NUM_VOXELS, 0.8, np.float32))
    ctx.DROP_full_tx_iteration(1)
    ctx.DROP_full_tx_iteration(2)
    ctx.set_reconstruction_histories(hist)
    ctx.DROP_full_tx_iteration(3)
    ctx.synchronize()
"""


def test_trace_reports_layout_and_graph_reuse():
    env = {**os.environ, "PCT_TRACE": "1", "PYTHONPATH": str(ROOT)}
    r = subprocess.run([sys.executable, "-c", SCRIPT], capture_output=True, text=True, env=env, cwd=str(ROOT),
                       timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stderr.splitlines() if l.startswith("pct_trace: iteration")]
    print("\n".join(lines))
    assert len(lines) == 3
    assert "layout built" in lines[0] and "graph captured" in lines[0]
    assert "layout kept" in lines[1] and "graph reused" in lines[1]
    assert "layout built" in lines[2] and "graph reused" in lines[2]
