"""SC / MSC / SM hull walks against the reference's own walk code.

tests/golden/ref_hull_walks*.npz were made by tests/golden/make_reference_fixtures.py on a B200: a
harness kernel (oracle/ref_harness.cu, command `walks`) runs the loop of SC_GPU / MSC_GPU / SM_GPU
(B.cu:6681-7099) with the reference's own compiled primitives calculate_voxel_GPU,
distance_remaining_GPU, take_2D_step_GPU and take_3D_step_GPU (B.cu:11091-11462), bounded by a step
limit and a stop before any negative voxel index (where the reference's loop never ends).  Two
configurations:
  * ref_hull_walks.npz: the reference's built-in grid (256 x 256 x 32, 0.0625 cm voxels), on the
    reference's own intersections stored in ref_intersections_binning.npz;
  * ref_hull_walks_head.npz: the head grid (200 x 200 x 32, 0.1 cm voxels; B.cu compiled with a
    patched B.h), on the reference's intersections of simulated head-phantom protons.
The outputs are integer images (SC carve flags, MSC and SM counts), which do not depend on the
order of the walks, so the bar is exact equality.  A difference would be a floating-point
boundary tie in a walk; each test lists the differing voxels before it fails.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import GEOM, PreOracle
from pct_reconstruction_b200 import Config

GOLDEN = Path(__file__).resolve().parent / "golden"
GEOM6 = ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit")
HEAD = dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, RECON_CYL_RADIUS=10.0, DROP_BLOCK_SIZE=60000, HISTORIES_PER_BLOCK=480)


def load(name):
    p = GOLDEN / name
    if not p.exists():
        pytest.fail(f"missing fixture {p}: run tests/golden/make_reference_fixtures.py on a machine with a B200")
    return dict(np.load(p))


def walk_case(name):
    """(configuration parameters, geometry, WEPL, missed, reference outputs) of one walk fixture."""
    f = load(name)
    w = f["walk_windows"]
    windows = dict(SC_LOWER_THRESHOLD=float(w[0]), SC_UPPER_THRESHOLD=float(w[1]), MSC_LOWER_THRESHOLD=float(w[2]),
                   MSC_UPPER_THRESHOLD=float(w[3]), SM_LOWER_THRESHOLD=float(w[4]), SC_ON=1, MSC_ON=1, SM_ON=1)
    if name == "ref_hull_walks.npz":
        src = load("ref_intersections_binning.npz")
        geom = {k: src["out_" + k] for k in GEOM6}
        wepl, missed = src["WEPL"], src["missed_recon_volume"]
        params = windows
    else:
        geom = {k: f["in_" + k] for k in GEOM6}
        wepl = f["in_WEPL"]
        missed = np.zeros(len(wepl), np.uint8)
        params = dict(HEAD, **windows)
    nv = int(f["num_voxels"])
    assert nv == Config(**params).NUM_VOXELS
    ref = {"SC_carved": np.unpackbits(f["out_SC_carved"])[:nv].astype(bool),
           "MSC": unsparse(f["out_MSC_delta"], f["out_MSC_values"], nv),
           "SM": unsparse(f["out_SM_delta"], f["out_SM_values"], nv),
           "status": f["out_status"]}
    return params, geom, wepl, missed, ref


def unsparse(delta, values, nv):
    a = np.zeros(nv, np.int32)
    a[np.cumsum(delta.astype(np.int64)) - 1] = values
    return a


def full_geometry(geom):
    g = {k: np.zeros(len(geom["x_entry"]), np.float32) for k in GEOM}
    g.update(geom)
    return g


def assert_same_image(got, ref, what):
    diff = np.nonzero(got != ref)[0]
    if len(diff):
        print(f"{what}: {len(diff)} voxels differ, first {diff[:20].tolist()}: "
              f"got {got[diff[:20]].tolist()} reference {ref[diff[:20]].tolist()}")
    assert len(diff) == 0, f"{what}: {len(diff)} voxels differ from the reference"


def report(name, ref):
    st = np.bincount(ref["status"], minlength=3)
    print(f"{name}: {int(ref['SC_carved'].sum())} carved voxels, {int(ref['MSC'].sum())} MSC and "
          f"{int(ref['SM'].sum())} SM visits; walks ended {st[0]}, stopped below index 0 {st[1]} "
          f"(never end in the reference), step bound {st[2]}")
    assert st[2] == 0


@pytest.mark.parametrize("name", ["ref_hull_walks.npz", "ref_hull_walks_head.npz"])
def test_oracle_hull_walks_match_reference(name):
    params, geom, wepl, missed, ref = walk_case(name)
    cfg = Config(**params)
    report(name, ref)
    o = PreOracle(cfg.struct)
    g = full_geometry(geom)
    nv = cfg.NUM_VOXELS
    sc, _ = o.hull_walks(0, g, wepl, missed, np.ones(nv, np.int32))
    msc, _ = o.hull_walks(1, g, wepl, missed, np.zeros(nv, np.int32))
    sm, _ = o.hull_walks(2, g, wepl, missed, np.zeros(nv, np.int32))
    assert_same_image(sc == 0, ref["SC_carved"], "oracle SC carve")
    assert_same_image(msc, ref["MSC"], "oracle MSC counts")
    assert_same_image(sm, ref["SM"], "oracle SM counts")


def engine_hulls(params, geom, wepl, missed, walks=True):
    """SC hull, MSC and SM count images of the engine's hull_detection stage on given
    intersections (the tracker data only sizes the arrays; the geometry is then replaced)."""
    from pct_reconstruction_b200 import Context
    n = len(wepl)
    tracker = {k: np.zeros(n, np.float32) for k in ("t_in_1", "t_in_2", "t_out_1", "t_out_2", "v_in_1", "v_in_2",
                                                    "v_out_1", "v_out_2")}
    for k, u in (("u_in_1", -15.0), ("u_in_2", -10.0), ("u_out_1", 10.0), ("u_out_2", 15.0)):
        tracker[k] = np.full(n, u, np.float32)
    tracker["WEPL"] = np.asarray(wepl, np.float32)
    tracker["gantry_angle"] = np.zeros(n, np.float32)
    c = Config(**params) if walks else Config(**dict(params, SC_ON=0, MSC_ON=0, SM_ON=0))
    with Context(c) as ctx:
        ctx.load_tracker_data(tracker, integer_angles=True)
        ctx.stage("recon_volume_intersections")
        for k in GEOM6:
            ctx.set_array(k, np.asarray(geom[k], np.float32))
        ctx.set_array("missed_recon_volume", np.asarray(missed, np.uint8))
        ctx.set_array("WEPL", np.asarray(wepl, np.float32))
        ctx.stage("hull_detection")
        out = (ctx.get_array("SC_hull"), ctx.get_array("MSC_counts"), ctx.get_array("SM_counts"))
        assert ctx.counters()["wait_expired"] == 0
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ref_hull_walks.npz", "ref_hull_walks_head.npz"])
def test_engine_hull_walks_match_reference(name):
    params, geom, wepl, missed, ref = walk_case(name)
    cfg = Config(**params)
    report(name, ref)
    sc, msc, sm = engine_hulls(params, geom, wepl, missed)
    init_sc, init_msc, init_sm = engine_hulls(params, geom, wepl, missed, walks=False)
    cyl = init_sc.astype(bool)
    assert cyl.sum() > 0.7 * cfg.NUM_VOXELS  # the cylinder inscribed in the grid (pi/4)
    # the hulls start from the cylinder (initialize_hull_GPU B.cu:6659); SC walks carve it, MSC and
    # SM walks add to their counts
    assert_same_image(sc[cyl] == 0, ref["SC_carved"][cyl], "engine SC carve inside the cylinder")
    assert_same_image(msc - init_msc, ref["MSC"], "engine MSC counts")
    assert_same_image(sm - init_sm, ref["SM"], "engine SM counts")
