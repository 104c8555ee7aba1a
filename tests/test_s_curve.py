"""S-curve attenuation of the DROP update (S_CURVE_ON; B.cu:9529-9534, 10606-10649).

With S_CURVE_ON the reference scales the update that entry j of an n-entry MLP path adds by
s_curve_scale_GPU(j, n): the curve S_CURVE at k = min(j, n-1-j) (DUAL_SIDED_S_CURVE) or k = j.
The reference's build always evaluates the sigmoid (its `#if (S_CURVE == SIGMOID)` compares two
enum constants, 0 == 0 in the preprocessor) and subtracts SIGMOID_MID_SHIFT from the unsigned k,
so every k below the shift scales by exactly 1.

Pins: tests/golden/ref_s_curve.npz holds the reference's five curve functions and
s_curve_scale_GPU as its device code evaluates them; ref_drop_scurve.npz one DROP iteration of the
reference built with S_CURVE_ON, on the ref_drop inputs.  Images are compared through their
updates x1 - x0, relative RMSE: the attenuation moves the updates by 5-11% (RMS), the float-atomic
order by about 1e-4.  CPU tests pin the oracle; GPU tests compare the engine through the C ABI.
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from oracle import Oracle
from pct_reconstruction_b200 import Config, PCTError

GOLDEN = Path(__file__).resolve().parent / "golden"
HIST = ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit", "xy_entry_angle", "xz_entry_angle",
        "xy_exit_angle", "xz_exit_angle", "WEPL", "first_MLP_voxel")
CURVES = ("SIGMOID", "TANH", "ATAN", "ERF", "LIN_OVER_ROOT")  # S_CURVES order (B.h:125)
UPDATE_TOL = 1e-3      # relative RMSE of the updates, same arithmetic, different atomic order
S_CURVE_EFFECT = 1e-2  # the attenuation must move the updates by more than this


def load(name):
    p = GOLDEN / name
    if not p.exists():
        pytest.fail(f"missing fixture {p}: run tests/golden/make_reference_fixtures.py on a machine with a B200")
    return dict(np.load(p))


def default_image(nv):
    i = np.arange(nv, dtype=np.uint64)
    return (0.5 + ((i * np.uint64(2654435761)) % np.uint64(1000)).astype(np.float64) / 1000.0).astype(np.float32)


def reference_image(f, x0):
    x = x0.copy()
    x[np.cumsum(f["changed_delta"].astype(np.int64)) - 1] = f["values"]
    return x


def update_rel(x1, ref1, x0):
    """Relative RMSE of the update x1 - x0 against ref1 - x0."""
    d, r = x1.astype(np.float64) - x0, ref1.astype(np.float64) - x0
    return float(np.sqrt(np.mean((d - r) ** 2) / np.mean(r ** 2)))


def ulp_distance(a, b):
    ia, ib = a.view(np.int32).astype(np.int64), b.view(np.int32).astype(np.int64)
    return np.abs(ia - ib)


def drop_inputs():
    f = load("ref_drop.npz")
    return f, {k: f[k] for k in HIST}, int(f["drop_block_size"])


# ---------------------------------------------------------------- configuration (CPU) -------

def test_s_curve_config_keys():
    c = Config()
    assert (c.S_CURVE_ON, c.S_CURVE, c.DUAL_SIDED_S_CURVE, c.SIGMOID_MID_SHIFT, c.SIGMOID_STEEPNESS) == \
        (0, 0, 1, 10, 1.25)  # B.h:178, 467-470
    c = Config(S_CURVE_ON="ON", S_CURVE="ERF", DUAL_SIDED_S_CURVE="OFF", SIGMOID_MID_SHIFT=4, SIGMOID_STEEPNESS=2.0)
    assert (c.S_CURVE_ON, c.S_CURVE, c.DUAL_SIDED_S_CURVE, c.SIGMOID_MID_SHIFT, c.SIGMOID_STEEPNESS) == \
        (1, 3, 0, 4, 2.0)


@pytest.mark.parametrize("bad", [dict(PRECISION="MIXED"), dict(PRECISION="MIXED_COMPENSATED"),
                                 dict(PROJECTION_ALGORITHM="ROBUSTA"), dict(PROJECTION_ALGORITHM="ROBUSTB"),
                                 dict(S_CURVE=5), dict(DUAL_SIDED_S_CURVE=2)])
def test_s_curve_config_rejections(bad):
    with pytest.raises(PCTError):
        Config(S_CURVE_ON=1, **bad)


# ---------------------------------------------------------------- oracle (CPU) --------------

def test_oracle_sigmoid_unsigned_shift():
    t = Oracle(Config(S_CURVE_ON=1).struct).s_curve_table(64)
    assert np.all(t[:10] == 1.0)  # k - 10 wraps to about 4.3e9: exp(-5.4e9) = 0
    assert t[10] == 0.5
    assert np.all(np.diff(t[10:]) >= 0) and t[40] == 1.0
    t0 = Oracle(Config(S_CURVE_ON=1, SIGMOID_MID_SHIFT=0).struct).s_curve_table(4)
    assert t0[0] == 0.5


def test_oracle_s_curve_matches_reference_device_code():
    f = load("ref_s_curve.npz")
    count = f["curves"].shape[1]
    for row, name in enumerate(CURVES):
        o = Oracle(Config(S_CURVE_ON=1, S_CURVE=name).struct).s_curve_table(count)
        d = ulp_distance(o, f["curves"][row])
        print(f"oracle {name}: {int((d == 0).sum())} of {count} bit-identical, max {int(d.max())} ulp")
        assert d.max() <= 2, name  # host libm vs CUDA's math functions


def test_reference_scale_index_rule():
    """s_curve_scale_GPU(j, n) of the reference equals its sigmoid at min(j, n-1-j): the build's
    curve is SIGMOID and DUAL_SIDED_S_CURVE is ON, the rule the engine and the oracle use."""
    f = load("ref_s_curve.npz")
    j, n = f["j"].astype(np.int64), f["n"].astype(np.int64)
    k = np.minimum(j, n - 1 - j)
    assert np.array_equal(f["scale"].view(np.uint32), f["curves"][0][k].view(np.uint32))


def test_oracle_drop_s_curve_matches_reference_device_code():
    f0, hist, block = drop_inputs()
    f = load("ref_drop_scurve.npz")
    cfg = Config(DROP_BLOCK_SIZE=block, S_CURVE_ON=1)
    x0 = default_image(cfg.NUM_VOXELS)
    ref = reference_image(f, x0)
    x1, _ = Oracle(cfg.struct).drop_iteration(hist, x0)
    r = update_rel(x1, ref, x0)
    effect = update_rel(reference_image(f0, x0), ref, x0)
    print(f"oracle vs reference S-curve DROP: update rel RMSE {r:.2e}; attenuation moves the updates {effect:.2e}")
    assert r < UPDATE_TOL
    assert effect > S_CURVE_EFFECT


# ---------------------------------------------------------------- engine (GPU) --------------

@pytest.mark.gpu
def test_engine_s_curve_table_matches_reference_device_code():
    from pct_reconstruction_b200 import Context
    f = load("ref_s_curve.npz")
    count = f["curves"].shape[1]
    for row, name in enumerate(CURVES):
        with Context(Config(S_CURVE_ON=1, S_CURVE=name)) as ctx:
            t = ctx.s_curve(count)
        d = ulp_distance(t, f["curves"][row])
        print(f"engine {name}: {int((d == 0).sum())} of {count} bit-identical, max {int(d.max())} ulp")
        assert np.array_equal(t.view(np.uint32), f["curves"][row].view(np.uint32)), name


@pytest.mark.gpu
def test_engine_drop_s_curve_matches_reference_device_code():
    from pct_reconstruction_b200 import Context
    f0, hist, block = drop_inputs()
    f = load("ref_drop_scurve.npz")
    cfg = Config(DROP_BLOCK_SIZE=block, S_CURVE_ON=1)
    x0 = default_image(cfg.NUM_VOXELS)
    ref = reference_image(f, x0)
    with Context(cfg) as ctx:
        ctx.set_reconstruction_histories(hist)
        ctx.x_host_2_GPU(x0)
        ctx.DROP_full_tx_iteration(1)
        g = ctx.x_GPU_2_host()
    r = update_rel(g, ref, x0)
    print(f"engine vs reference S-curve DROP: update rel RMSE {r:.2e}")
    assert r < UPDATE_TOL
    assert update_rel(reference_image(f0, x0), ref, x0) > S_CURVE_EFFECT


@pytest.mark.gpu
@pytest.mark.parametrize("curve,dual,mode,route", [
    ("SIGMOID", 1, "ATOMIC", "iteration"), ("TANH", 0, "ATOMIC", "iteration"),
    ("ATAN", 1, "DETERMINISTIC", "iteration"), ("ERF", 0, "DETERMINISTIC", "iteration"),
    ("LIN_OVER_ROOT", 1, "ATOMIC", "reuse"), ("SIGMOID", 0, "ATOMIC", "single_pass")])
def test_engine_drop_s_curve_matches_oracle(curve, dual, mode, route):
    """Every curve, both index rules and both scatter modes against the oracle: through the
    iteration graph (two phases), with precomputed paths, and through the single-pass block kernel
    (pct_calculate_x_update + pct_image_update)."""
    from pct_reconstruction_b200 import Context
    _, hist, block = drop_inputs()
    cfg = Config(DROP_BLOCK_SIZE=block, HISTORIES_PER_BLOCK=0, S_CURVE_ON=1, S_CURVE=curve,
                 DUAL_SIDED_S_CURVE=dual, SCATTER_MODE=mode, SIGMOID_MID_SHIFT=6, SIGMOID_STEEPNESS=0.9)
    x0 = default_image(cfg.NUM_VOXELS)
    n = len(hist["WEPL"])
    iterations = 2 if route == "reuse" else 1
    o, _ = Oracle(cfg.struct).drop_iteration(hist, x0, iterations=iterations)
    plain = Config(DROP_BLOCK_SIZE=block, HISTORIES_PER_BLOCK=0, SCATTER_MODE=mode)
    p, _ = Oracle(plain.struct).drop_iteration(hist, x0, iterations=iterations)
    with Context(cfg) as ctx:
        ctx.set_reconstruction_histories(hist)
        ctx.x_host_2_GPU(x0)
        if route == "single_pass":
            for start in range(0, n, block):
                ctx.calculate_x_update(start, min(block, n - start))
                ctx.image_update()
        else:
            if route == "reuse":
                ctx.set_path_reuse(True)
            for it in range(iterations):
                ctx.DROP_full_tx_iteration(it + 1)
        g = ctx.x_GPU_2_host()
        assert not any(ctx.counters().values())
    r = update_rel(g, o, x0)
    effect = update_rel(p, o, x0)
    print(f"{curve} dual={dual} {mode} {route}: engine vs oracle {r:.2e}, attenuation {effect:.2e}")
    assert r < UPDATE_TOL
    assert effect > S_CURVE_EFFECT


@pytest.mark.gpu
def test_engine_s_curve_of_ones_is_the_plain_update():
    """With every k below SIGMOID_MID_SHIFT the sigmoid is exactly 1 and 1 * L = L, so the S-curve
    kernel's updates equal the plain kernel's; the fixed-point scatter makes the images bit-equal."""
    from pct_reconstruction_b200 import Context
    _, hist, block = drop_inputs()
    images = []
    for extra in (dict(), dict(S_CURVE_ON=1, SIGMOID_MID_SHIFT=2000)):
        cfg = Config(DROP_BLOCK_SIZE=block, SCATTER_MODE="DETERMINISTIC", **extra)
        with Context(cfg) as ctx:
            if extra:
                assert np.all(ctx.s_curve() == 1.0)
            ctx.set_reconstruction_histories(hist)
            ctx.x_host_2_GPU(default_image(cfg.NUM_VOXELS))
            ctx.DROP_full_tx_iteration(1)
            images.append(ctx.x_GPU_2_host())
    assert np.array_equal(images[0].view(np.uint32), images[1].view(np.uint32))


@pytest.mark.gpu
def test_engine_s_curve_state_and_no_alloc_rejection():
    from pct_reconstruction_b200 import Context, _abi
    import torch
    with Context(Config()) as ctx:
        with pytest.raises(PCTError):
            ctx.s_curve()
    cfg = Config(S_CURVE_ON=1)
    with Context(cfg) as ctx:
        lib = _abi.load_library()
        x = torch.zeros(cfg.NUM_VOXELS, dtype=torch.float32, device="cuda")
        h = _abi.pct_histories()
        torch.cuda.synchronize()
        st = lib.pct_drop_block_update_noalloc(ctx._h, C.byref(h), 0, C.c_void_p(x.data_ptr()))
        assert st == _abi.PCT_ERR_ARG
        assert b"S_CURVE_ON" in lib.pct_last_error(ctx._h)
