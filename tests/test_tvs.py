"""Total variation superiorization (NTVS): oracle known answers on CPU, engine vs oracle on GPU.

The oracle (oracle/pct_oracle_tvs.c) restates calculate_total_variation (B.cu:10163),
generate_perturbation_array (B.cu:10246) and iteratively_perturb_image (B.cu:10476).  The GPU
test compares the engine with the oracle's engine-arithmetic mode (double accumulation): the L
sequence must be identical and the image equal to float rounding (rtol 1e-6; the ||G|| sums are
double sums in different orders).
"""
import numpy as np
import pytest

from oracle import TVS_ENGINE, TVS_REFERENCE, TvsOracle
from pct_reconstruction_b200 import Config

SMALL = dict(COLUMNS=48, ROWS=44, SLICES=3, VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, RECON_CYL_RADIUS=2.4)


def noisy_image(cfg, seed, noise=0.05):
    rng = np.random.default_rng(seed)
    C, R, S = cfg.COLUMNS, cfg.ROWS, cfg.SLICES
    yy, xx = np.mgrid[0:R, 0:C]
    disk = ((xx - C / 2) ** 2 + (yy - R / 2) ** 2 < (0.4 * C) ** 2).astype(np.float32)
    vol = np.stack([disk * (1.0 + 0.1 * s) for s in range(S)])
    return (vol + noise * rng.normal(size=vol.shape)).astype(np.float32).ravel(), \
        np.stack([((xx - C / 2) ** 2 + (yy - R / 2) ** 2 < (0.45 * C) ** 2)] * S).astype(np.uint8).ravel()


def numpy_tv(cfg, x):
    v = x.reshape(cfg.SLICES, cfg.ROWS, cfg.COLUMNS)
    dy = v[:, 1:, :-1] - v[:, :-1, :-1]
    dx = v[:, :-1, 1:] - v[:, :-1, :-1]
    return float(np.sqrt(dy.astype(np.float32) ** 2 + dx.astype(np.float32) ** 2).astype(np.float64).sum())


def numpy_direction(cfg, x):
    """Independent restatement of the subgradient scatter (reference loop order)."""
    C, R, S = cfg.COLUMNS, cfg.ROWS, cfg.SLICES
    G = np.zeros(cfg.NUM_VOXELS, np.float32)
    f = np.float32
    for s in range(S):
        for r in range(R - 1):
            for c in range(C - 1):
                p = c + r * C + s * R * C
                gx, gy = f(x[p + 1] - x[p]), f(x[p + C] - x[p])
                gn = f(np.sqrt(np.float64(gx) ** 2 + np.float64(gy) ** 2))
                if gn > 0:
                    G[p] = f(G[p] - f(f(gx + gy) / gn))
                    G[p + C] = f(G[p + C] + f(gy / gn))
                    G[p + 1] = f(G[p + 1] + f(gx / gn))
    return G


# ---------------------------------------------------------------- oracle (CPU) ------------

def test_eta_table_is_powers_of_A():
    o = TvsOracle(Config(**SMALL).struct)
    eta = o.eta()
    assert len(eta) == 132  # int(log(1e-40)/log(0.5)) exponents 0..131
    np.testing.assert_array_equal(eta, np.float32(0.5) ** np.arange(132, dtype=np.float32))
    o3 = TvsOracle(Config(**SMALL, TVS_A=0.75, TVS_L_0=2).struct)
    assert len(o3.eta()) == int(np.log(1e-40) / np.log(0.75)) - 2


def test_randi_range_and_determinism():
    o = TvsOracle(Config(**SMALL).struct)
    draws = [o.randi(3, 9, k) for k in range(1, 200)]
    assert min(draws) >= 3 and max(draws) <= 9 and len(set(draws)) == 7
    assert draws == [o.randi(3, 9, k) for k in range(1, 200)]
    assert o.randi(5, 2, 1) == 5  # empty range: lower bound


def test_total_variation_known_answers():
    cfg = Config(**SMALL)
    o = TvsOracle(cfg.struct)
    assert o.total_variation(np.full(cfg.NUM_VOXELS, 1.7, np.float32)) == 0.0
    x = np.zeros(cfg.NUM_VOXELS, np.float32)
    x[5 + 7 * cfg.COLUMNS] = 1.0  # one bright voxel: terms at itself (sqrt 2), left and upper neighbour (1 each)
    assert o.total_variation(x) == pytest.approx(np.sqrt(2) + 2.0, rel=1e-7)
    xr, _ = noisy_image(cfg, 3)
    assert o.total_variation(xr) == pytest.approx(numpy_tv(cfg, xr), rel=1e-9)
    assert TvsOracle(cfg.struct, TVS_REFERENCE).total_variation(xr) == pytest.approx(numpy_tv(cfg, xr), rel=1e-4)


def test_direction_matches_numpy_scatter():
    cfg = Config(**dict(SMALL, SLICES=1))
    x, _ = noisy_image(cfg, 4)
    G, v, norm = TvsOracle(cfg.struct).direction(x)
    np.testing.assert_array_equal(G, numpy_direction(cfg, x))
    assert norm == pytest.approx(float(np.sqrt((G.astype(np.float64) ** 2).sum())), rel=1e-6)
    assert float(np.linalg.norm(v.astype(np.float64))) == pytest.approx(1.0, rel=1e-5)
    assert abs(float(G.astype(np.float64).sum())) < 1e-3  # each scatter adds and removes the same amount


def test_ntvs_lowers_tv_and_reference_mode_agrees():
    cfg = Config(**SMALL)
    x, hull = noisy_image(cfg, 5)
    eng, ref = TvsOracle(cfg.struct, TVS_ENGINE), TvsOracle(cfg.struct, TVS_REFERENCE)
    xe, xr, Le, Lr = x, x, 0, 0
    for k in range(1, 4):
        tv0 = eng.total_variation(xe)
        xe, Le, acc_e = eng.ntvs_iteration(xe, hull, k, Le)
        xr, Lr, acc_r = ref.ntvs_iteration(xr, hull, k, Lr)
        assert eng.total_variation(xe) <= tv0
        assert len(acc_e) == 5 and acc_e == sorted(acc_e)
        assert acc_e == acc_r  # float vs double sums decide alike away from ties
    np.testing.assert_allclose(xe, xr, rtol=1e-4, atol=1e-4)  # float vs double norm of G
    assert np.all(xe[hull == 0] == x[hull == 0])  # only hull voxels move


def test_unconditioned_and_old_variants():
    cfg = Config(**dict(SMALL, TVS_CONDITIONED=0))
    x, hull = noisy_image(cfg, 6)
    _, L, acc = TvsOracle(cfg.struct).ntvs_iteration(x, hull, 1, 0)
    assert acc == [1, 2, 3, 4, 5] and L == 5
    cfg_old = Config(**dict(SMALL, TVS_OLD=1))
    _, L, acc = TvsOracle(cfg_old.struct).ntvs_iteration(x, hull, 4, 7)  # no draw, one repetition
    assert len(acc) == 1 and acc[0] >= 8


def test_config_keys():
    cfg = Config(A=0.75, L_0=1, TVS_REPETITIONS=3, TVS_SEED=12345)
    assert cfg.TVS_A == 0.75 and cfg.TVS_L_0 == 1 and cfg.TVS_REPETITIONS == 3 and cfg.TVS_SEED == 12345
    d = Config()
    assert d.TVS_ON == 1 and d.TVS_FIRST == 1 and d.TVS_CONDITIONED == 1 and d.TV_THRESHOLD == 0.0


# ---------------------------------------------------------------- engine (GPU) ------------

@pytest.mark.gpu
def test_engine_total_variation_matches_oracle():
    from pct_reconstruction_b200 import Context
    cfg = Config(**dict(SMALL, COLUMNS=160, ROWS=150, SLICES=8))
    x, _ = noisy_image(cfg, 7)
    with Context(cfg) as ctx:
        ctx.x_host_2_GPU(x)
        tv = ctx.total_variation()
    assert tv == pytest.approx(TvsOracle(cfg.struct).total_variation(x), rel=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [{}, {"TVS_CONDITIONED": 0}, {"TVS_OLD": 1}, {"TVS_A": 0.75}])
def test_engine_ntvs_matches_oracle(variant):
    from pct_reconstruction_b200 import Context
    cfg = Config(**dict(SMALL, COLUMNS=160, ROWS=150, SLICES=8, **variant))
    x, hull = noisy_image(cfg, 8)
    o = TvsOracle(cfg.struct)
    with Context(cfg) as ctx:
        ctx.x_host_2_GPU(x)
        ctx.set_array("hull", hull)
        L = ctx.tvs_L
        assert L == 0
        xo = x
        for k in range(1, 5):
            xo, L, _ = o.ntvs_iteration(xo, hull, k, L)
            ctx.NTVS_iteration(k)
            assert ctx.tvs_L == L, f"iteration {k}"
            np.testing.assert_allclose(ctx.x_GPU_2_host(), xo, rtol=1e-6, atol=1e-7, err_msg=f"iteration {k}")
        assert ctx.counters()["wait_expired"] == 0


@pytest.mark.gpu
def test_ntvs_needs_hull():
    from pct_reconstruction_b200 import Context
    from pct_reconstruction_b200.engine import PCTError
    with Context(Config(**SMALL)) as ctx:
        with pytest.raises(PCTError) as ei:
            ctx.NTVS_iteration(1)
        assert ei.value.status == 5  # PCT_ERR_STATE
