"""History ordering (prime permutation), robust DROP variants and the air threshold.

apply_history_sequence (B.cu:8691) reorders the reconstruction histories by
sequence[i] = (sequence[i-1] + PRIME_OFFSET) mod N; the robust updates restate
DROP_blocks_robust1 / DROP_blocks_robust2 + DROP_update_robust2 (O.cu:7537-7583); the air
threshold is image_update_GPU's IDENTIFY_X_N_AIR branch (B.cu:9411).  GPU images are compared with
the oracle at the DROP tolerance (float atomics, path-sum order).
"""
import numpy as np
import pytest

from oracle import Oracle
from pct_reconstruction_b200 import Config
from pct_reconstruction_b200 import phantoms as P

IMAGE_REL_RMSE = 1e-6
IMAGE_ATOL = 1e-5


def reference_sequence(n, prime):
    seq = np.zeros(n, np.int64)
    for i in range(1, n):
        seq[i] = (seq[i - 1] + prime) % n
    return seq


def test_prime_sequence_closed_form():
    for n, p in [(1000, 26410633), (997, 5038457), (12, 5)]:
        seq = reference_sequence(n, p)
        np.testing.assert_array_equal(seq, (np.arange(n, dtype=np.int64) * (p % n)) % n)
        if np.gcd(p % n, n) == 1:
            assert len(np.unique(seq)) == n


def test_config_keys_and_validation():
    cfg = Config(PROJECTION_ALGORITHM="ROBUSTA", RECON_HISTORY_ORDERING="PRIME_PERMUTATION", ETA=1.5, PSI_SIGN=-1,
                 PRIME_OFFSET=5038457, IDENTIFY_X_N_AIR=1, X_N_AIR_THRESHOLD=0.2)
    assert cfg.PROJECTION_ALGORITHM == 5 and cfg.RECON_HISTORY_ORDERING == 1 and cfg.PSI_SIGN == -1
    assert cfg.PRIME_OFFSET == 5038457 and cfg.ETA == 1.5 and cfg.IDENTIFY_X_N_AIR == 1
    d = Config()
    assert d.PROJECTION_ALGORITHM == 2 and d.RECON_HISTORY_ORDERING == 0 and d.PRIME_OFFSET == 26410633
    from pct_reconstruction_b200.engine import PCTError
    with pytest.raises(PCTError):
        Config(PROJECTION_ALGORITHM=0)  # ART: not a projection algorithm of the built reference
    with pytest.raises(PCTError):
        Config(PSI_SIGN=2)


@pytest.fixture(scope="module")
def c1_hist(c1_params):
    cfg = Config(**c1_params)
    tr = P.simulate_tracks(P.water_cylinder_phantom(6.0), 20000, seed=61)
    hist = {k: v.numpy() for k, v in P.reconstruction_histories(cfg, tr).items()}
    rng = np.random.default_rng(7)
    x = (0.5 + rng.random(cfg.NUM_VOXELS)).astype(np.float32)
    return hist, x


def test_oracle_robustb_without_perturbation_is_drop(c1_params, c1_hist):
    hist, x = c1_hist
    o_drop, _ = Oracle(Config(**c1_params).struct).drop_iteration(hist, x, iterations=1)
    o_rb, _ = Oracle(Config(**dict(c1_params, PROJECTION_ALGORITHM="ROBUSTB", ETA=0.0)).struct).drop_iteration(
        hist, x, iterations=1)
    np.testing.assert_allclose(o_rb, o_drop, rtol=1e-6, atol=1e-7)  # ||a||^2/(||a||^2 + 0) = 1


def test_oracle_air_threshold(c1_params, c1_hist):
    hist, x = c1_hist
    one_block = dict(c1_params, DROP_BLOCK_SIZE=1 << 20, HISTORIES_PER_BLOCK=0)  # one update per voxel
    base, _ = Oracle(Config(**one_block).struct).drop_iteration(hist, x, iterations=1)
    air, _ = Oracle(Config(**dict(one_block, IDENTIFY_X_N_AIR=1, X_N_AIR_THRESHOLD=0.9)).struct).drop_iteration(
        hist, x, iterations=1)
    moved = base != x
    assert np.all(air[moved & (base >= 0.9)] == base[moved & (base >= 0.9)])
    assert np.all(air[moved & (base < 0.9)] == 0)


def assert_image_close(g, o):
    rel = float(np.sqrt(np.mean((g.astype(np.float64) - o) ** 2)) / np.sqrt(np.mean(o.astype(np.float64) ** 2)))
    assert rel < IMAGE_REL_RMSE, rel
    np.testing.assert_allclose(g, o, rtol=0, atol=IMAGE_ATOL)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [dict(PROJECTION_ALGORITHM="ROBUSTA"),
                                     dict(PROJECTION_ALGORITHM="ROBUSTA", PSI_SIGN=-1, ETA=0.5),
                                     dict(PROJECTION_ALGORITHM="ROBUSTB"),
                                     dict(IDENTIFY_X_N_AIR=1, X_N_AIR_THRESHOLD=0.9)])
def test_engine_variants_match_oracle(c1_params, c1_hist, variant):
    from pct_reconstruction_b200 import Context
    hist, x = c1_hist
    if variant.get("PROJECTION_ALGORITHM") == "ROBUSTA":
        # keep <a,a> + Psi_j away from 0 (Psi_j = (1 - x_j) ETA): near 0 the update is ill-conditioned
        # and the order of the path sum decides the result
        x = (0.95 + 0.1 * np.random.default_rng(8).random(len(x))).astype(np.float32)
    cfg = Config(**dict(c1_params, **variant))
    with Context(cfg) as ctx:
        ctx.set_reconstruction_histories(hist)
        ctx.x_host_2_GPU(x)
        for it in (1, 2):
            ctx.DROP_full_tx_iteration(it)
        g = ctx.x_GPU_2_host()
    o, _ = Oracle(cfg.struct).drop_iteration(hist, x, iterations=2)
    assert (o != x).sum() > 1000
    assert_image_close(g, o)


@pytest.mark.gpu
def test_robust_needs_path_storage(c1_params, c1_hist):
    from pct_reconstruction_b200 import Context
    from pct_reconstruction_b200.engine import PCTError
    hist, x = c1_hist
    with Context(Config(**dict(c1_params, PROJECTION_ALGORITHM="ROBUSTB"))) as ctx:
        ctx.set_reconstruction_histories(hist)
        ctx.set_path_storage_limit(-1)
        with pytest.raises(PCTError) as ei:
            ctx.DROP_full_tx_iteration(1)
        assert ei.value.status == 5


@pytest.mark.gpu
def test_history_sequence_permutes_and_drop_follows(c1_params, c1_hist):
    from pct_reconstruction_b200 import Context
    from pct_reconstruction_b200.engine import PCTError
    hist, x = c1_hist
    cfg = Config(**c1_params)
    n = len(hist["WEPL"])
    prime = 5038457
    if np.gcd(prime % n, n) != 1:
        prime = 26410633
    seq = (np.arange(n, dtype=np.int64) * (prime % n)) % n
    permuted = {k: v[seq] for k, v in hist.items()}
    with Context(cfg) as ctx:
        ctx.set_reconstruction_histories(hist)
        ctx.apply_history_sequence(prime)
        for k in ("x_entry", "xz_exit_angle", "WEPL", "first_MLP_voxel"):
            np.testing.assert_array_equal(ctx.get_array(k + "_reconstruction"), permuted[k], err_msg=k)
        ctx.x_host_2_GPU(x)
        ctx.DROP_full_tx_iteration(1)
        g = ctx.x_GPU_2_host()
        with pytest.raises(PCTError):
            ctx.apply_history_sequence(n * 2)  # shares a factor with n
    o, _ = Oracle(cfg.struct).drop_iteration(permuted, x, iterations=1)
    assert_image_close(g, o)
