"""Precomputed-path DROP and preprocessed-data export/import (GPU).

Precomputed-path DROP keeps the MLP voxel lists of the first iteration for the later ones; the
paths do not depend on the image, so the images must match recomputing them up to the float
atomic scatter order.  Export writes the histories, paths, chords, image and hull; an import into
a fresh context must reproduce the histories, image and hull exactly and let precomputed-path DROP
start without the path kernel.
"""
import numpy as np
import pytest

from pct_reconstruction_b200 import Config
from pct_reconstruction_b200 import phantoms as P

ATOMIC = dict(rtol=1e-4, atol=1e-5)  # float atomics: scatter order differs run to run


@pytest.fixture(scope="module")
def scan(c1_params):
    cfg = Config(**dict(c1_params, DROP_BLOCK_SIZE=3000, HISTORIES_PER_BLOCK=640))  # 3000 mod 640 = 440 skipped
    tr = P.simulate_tracks(P.water_cylinder_phantom(6.0), 120000, seed=51, continuous_angles=False,
                           angle_interval_deg=4.0, t_extent=16.0, v_extent=3.5)
    td = {k: v.numpy() for k, v in P.tracker_data(tr).items()}
    return cfg, td


def launches_of(ctx, fn):
    before = ctx.kernel_launches
    fn()
    return ctx.kernel_launches - before


@pytest.mark.gpu
def test_path_reuse_matches_recompute(scan):
    from pct_reconstruction_b200 import Context
    cfg, td = scan
    with Context(cfg) as a, Context(cfg) as b:
        na = a.preprocessing(td, integer_angles=True)
        b.preprocessing(td, integer_angles=True)
        a.set_path_reuse(True)
        assert a.path_storage_superblocks == 1 and b.path_storage_superblocks == 1  # (lays out paths)
        la = [launches_of(a, lambda: a.DROP_full_tx_iteration(i)) for i in (1, 2, 3)]
        lb = [launches_of(b, lambda: b.DROP_full_tx_iteration(i)) for i in (1, 2, 3)]
        assert la[0] == lb[0] == lb[1] == lb[2] and la[1] == la[2] == lb[1] - 1  # the path kernel runs once
        np.testing.assert_allclose(a.x_GPU_2_host(), b.x_GPU_2_host(), **ATOMIC)
        assert na > 4 * cfg.DROP_BLOCK_SIZE
        ca, cb = a.counters(), b.counters()  # path-kernel counters: once vs every iteration
        assert all(cb[k] == 3 * ca[k] for k in ca)


@pytest.mark.gpu
def test_path_reuse_with_superblocks_recomputes(scan):
    from pct_reconstruction_b200 import Context
    cfg, td = scan
    with Context(cfg) as a:
        a.preprocessing(td, integer_angles=True)
        a.set_path_storage_limit(3_000_000)
        a.set_path_reuse(True)
        assert a.path_storage_superblocks > 1
        l1 = launches_of(a, lambda: a.DROP_full_tx_iteration(1))
        l2 = launches_of(a, lambda: a.DROP_full_tx_iteration(2))
        assert l1 == l2  # paths do not stay resident: recomputed every iteration


@pytest.mark.gpu
def test_export_import_roundtrip(scan, tmp_path):
    from pct_reconstruction_b200 import Context
    cfg, td = scan
    with Context(cfg) as a, Context(cfg) as b:
        n = a.preprocessing(td, integer_angles=True)
        x0 = a.x_GPU_2_host()
        a.export_preprocessed(tmp_path)
        # file contents against the engine's own voxel lists
        counts, voxels, chord, _ = a.mlp_paths()
        B, hpb = cfg.DROP_BLOCK_SIZE, cfg.HISTORIES_PER_BLOCK
        covered = (np.arange(n) % B) < min((B // hpb) * hpb, B)
        last = n - (n // B) * B
        if last:  # the last, partial block covers floor(last/HPB)*HPB histories
            covered[(n // B) * B:] = np.arange(last) < (last // hpb) * hpb
        vpp = np.fromfile(tmp_path / "voxels_per_path.bin", np.uint32)
        assert vpp[0] == n
        np.testing.assert_array_equal(vpp[1:], np.where(covered, counts, 0))
        ch = np.fromfile(tmp_path / "avg_chord_lengths.bin", np.uint8)
        ch = np.frombuffer(ch[4:].tobytes(), np.float64)
        np.testing.assert_array_equal(ch[covered], chord[covered])
        paths = np.fromfile(tmp_path / "MLP_paths.bin", np.uint32)
        assert paths[0] == n
        expect = np.concatenate([voxels[i, :counts[i]] for i in np.nonzero(covered)[0]])
        np.testing.assert_array_equal(paths[1:], expect)
        np.testing.assert_array_equal(np.fromfile(tmp_path / "x_0.bin", np.float32), x0)
        # import into a fresh context
        assert b.import_preprocessed(tmp_path) == n
        np.testing.assert_array_equal(b.x_GPU_2_host(), x0)
        np.testing.assert_array_equal(b.get_array("hull"), a.get_array("hull"))
        b.set_path_reuse(True)
        a.set_path_reuse(True)  # export left a's paths resident too
        lb1 = launches_of(b, lambda: b.DROP_full_tx_iteration(1))
        lb2 = launches_of(b, lambda: b.DROP_full_tx_iteration(2))
        la1 = launches_of(a, lambda: a.DROP_full_tx_iteration(1))
        assert lb1 == lb2 == la1  # imported paths: no path kernel at all
    # imported paths against paths recomputed inside each block (single-pass kernel)
    with Context(cfg) as c, Context(cfg) as d:
        c.import_preprocessed(tmp_path)
        c.set_path_reuse(True)
        c.DROP_full_tx_iteration(1)
        d.import_preprocessed(tmp_path)
        d.set_path_storage_limit(-1)
        d.DROP_full_tx_iteration(1)
        np.testing.assert_allclose(c.x_GPU_2_host(), d.x_GPU_2_host(), **ATOMIC)


@pytest.mark.gpu
def test_import_rejects_inconsistent_files(scan, tmp_path):
    from pct_reconstruction_b200 import Context
    from pct_reconstruction_b200.engine import PCTError
    cfg, td = scan
    with Context(cfg) as a:
        a.preprocessing(td, integer_angles=True)
        a.export_preprocessed(tmp_path)
    p = tmp_path / "MLP_paths.bin"
    p.write_bytes(p.read_bytes()[:-4])  # one voxel short
    with Context(cfg) as b:
        with pytest.raises(PCTError) as ei:
            b.import_preprocessed(tmp_path)
        assert ei.value.status == 7


def read_exported(directory):
    """Independent reader of the exported files, in the layout of O.cu's exporters (a uint32 history
    count, then the arrays; O.cu:6540-6612): histories (ten float geometry arrays and the uint32
    first MLP voxel), WEPL, voxels per path, chord lengths (double), the packed MLP paths, x_0."""
    fields = ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit", "xy_entry_angle", "xz_entry_angle",
              "xy_exit_angle", "xz_exit_angle")
    raw = np.fromfile(directory / "histories.bin", np.uint8)
    n = int(np.frombuffer(raw[:4].tobytes(), np.uint32)[0])
    body = raw[4:]
    assert len(body) == 4 * n * 11
    hist = {k: np.frombuffer(body[4 * n * i:4 * n * (i + 1)].tobytes(), np.float32) for i, k in enumerate(fields)}
    hist["first_MLP_voxel"] = np.frombuffer(body[40 * n:44 * n].tobytes(), np.uint32)
    wepl = np.fromfile(directory / "WEPL.bin", np.uint8)
    assert int(np.frombuffer(wepl[:4].tobytes(), np.uint32)[0]) == n
    hist["WEPL"] = np.frombuffer(wepl[4:].tobytes(), np.float32)
    vpp = np.fromfile(directory / "voxels_per_path.bin", np.uint32)
    ch = np.fromfile(directory / "avg_chord_lengths.bin", np.uint8)
    chord = np.frombuffer(ch[4:].tobytes(), np.float64)
    paths = np.fromfile(directory / "MLP_paths.bin", np.uint32)
    assert vpp[0] == n and paths[0] == n and len(chord) == n and len(paths) == 1 + int(vpp[1:].sum())
    return n, hist, vpp[1:], chord, paths[1:]


@pytest.mark.gpu
def test_exported_files_and_path_reuse_against_oracle(scan, tmp_path, c1_params):
    """The exported files read back by an independent reader agree with the CPU oracle (voxel lists
    with counted ties, chords, WEPL), and precomputed-path DROP over three iterations agrees with the
    oracle's DROP, which recomputes every path."""
    from oracle import Oracle
    from pct_reconstruction_b200 import Context
    _, td = scan
    cfg = Config(**dict(c1_params, DROP_BLOCK_SIZE=3000, HISTORIES_PER_BLOCK=0))  # every history processed
    with Context(cfg) as a:
        n_ctx = a.preprocessing(td, integer_angles=True)
        x0 = a.x_GPU_2_host()
        a.export_preprocessed(tmp_path)
        a.set_path_reuse(True)
        for it in (1, 2, 3):
            a.DROP_full_tx_iteration(it)
        x3 = a.x_GPU_2_host()
    n, hist, vpp, chord, packed = read_exported(tmp_path)
    assert n == n_ctx
    o = Oracle(cfg.struct)
    oc, ov, ochord, _, _ = o.mlp_paths(hist, x0)
    off = np.concatenate([[0], np.cumsum(vpp.astype(np.int64))])
    ties = sum(1 for i in range(n) if vpp[i] != oc[i] or not np.array_equal(packed[off[i]:off[i + 1]], ov[i, :oc[i]]))
    print(f"exported voxel lists vs oracle: {ties} tie histories of {n}")
    assert ties <= 2e-3 * n
    np.testing.assert_allclose(chord, ochord, rtol=1e-6)
    ox, _ = o.drop_iteration(hist, x0, iterations=3)
    rel = float(np.sqrt(np.mean((x3.astype(np.float64) - ox) ** 2)) / np.sqrt(np.mean(ox.astype(np.float64) ** 2)))
    print(f"precomputed-path DROP (3 iterations) vs oracle: rel RMSE {rel:.2e}")
    assert rel < 1e-6
