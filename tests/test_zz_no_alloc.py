"""The allocation-free DROP block update (pct_drop_block_update_noalloc), on a GPU.

It is for callers that cannot call cudaMalloc/cudaFree while reconstructing (a real-time service
whose allocations would stall other streams, or a host with a fixed device-memory budget).  The
test calls it through the C ABI on two DROP blocks in a row and compares each result with the
ordinary path (pct_calculate_x_update + pct_image_update, which uses context-owned scratch), within
the image tolerance of the other DROP tests, on an even and an odd voxel count.  The second call
checks that the shared static accumulator starts each call cleared.  The argument checks (scatter
mode, projection algorithm, image alignment, grid size, n = 0) are exercised without a kernel
launch that could fault.  This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

from pct_reconstruction_b200 import Config, Context, _abi
from pct_reconstruction_b200 import phantoms as P

pytestmark = pytest.mark.gpu

IMAGE_REL_RMSE = 1e-6
IMAGE_ATOL = 1e-5


def close(g, o):
    g64, o64 = g.astype(np.float64), o.astype(np.float64)
    rel = float(np.sqrt(np.mean((g64 - o64) ** 2)) / np.sqrt(np.mean(o64 ** 2)))
    assert rel < IMAGE_REL_RMSE, rel
    np.testing.assert_allclose(g, o, rtol=0, atol=IMAGE_ATOL)


def noalloc(lib, ctx, dev, start, n, x_ptr):
    """One call of the entry point through the C ABI on caller-owned device buffers."""
    ptrs = [ctypes.c_void_p(dev[k].data_ptr() + 4 * start) for k in _abi.HISTORY_FIELDS]
    h = _abi.pct_histories(*ptrs)
    return lib.pct_drop_block_update_noalloc(ctx._h, ctypes.byref(h), n, ctypes.c_void_p(x_ptr))


def compare_two_blocks(cfg, n_tracks, seed, block):
    """Two DROP blocks in a row through the entry point vs the ordinary path (context-owned
    accumulator); also checks that the walk-flag counters advance alike."""
    tracks = P.simulate_tracks(P.water_cylinder_phantom(0.95 * cfg.RECON_CYL_RADIUS), n_tracks, seed=seed)
    hist = {k: v.numpy() for k, v in P.reconstruction_histories(cfg, tracks).items()}
    assert len(hist["WEPL"]) >= 2 * block
    rng = np.random.default_rng(9)
    x0 = (0.5 + rng.random(cfg.NUM_VOXELS)).astype(np.float32)
    lib = _abi.load_library()
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in hist.items()}
    with Context(cfg) as ctx:
        ctx.set_reconstruction_histories(hist)
        ctx.x_host_2_GPU(x0)
        x_dev = torch.from_numpy(x0.copy()).cuda()
        for b in range(2):
            start = b * block
            # ordinary path: context-owned image and accumulator
            c0 = ctx.counters()
            ctx.calculate_x_update(start, block)
            ctx.image_update()
            expect = ctx.x_GPU_2_host()
            c1 = ctx.counters()
            # allocation-free path: caller-owned histories and image
            st = noalloc(lib, ctx, dev, start, block, x_dev.data_ptr())
            assert st == _abi.PCT_OK, lib.pct_last_error(ctx._h)
            ctx.synchronize()
            c2 = ctx.counters()
            got = x_dev.cpu().numpy()
            assert (got != x0).sum() > 1000
            close(got, expect)
            for k in ("path_overflow", "table_range"):
                assert c2[k] - c1[k] == c1[k] - c0[k], (k, c0, c1, c2)


def test_noalloc_block_update_matches_ordinary_path():
    cfg = Config(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=6.4, SSD_V_SIZE=5.0,
                 DROP_BLOCK_SIZE=3200, HISTORIES_PER_BLOCK=0, MLP_U_STEP=0.1)
    compare_two_blocks(cfg, 12000, 21, 3200)


def test_noalloc_odd_voxel_count_matches_ordinary_path():
    # 129 x 129 x 15 voxels: the image update's last voxel takes its single-voxel tail on the
    # caller's unpadded buffer
    cfg = Config(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=6.45, SSD_V_SIZE=4.75,
                 DROP_BLOCK_SIZE=3000, HISTORIES_PER_BLOCK=0, MLP_U_STEP=0.1)
    assert cfg.NUM_VOXELS % 2 == 1
    compare_two_blocks(cfg, 12000, 22, 3000)


def test_noalloc_argument_checks():
    base = dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=6.4, SSD_V_SIZE=5.0,
                DROP_BLOCK_SIZE=3200, HISTORIES_PER_BLOCK=0, MLP_U_STEP=0.1)
    lib = _abi.load_library()
    tracks = P.simulate_tracks(P.water_cylinder_phantom(6.0), 3000, seed=23)
    hist = {k: v.numpy() for k, v in P.reconstruction_histories(Config(**base), tracks).items()}
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in hist.items()}
    n = min(1000, len(hist["WEPL"]))
    for extra, word in ((dict(SCATTER_MODE="DETERMINISTIC"), b"ATOMIC"), (dict(PROJECTION_ALGORITHM="ROBUSTB"), b"DROP")):
        cfg = Config(**base, **extra)
        x = torch.ones(cfg.NUM_VOXELS + 2, dtype=torch.float32, device="cuda")
        with Context(cfg) as ctx:
            assert noalloc(lib, ctx, dev, 0, n, x.data_ptr()) == _abi.PCT_ERR_ARG
            assert word in lib.pct_last_error(ctx._h)
    cfg = Config(**base)
    x = torch.ones(cfg.NUM_VOXELS + 2, dtype=torch.float32, device="cuda")
    with Context(cfg) as ctx:
        # a pointer 4 bytes into the buffer: rejected before any kernel runs
        assert noalloc(lib, ctx, dev, 0, n, x.data_ptr() + 4) == _abi.PCT_ERR_ARG
        assert b"aligned" in lib.pct_last_error(ctx._h)
        # no histories: success, image untouched
        assert noalloc(lib, ctx, dev, 0, 0, x.data_ptr()) == _abi.PCT_OK
        ctx.synchronize()
        assert bool(torch.all(x == 1.0))
        # and a real call afterwards still works on the same context
        assert noalloc(lib, ctx, dev, 0, n, x.data_ptr()) == _abi.PCT_OK, lib.pct_last_error(ctx._h)
        ctx.synchronize()
        assert int((x[:cfg.NUM_VOXELS] != 1.0).sum()) > 100
        assert bool(torch.all(x[cfg.NUM_VOXELS:] == 1.0))


def test_noalloc_rejects_grids_beyond_its_static_accumulator():
    cfg = Config()  # the reference defaults: 256 x 256 x 32 = 2097152 voxels fit
    big = Config(COLUMNS=300, ROWS=300, SLICES=40)
    lib = _abi.load_library()
    with Context(big) as ctx:
        h = _abi.pct_histories()
        st = lib.pct_drop_block_update_noalloc(ctx._h, ctypes.byref(h), 0, ctypes.c_void_p(256))
        assert st == _abi.PCT_ERR_ARG
        assert b"static" in lib.pct_last_error(ctx._h)
    assert cfg.NUM_VOXELS <= 2359296
