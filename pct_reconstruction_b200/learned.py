"""Learned DROP initializer: host side of the encoder-decoder in libpct_b200.so (pct_unet_*).

The network, its training kernels and its inference run on the GPU behind the C ABI; this module
wraps them for torch CUDA tensors and holds the recipe that makes training pairs with the plain
pipeline: a synthetic phantom is scanned, preprocessed (FBP, hull, x_0 = FBP_median x hull) and
reconstructed by DROP; the pair is (x_0, hull) -> the DROP image after ITERATIONS iterations.
Starting DROP from the network's output instead of x_0 is pct_learned_initial_iterate; the FBP
start stays the fallback and the reference point for the learned start's error.
"""
from __future__ import annotations

import ctypes as C
import time
from pathlib import Path

import numpy as np

from . import _abi
from .engine import Config, Context, PCTError, _torch_fence

PARAMS_MAGIC = b"PCTUNET1"


def _ptr(t) -> int:
    return 0 if t is None else t.data_ptr()


def _stream(stream) -> C.c_void_p:
    return C.c_void_p(0 if stream is None else int(stream.cuda_stream))


class UNet:
    """The encoder-decoder for one grid (columns, rows, slices, each divisible by 8)."""

    def __init__(self, columns: int, rows: int, slices: int, seed: int = 0, device: int = 0):
        self.lib = _abi.load_library()
        self.shape = (slices, rows, columns)
        self._h = C.c_void_p()
        st = self.lib.pct_unet_create(columns, rows, slices, seed, device, C.byref(self._h))
        if st != _abi.PCT_OK:
            raise PCTError(st, "pct_unet_create")
        n = C.c_int64()
        self._chk(self.lib.pct_unet_param_count(self._h, C.byref(n)), "pct_unet_param_count")
        self.param_count = n.value

    def _chk(self, status, where):
        if status != _abi.PCT_OK:
            raise PCTError(status, where, self.lib.pct_unet_last_error(self._h).decode(errors="replace"))

    def close(self):
        if self._h:
            self.lib.pct_unet_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # parameters ---------------------------------------------------------------------------
    def get_params(self) -> np.ndarray:
        p = np.empty(self.param_count, np.float32)
        self._chk(self.lib.pct_unet_get_params(self._h, p.ctypes.data, self.param_count), "pct_unet_get_params")
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.param_count:
            raise ValueError(f"expected {self.param_count} parameters, got {p.size}")
        self._chk(self.lib.pct_unet_set_params(self._h, p.ctypes.data, self.param_count), "pct_unet_set_params")

    def save(self, path) -> None:
        p = self.get_params()
        with open(path, "wb") as f:
            f.write(PARAMS_MAGIC + np.int64(p.size).tobytes() + p.tobytes())

    def load(self, path) -> None:
        raw = Path(path).read_bytes()
        if raw[:8] != PARAMS_MAGIC:
            raise ValueError(f"{path}: not a network parameter file")
        n = int(np.frombuffer(raw[8:16], np.int64)[0])
        self.set_params(np.frombuffer(raw[16:16 + 4 * n], np.float32))

    # compute (torch CUDA tensors: x0 float32, hull uint8, target float32, each NUM_VOXELS) ----
    def forward(self, x0, hull, out=None):
        import torch
        if out is None:
            out = torch.empty_like(x0)
        _torch_fence(x0, hull, out)
        self._chk(self.lib.pct_unet_forward(self._h, C.c_void_p(_ptr(x0)), C.c_void_p(_ptr(hull)),
                                            C.c_void_p(_ptr(out))), "pct_unet_forward")
        return out

    def gradients(self, x0, hull, target):
        g = np.empty(self.param_count, np.float32)
        loss = C.c_double()
        _torch_fence(x0, hull, target)
        self._chk(self.lib.pct_unet_gradients(self._h, C.c_void_p(_ptr(x0)), C.c_void_p(_ptr(hull)),
                                              C.c_void_p(_ptr(target)), g.ctypes.data, C.byref(loss)),
                  "pct_unet_gradients")
        return loss.value, g

    def train_step(self, x0, hull, target, lr: float) -> float:
        loss = C.c_double()
        _torch_fence(x0, hull, target)
        self._chk(self.lib.pct_unet_train_step(self._h, C.c_void_p(_ptr(x0)), C.c_void_p(_ptr(hull)),
                                               C.c_void_p(_ptr(target)), C.c_float(lr), C.byref(loss)),
                  "pct_unet_train_step")
        return loss.value

    def initial_iterate(self, ctx: Context) -> None:
        """Replace the context's x_0 by the network's estimate (pct_learned_initial_iterate)."""
        ctx._chk(self.lib.pct_learned_initial_iterate(ctx._h, self._h), "pct_learned_initial_iterate")


def conv3d(inp, cin, shape, weight, cout, *, upsample=False, bias=None, residual=None, mask=None, relu=False,
           stream=None):
    """One network convolution (pct_conv3d_bf16) on channels-last bf16 CUDA tensors; shape is the
    output grid (slices, rows, columns)."""
    import torch
    lib = _abi.load_library()
    out = torch.empty(int(np.prod(shape)) * cout, dtype=torch.bfloat16, device=inp.device)
    st = lib.pct_conv3d_bf16(C.c_void_p(_ptr(inp)), cin, shape[2], shape[1], shape[0], int(bool(upsample)),
                             C.c_void_p(_ptr(weight)), cout, C.c_void_p(_ptr(bias)), C.c_void_p(_ptr(residual)),
                             C.c_void_p(_ptr(mask)), int(bool(relu)), C.c_void_p(_ptr(out)), _stream(stream))
    if st != _abi.PCT_OK:
        raise PCTError(st, "pct_conv3d_bf16")
    return out


def conv3d_wgrad(inp, cin, shape, dz, cout, *, upsample=False, stream=None):
    """Weight gradient of a network convolution (pct_conv3d_bf16_wgrad), fp32 [cout, 27, cin]."""
    import torch
    lib = _abi.load_library()
    dw = torch.zeros(cout * 27 * cin, dtype=torch.float32, device=inp.device)
    st = lib.pct_conv3d_bf16_wgrad(C.c_void_p(_ptr(inp)), cin, shape[2], shape[1], shape[0], int(bool(upsample)),
                                   C.c_void_p(_ptr(dz)), cout, C.c_void_p(_ptr(dw)), _stream(stream))
    if st != _abi.PCT_OK:
        raise PCTError(st, "pct_conv3d_bf16_wgrad")
    return dw


# -- training pairs from the plain pipeline ------------------------------------------------------

def scan_config(grid=(200, 200, 32), block_size=60000, iterations=12, **extra) -> dict:
    """Plain-pipeline parameters for a grid of 1 x 1 x 2.5 mm voxels (columns, rows, slices),
    with MSC and SM hulls as the head-size configuration uses them."""
    cols, rows, slices = grid
    assert cols == rows
    R = cols * 0.05
    p = dict(VOXEL_WIDTH=0.1, VOXEL_HEIGHT=0.1, VOXEL_THICKNESS=0.25, RECON_CYL_RADIUS=R,
             SSD_V_SIZE=slices * 0.25 + 1.0, T_BIN_SIZE=0.1, V_BIN_SIZE=0.25, ANGULAR_BIN_SIZE=4.0,
             DROP_BLOCK_SIZE=block_size, HISTORIES_PER_BLOCK=0, ITERATIONS=iterations, LAMBDA=0.0001,
             SC_ON=1, MSC_ON=1, SM_ON=1, SC_LOWER_THRESHOLD=-10.0, SC_UPPER_THRESHOLD=0.0, MSC_DIFF_THRESH=50)
    p.update(extra)
    return p


def scan_phantom(cfg, seed: int, histories: int, device):
    """Seeded random-ellipsoid phantom (RSP of the inserts uniform in [0.2, 1.8]) and its simulated
    tracker data with continuous gantry angles, as torch CUDA tensors."""
    import torch
    from . import phantoms as P
    R, H = cfg.RECON_CYL_RADIUS, cfg.RECON_CYL_HEIGHT
    ph = P.random_ellipsoid_phantom(seed, extent=(0.8 * R, 0.8 * R, 0.4 * H))
    parts, k = [], 0
    left = histories
    while left > 0:
        m = min(8_000_000, left)
        tr = P.simulate_tracks(ph, m, seed=seed * 1000 + k, device=device, continuous_angles=True,
                               t_extent=2.2 * R, v_extent=0.9 * H)
        parts.append(P.tracker_data(tr))
        left -= m
        k += 1
    td = {key: torch.cat([p_[key] for p_ in parts]).contiguous() for key in parts[0]}
    return ph, td


def reconstruct(cfg, tracker, iterations: int, unet: UNet | None = None, reference=None, tolerance=None):
    """Preprocess one scan and run DROP from x_0 (or, with unet, from the network's estimate).

    Returns a dict: x0 and hull (CUDA tensors), start (the first iterate), start_ms (host time of
    the network call, 0 without it), iteration_ms (host-timed DROP iterations, synchronised),
    images (each iteration's image when reference is None) or rel_rmse (relative RMSE inside the
    hull against reference, starting with the first iterate; stops early once below tolerance)."""
    import torch
    out = {"iteration_ms": [], "rel_rmse": [], "images": []}
    nv = cfg.NUM_VOXELS
    with Context(cfg) as ctx:
        ctx.preprocessing(tracker)
        hull = torch.from_numpy(ctx.get_array("hull").astype(np.uint8)).cuda()
        x0 = ctx.x_GPU_2_host(out=torch.empty(nv, dtype=torch.float32, device="cuda"))
        out["x0"], out["hull"] = x0, hull
        out["start_ms"] = 0.0
        if unet is not None:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            unet.initial_iterate(ctx)
            out["start_ms"] = (time.perf_counter() - t0) * 1e3
        start = ctx.x_GPU_2_host(out=torch.empty(nv, dtype=torch.float32, device="cuda"))
        out["start"] = start
        if reference is not None:
            out["rel_rmse"].append(rel_rmse(start, reference, hull))
        for it in range(1, iterations + 1):
            if reference is not None and tolerance is not None and out["rel_rmse"][-1] <= tolerance:
                break
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.DROP_full_tx_iteration(it)
            ctx.synchronize()
            out["iteration_ms"].append((time.perf_counter() - t0) * 1e3)
            x = ctx.x_GPU_2_host(out=torch.empty(nv, dtype=torch.float32, device="cuda"))
            if reference is not None:
                out["rel_rmse"].append(rel_rmse(x, reference, hull))
            else:
                out["images"].append(x)
        out["histories"] = ctx.reconstruction_histories
    return out


def rel_rmse(x, ref, hull) -> float:
    m = hull.bool()
    d = (x[m] - ref[m]).double()
    return float(d.pow(2).mean().sqrt() / ref[m].double().pow(2).mean().sqrt())


def make_pair(cfg, seed: int, histories: int, iterations: int, device):
    """One training pair from the plain pipeline: (x_0, hull) and the DROP image after
    `iterations` iterations from x_0, all CUDA tensors."""
    _, td = scan_phantom(cfg, seed, histories, device)
    out = reconstruct(cfg, td, iterations)
    return out["x0"], out["hull"], out["images"][-1]


def train(net: UNet, pairs, steps: int, lr: float = 1e-3, lr_end: float = 1e-5, seed: int = 0, log=None):
    """Adam over the pairs in a seeded random order, learning rate decayed geometrically from lr
    to lr_end.  Returns the per-step losses."""
    rng = np.random.default_rng(seed)
    losses = []
    order = []
    for s in range(steps):
        if not order:
            order = list(rng.permutation(len(pairs)))
        x0, hull, target = pairs[order.pop()]
        rate = lr * (lr_end / lr) ** (s / max(steps - 1, 1))
        losses.append(net.train_step(x0, hull, target, rate))
        if log and (s % 500 == 0 or s == steps - 1):
            log(f"step {s}: loss {np.mean(losses[-100:]):.3e} lr {rate:.2e}")
    return losses


def evaluate_scan(cfg, tracker, net: UNet, iterations: int, tolerance: float):
    """Both starts on one scan.  The reference image is the FBP-started DROP image after
    `iterations` iterations; for each start, the relative RMSE inside the hull after every
    iteration, the iterations and the device-synchronised wall time (ms) it takes to come within
    `tolerance` of the reference (network call included for the learned start; None if never)."""
    import torch
    nv = cfg.NUM_VOXELS
    res = {}
    with Context(cfg) as ctx:
        ctx.preprocessing(tracker)
        hull = torch.from_numpy(ctx.get_array("hull").astype(np.uint8)).cuda()
        x0 = ctx.x_GPU_2_host(out=torch.empty(nv, dtype=torch.float32, device="cuda"))
        # one-time setup (path layout, graph capture, the network's first call) outside the timing
        ctx.DROP_full_tx_iteration(1)
        net.forward(x0, hull)
        ctx.x_host_2_GPU(x0)
        images, times = [x0.clone()], [0.0]
        for it in range(1, iterations + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.DROP_full_tx_iteration(it)
            ctx.synchronize()
            times.append((time.perf_counter() - t0) * 1e3)
            images.append(ctx.x_GPU_2_host(out=torch.empty(nv, dtype=torch.float32, device="cuda")))
        ref = images[-1]
        res["fbp"] = {"rel_rmse": [rel_rmse(x, ref, hull) for x in images], "iteration_ms": times[1:]}
        # learned start on the same preprocessed scan
        ctx.x_host_2_GPU(x0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        net.initial_iterate(ctx)
        torch.cuda.synchronize()
        start_ms = (time.perf_counter() - t0) * 1e3
        x = ctx.x_GPU_2_host(out=torch.empty(nv, dtype=torch.float32, device="cuda"))
        errs, ltimes = [rel_rmse(x, ref, hull)], [start_ms]
        for it in range(1, iterations + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.DROP_full_tx_iteration(it)
            ctx.synchronize()
            ltimes.append((time.perf_counter() - t0) * 1e3)
            errs.append(rel_rmse(ctx.x_GPU_2_host(out=torch.empty(nv, dtype=torch.float32, device="cuda")), ref, hull))
        res["learned"] = {"rel_rmse": errs, "iteration_ms": ltimes[1:], "start_ms": start_ms}
        res["histories"] = ctx.reconstruction_histories
    for key, extra in (("fbp", 0.0), ("learned", res["learned"]["start_ms"])):
        r = res[key]
        k = next((i for i, e in enumerate(r["rel_rmse"]) if e <= tolerance), None)
        r["iterations_to_tolerance"] = k
        r["ms_to_tolerance"] = None if k is None else extra + float(sum(r["iteration_ms"][:k]))
    return res


def evaluate_scan_truth(cfg, phantom, tracker, net: UNet, iterations: int):
    """Both starts on one scan, judged against the phantom's true RSP (sampled at the voxel
    centres, phantoms.truth_image), inside the hull -- a target the network was not trained on
    (its training target is the FBP-started DROP image).  For each start: the relative RMSE to
    the truth of the start and after every DROP iteration, and the device-synchronised wall time of
    each iteration (the learned start adds its network call).  The common error level is the
    larger of the two starts' best errors over the iterations, so both starts reach it; the time to
    reach it is reported for each start, next to both starts' error after the last iteration."""
    import torch
    from . import phantoms as P
    nv = cfg.NUM_VOXELS
    truth = P.truth_image(cfg, phantom, device="cuda")
    res = {}
    with Context(cfg) as ctx:
        ctx.preprocessing(tracker)
        hull = torch.from_numpy(ctx.get_array("hull").astype(np.uint8)).cuda()
        x0 = ctx.x_GPU_2_host(out=torch.empty(nv, dtype=torch.float32, device="cuda"))
        ctx.DROP_full_tx_iteration(1)  # one-time path layout and graph capture, outside the timing
        net.forward(x0, hull)          # the network's first call, outside the timing
        for key in ("fbp", "learned"):
            ctx.x_host_2_GPU(x0)
            start_ms = 0.0
            if key == "learned":
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                net.initial_iterate(ctx)
                torch.cuda.synchronize()
                start_ms = (time.perf_counter() - t0) * 1e3
            x = ctx.x_GPU_2_host(out=torch.empty(nv, dtype=torch.float32, device="cuda"))
            errs, times = [rel_rmse(x, truth, hull)], []
            for it in range(1, iterations + 1):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                ctx.DROP_full_tx_iteration(it)
                ctx.synchronize()
                times.append((time.perf_counter() - t0) * 1e3)
                errs.append(rel_rmse(ctx.x_GPU_2_host(out=torch.empty(nv, dtype=torch.float32, device="cuda")),
                                     truth, hull))
            res[key] = {"rel_rmse_to_truth": errs, "iteration_ms": times, "start_ms": start_ms}
        res["histories"] = ctx.reconstruction_histories
    level = max(min(res["fbp"]["rel_rmse_to_truth"]), min(res["learned"]["rel_rmse_to_truth"]))
    res["common_level"] = level
    for key in ("fbp", "learned"):
        r = res[key]
        k = next(i for i, e in enumerate(r["rel_rmse_to_truth"]) if e <= level)
        r["iterations_to_level"] = k
        r["ms_to_level"] = r["start_ms"] + float(sum(r["iteration_ms"][:k]))
        r["final_rel_rmse_to_truth"] = r["rel_rmse_to_truth"][-1]
    return res
