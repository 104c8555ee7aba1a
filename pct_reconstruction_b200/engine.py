"""Python host API over the C ABI (include/pct_api.h).

Mirrors the reference's stage names (DROP_GPU, DROP_full_tx_iteration, x_host_2_GPU, ...)
so a caller of the reference finds the same steps.  Arrays may be numpy arrays (host memory) or
torch CUDA tensors (device memory); every call goes through libpct_b200.so.
"""
from __future__ import annotations

import ctypes as C
from typing import Mapping

import numpy as np

from . import _abi
from ._abi import (HISTORY_FIELDS, PCT_DEVICE, PCT_HOST, PCT_MLP_PATH_CAP, PROJECTION_FIELDS, TRACKER_FIELDS,
                   pct_config, pct_histories, pct_projection_arrays, pct_projection_header, pct_tracker_data)

# element types of the named arrays that are not float32
_ARRAY_DTYPES = {"missed_recon_volume": np.uint8, "SC_hull": np.uint8, "FBP_hull": np.uint8, "hull": np.uint8,
                 "bin_num": np.int32, "bin_num_vector": np.int32, "bin_counts": np.int32, "MSC_counts": np.int32,
                 "SM_counts": np.int32, "first_MLP_voxel_vector": np.uint32,
                 "first_MLP_voxel_reconstruction": np.uint32}


class PCTError(RuntimeError):
    def __init__(self, status: int, where: str, message: str = ""):
        lib = _abi.load_library()
        name = lib.pct_status_string(status).decode()
        super().__init__(f"{where}: {name}" + (f" ({message})" if message else ""))
        self.status = status


def _check(status: int, where: str, ctx=None, config=False):
    if status != _abi.PCT_OK:
        msg = ""
        if ctx:
            msg = _abi.load_library().pct_last_error(ctx).decode(errors="replace")
        elif config:
            msg = _abi.load_library().pct_config_last_error().decode(errors="replace")
        raise PCTError(status, where, msg)


# -- projection data files (PCTD / PCTN, versions 0 and 1) -----------------------------------
_HEADER_SCALARS = ("continuous", "version", "num_histories", "projection_angle", "beam_energy",
                   "generation_date", "preprocess_date", "has_angles", "data_offset")
_HEADER_STRINGS = ("phantom_name", "data_source", "prepared_by")


def _header_dict(h: pct_projection_header) -> dict:
    d = {k: getattr(h, k) for k in _HEADER_SCALARS}
    d.update({k: getattr(h, k).decode(errors="replace") for k in _HEADER_STRINGS})
    return d


def projection_file_name(angle: int) -> str:
    """File name of one gantry angle's projection data (B.h:596-597)."""
    return f"projection_{int(angle):03d}.bin"


def read_projection_header(path) -> dict:
    """Header of one projection data file (count_histories_v0, B.cu:3578)."""
    h = pct_projection_header()
    _check(_abi.load_library().pct_read_projection_header(str(path).encode(), C.byref(h)),
           f"pct_read_projection_header({path})")
    return _header_dict(h)


def read_projection_file(path) -> tuple[dict, dict]:
    """(header, arrays) of one file in file units (mm); arrays keyed by pct_projection_arrays names."""
    lib = _abi.load_library()
    hdr = read_projection_header(path)
    n = hdr["num_histories"]
    arrays = {k: np.empty(n, np.float32) for k in PROJECTION_FIELDS[:-1]}
    if hdr["has_angles"]:
        arrays["projection_angle"] = np.empty(n, np.float32)
    s = pct_projection_arrays(*[C.c_void_p(arrays[k].ctypes.data) if k in arrays else C.c_void_p(0)
                                for k in PROJECTION_FIELDS])
    h = pct_projection_header()
    _check(lib.pct_read_projection_file(str(path).encode(), n, C.byref(s), C.byref(h)),
           f"pct_read_projection_file({path})")
    return _header_dict(h), arrays


def write_projection_file(path, arrays: Mapping[str, object], projection_angle: float, *, continuous: bool = False,
                          version: int = 0, beam_energy: float = 200.0, generation_date: int = 0,
                          preprocess_date: int = 0, phantom_name: str = "", data_source: str = "",
                          prepared_by: str = "") -> None:
    """Write one projection data file; arrays in mm, "projection_angle" (per history) optional."""
    keep = {k: _host_array(arrays[k], np.float32) for k in PROJECTION_FIELDS if k in arrays}
    n = len(keep["WEPL"])
    h = pct_projection_header(continuous=int(bool(continuous)), version=version, projection_angle=projection_angle,
                              beam_energy=beam_energy, generation_date=generation_date,
                              preprocess_date=preprocess_date, phantom_name=phantom_name.encode()[:255],
                              data_source=data_source.encode()[:255], prepared_by=prepared_by.encode()[:255])
    s = pct_projection_arrays(*[C.c_void_p(keep[k].ctypes.data) if k in keep else C.c_void_p(0)
                                for k in PROJECTION_FIELDS])
    _check(_abi.load_library().pct_write_projection_file(str(path).encode(), C.byref(h), C.byref(s), n),
           f"pct_write_projection_file({path})")


class Config:
    """Runtime configuration with the reference's parameter names (B.h / settings.cfg keys)."""

    def __init__(self, path: str | None = None, **params):
        lib = _abi.load_library()
        self._c = pct_config()
        lib.pct_config_default(C.byref(self._c))
        if path is not None:
            _check(lib.pct_config_load(C.byref(self._c), str(path).encode()), f"pct_config_load({path})", config=True)
        for k, v in params.items():
            self.set(k, v)
        self.finalize()

    def set(self, key: str, value) -> None:
        if isinstance(value, bool):
            value = int(value)
        s = repr(float(value)) if isinstance(value, float) else str(value)
        _check(_abi.load_library().pct_config_set(C.byref(self._c), key.encode(), s.encode()),
               f"pct_config_set({key}={value})", config=True)

    def finalize(self) -> None:
        _check(_abi.load_library().pct_config_finalize(C.byref(self._c)), "pct_config_finalize", config=True)

    def __getattr__(self, name):
        c = self.__dict__.get("_c")
        if c is not None and name in dict(_abi.CONFIG_FIELDS):
            return getattr(c, name)
        raise AttributeError(name)

    def as_dict(self) -> dict:
        return {k: getattr(self._c, k) for k, _ in _abi.CONFIG_FIELDS if not k.startswith("pad")}

    @property
    def struct(self) -> pct_config:
        return self._c


def _is_cuda_tensor(a) -> bool:
    return hasattr(a, "is_cuda") and a.is_cuda


def _torch_fence(*arrays) -> bool:
    """The library reads and writes CUDA tensors on the context's own stream, which is not ordered
    with torch's streams.  When any argument is a CUDA tensor, wait for the work torch has queued on
    its device (the kernels that produced or still use the tensor) before the library touches it.
    Returns whether a CUDA tensor was seen."""
    for a in arrays:
        if _is_cuda_tensor(a):
            import torch
            torch.cuda.current_stream(a.device).synchronize()
            return True
    return False


def _ptr(a) -> int:
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def _host_array(a, dtype) -> np.ndarray:
    """Contiguous host view (no copy when the layout already fits; signed/unsigned 32-bit
    integers are reinterpreted, so pinned buffers stay pinned)."""
    if hasattr(a, "detach"):
        a = a.detach().cpu().numpy()
    a = np.asarray(a)
    dt = np.dtype(dtype)
    if a.dtype != dt and a.dtype.kind in "iu" and dt.kind in "iu" and a.dtype.itemsize == dt.itemsize:
        a = a.view(dt)
    return np.ascontiguousarray(a, dtype=dt)


class Context:
    """One reconstruction context on one CUDA device (pct_create / pct_destroy)."""

    def __init__(self, config: Config, device: int = 0):
        self.lib = _abi.load_library()
        self.config = config
        h = C.c_void_p()
        st = self.lib.pct_create(C.byref(config.struct), int(device), C.byref(h))
        if st != _abi.PCT_OK:  # the context is gone; pct_last_error(NULL) holds the reason
            raise PCTError(st, "pct_create", self.lib.pct_last_error(None).decode(errors="replace"))
        self._h = h
        self._keep = []  # keeps host arrays alive across async copies

    # -- lifetime -------------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self.lib.pct_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, status, where):
        _check(status, where, self._h)

    def set_stream(self, stream_ptr: int | None):
        self._chk(self.lib.pct_set_stream(self._h, C.c_void_p(stream_ptr or 0)), "pct_set_stream")

    def synchronize(self):
        self._chk(self.lib.pct_synchronize(self._h), "pct_synchronize")

    # -- data -----------------------------------------------------------------------------
    def set_reconstruction_histories(self, hist: Mapping[str, object]) -> int:
        """Load the DROP-stage arrays (dict with the pct_histories field names)."""
        arrays = [hist[k] for k in HISTORY_FIELDS]
        n = len(arrays[0])
        if any(len(a) != n for a in arrays):
            raise ValueError("history arrays differ in length")
        on_device = _is_cuda_tensor(arrays[0])
        if on_device:
            if not all(_is_cuda_tensor(a) and a.is_contiguous() for a in arrays):
                raise ValueError("mixed host/device or non-contiguous history arrays")
            keep = arrays
            _torch_fence(*arrays)
        else:
            keep = [_host_array(a, np.uint32 if k == "first_MLP_voxel" else np.float32)
                    for k, a in zip(HISTORY_FIELDS, arrays)]
        s = pct_histories(*[C.c_void_p(_ptr(a)) for a in keep])
        self._chk(self.lib.pct_set_reconstruction_histories(self._h, C.byref(s), n,
                                                            PCT_DEVICE if on_device else PCT_HOST),
                  "pct_set_reconstruction_histories")
        self.synchronize()  # the caller's arrays may be freed or reused after return
        return n

    def stage_reconstruction_histories(self, hist: Mapping[str, object]) -> int:
        """Start uploading the next set of histories on the copy stream (returns at once; the
        current histories stay in use).  Host arrays should be pinned to overlap; they are kept
        referenced here until two later stage calls have been made."""
        arrays = [hist[k] for k in HISTORY_FIELDS]
        n = len(arrays[0])
        if any(len(a) != n for a in arrays):
            raise ValueError("history arrays differ in length")
        on_device = _is_cuda_tensor(arrays[0])
        if on_device:
            keep = arrays
            _torch_fence(*arrays)
        else:
            keep = [_host_array(a, np.uint32 if k == "first_MLP_voxel" else np.float32)
                    for k, a in zip(HISTORY_FIELDS, arrays)]
        s = pct_histories(*[C.c_void_p(_ptr(a)) for a in keep])
        self._chk(self.lib.pct_stage_reconstruction_histories(self._h, C.byref(s), n,
                                                              PCT_DEVICE if on_device else PCT_HOST),
                  "pct_stage_reconstruction_histories")
        self._staged_refs = (getattr(self, "_staged_refs", ())[-1:]) + (keep,)
        return n

    def use_staged_histories(self) -> None:
        """Make the staged histories the reconstruction histories (pct_use_staged_histories)."""
        self._chk(self.lib.pct_use_staged_histories(self._h), "pct_use_staged_histories")

    @property
    def reconstruction_histories(self) -> int:
        return int(self.lib.pct_reconstruction_histories(self._h))

    def apply_history_sequence(self, prime_offset: int) -> None:
        """Prime-permutation reconstruction order (apply_history_sequence)."""
        self._chk(self.lib.pct_apply_history_sequence(self._h, int(prime_offset)), "pct_apply_history_sequence")

    def x_host_2_GPU(self, x) -> None:
        """Set the image (NUM_VOXELS float32; numpy or CUDA tensor)."""
        if _torch_fence(x):
            self._chk(self.lib.pct_set_image(self._h, C.c_void_p(_ptr(x)), PCT_DEVICE), "pct_set_image")
            self.synchronize()
        else:
            a = _host_array(x, np.float32)
            if a.size != self.config.NUM_VOXELS:
                raise ValueError("image size != NUM_VOXELS")
            self._chk(self.lib.pct_set_image(self._h, C.c_void_p(a.ctypes.data), PCT_HOST), "pct_set_image")

    set_image = x_host_2_GPU

    def x_GPU_2_host(self, out=None):
        """Return the image (numpy float32), or copy it into a CUDA tensor `out`."""
        if out is not None and _torch_fence(out):
            self._chk(self.lib.pct_get_image(self._h, C.c_void_p(_ptr(out)), PCT_DEVICE), "pct_get_image")
            self.synchronize()
            return out
        a = np.empty(self.config.NUM_VOXELS, dtype=np.float32)
        self._chk(self.lib.pct_get_image(self._h, C.c_void_p(a.ctypes.data), PCT_HOST), "pct_get_image")
        return a

    get_image = x_GPU_2_host

    # -- DROP -----------------------------------------------------------------------------
    def DROP_full_tx_iteration(self, iteration: int = 1) -> None:
        self._chk(self.lib.pct_drop_full_tx_iteration(self._h, int(iteration)), "pct_drop_full_tx_iteration")

    def DROP_GPU(self) -> None:
        self._chk(self.lib.pct_drop_gpu(self._h), "pct_drop_gpu")

    # -- total variation superiorization -----------------------------------------------------
    def NTVS_iteration(self, iteration: int) -> None:
        """NTVS on the device image before/after DROP iteration `iteration` (1-based)."""
        self._chk(self.lib.pct_ntvs_iteration(self._h, int(iteration)), "pct_ntvs_iteration")

    def total_variation(self) -> float:
        tv = C.c_double(0.0)
        self._chk(self.lib.pct_total_variation(self._h, C.byref(tv)), "pct_total_variation")
        return tv.value

    @property
    def tvs_L(self) -> int:
        L = C.c_int32(0)
        self._chk(self.lib.pct_tvs_L(self._h, C.byref(L), None), "pct_tvs_L")
        return L.value

    @tvs_L.setter
    def tvs_L(self, value: int) -> None:
        L = C.c_int32(int(value))
        self._chk(self.lib.pct_tvs_L(self._h, None, C.byref(L)), "pct_tvs_L")

    def profile_drop_iteration(self) -> dict:
        """One DROP iteration with per-launch CUDA events; summed ms and launch counts per group."""
        ms = (C.c_double * 3)()
        nl = (C.c_int64 * 3)()
        self._chk(self.lib.pct_profile_drop_iteration(self._h, ms, nl), "pct_profile_drop_iteration")
        names = ("path", "block", "update")
        return {k: {"ms": ms[i], "launches": nl[i]} for i, k in enumerate(names)}

    def set_path_storage_limit(self, nbytes: int) -> None:
        """0: automatic, > 0: byte cap, < 0: no path storage (single-pass kernel)."""
        self._chk(self.lib.pct_set_path_storage_limit(self._h, int(nbytes)), "pct_set_path_storage_limit")

    def autotune(self) -> int:
        """Pick the fastest schedule for the loaded histories (pct_autotune); returns the chosen
        PATH_CHUNK_BLOCKS."""
        out = C.c_int32()
        self._chk(self.lib.pct_autotune(self._h, C.byref(out)), "pct_autotune")
        return out.value

    def autotune_schedule(self) -> dict:
        """Pick the fastest PATH_CHUNK_BLOCKS, PATH_CTA_THREADS and PATH_ORDER_WINDOW for the
        loaded histories (pct_autotune_schedule); returns the three."""
        out = (C.c_int32 * 3)()
        self._chk(self.lib.pct_autotune_schedule(self._h, out), "pct_autotune_schedule")
        return {"PATH_CHUNK_BLOCKS": out[0], "PATH_CTA_THREADS": out[1], "PATH_ORDER_WINDOW": out[2]}

    def set_l2_window(self, enable: bool) -> None:
        """Keep the image and accumulator in persisting L2 lines during DROP (pct_set_l2_window)."""
        self._chk(self.lib.pct_set_l2_window(self._h, int(bool(enable))), "pct_set_l2_window")

    def set_path_reuse(self, enable: bool) -> None:
        """Precomputed-path DROP: keep the MLP paths of the first iteration for the later ones."""
        self._chk(self.lib.pct_set_path_reuse(self._h, int(bool(enable))), "pct_set_path_reuse")

    @property
    def path_storage_superblocks(self) -> int:
        return int(self.lib.pct_path_storage_superblocks(self._h))

    def calculate_x_update(self, start_position: int, num_histories: int) -> None:
        """One block's MLP + scatter launch (no synchronisation)."""
        self._chk(self.lib.pct_calculate_x_update(self._h, int(start_position), int(num_histories)),
                  "pct_calculate_x_update")

    def image_update(self) -> None:
        self._chk(self.lib.pct_image_update(self._h), "pct_image_update")

    def mlp_paths(self, start: int = 0, n: int | None = None, stride: int = PCT_MLP_PATH_CAP):
        """MLP voxel lists (host numpy): counts[n], voxels[n, stride], chord[n], a_dot_x[n]."""
        if n is None:
            n = self.reconstruction_histories - start
        counts = np.zeros(n, np.uint32)
        voxels = np.zeros((n, stride), np.uint32)
        chord = np.zeros(n, np.float64)
        adx = np.zeros(n, np.float64)
        self._chk(self.lib.pct_mlp_paths(self._h, start, n, stride, counts.ctypes.data, voxels.ctypes.data,
                                         chord.ctypes.data, adx.ctypes.data, PCT_HOST), "pct_mlp_paths")
        return counts, voxels, chord, adx

    def mlp_precision(self, start: int = 0, n: int | None = None):
        """Exact vs mixed-precision MLP points: per history max |dt|, |dv| (cm) and mismatched
        steps over the well-posed steps, and the number of ill-posed steps."""
        if n is None:
            n = self.reconstruction_histories - start
        dt, dv = np.zeros(n), np.zeros(n)
        mm, ip = np.zeros(n, np.int32), np.zeros(n, np.int32)
        self._chk(self.lib.pct_mlp_precision(self._h, start, n, dt.ctypes.data, dv.ctypes.data, mm.ctypes.data,
                                             ip.ctypes.data, PCT_HOST), "pct_mlp_precision")
        return dt, dv, mm, ip

    def mlp_steps_device(self, start, n, steps):
        """MLP points (loop trips) per history into a CUDA int32 tensor (pct_mlp_steps)."""
        _torch_fence(steps)
        self._chk(self.lib.pct_mlp_steps(self._h, start, n, C.c_void_p(_ptr(steps)), PCT_DEVICE), "pct_mlp_steps")
        self.synchronize()

    def mlp_paths_device(self, start, n, stride, counts, voxels, chord, a_dot_x):
        """Device-memory form of mlp_paths (CUDA tensors, any may be None)."""
        p = lambda t: C.c_void_p(_ptr(t)) if t is not None else C.c_void_p(0)
        _torch_fence(counts, voxels, chord, a_dot_x)
        self._chk(self.lib.pct_mlp_paths(self._h, start, n, stride, p(counts), p(voxels), p(chord), p(a_dot_x),
                                         PCT_DEVICE), "pct_mlp_paths")
        self.synchronize()

    # -- preprocessing ----------------------------------------------------------------------
    def load_tracker_data(self, tracker: Mapping[str, object], integer_angles: bool = False) -> int:
        """Tracker hits (dict with pct_tracker_data field names; numpy or CUDA tensors)."""
        arrays = [tracker[k] for k in TRACKER_FIELDS]
        n = len(arrays[0])
        on_device = _is_cuda_tensor(arrays[0])
        keep = arrays if on_device else [_host_array(a, np.float32) for a in arrays]
        _torch_fence(*keep)
        s = pct_tracker_data(*[C.c_void_p(_ptr(a)) for a in keep])
        self._chk(self.lib.pct_load_tracker_data(self._h, C.byref(s), n, PCT_DEVICE if on_device else PCT_HOST,
                                                 int(bool(integer_angles))), "pct_load_tracker_data")
        if on_device:
            self.synchronize()
        return n

    def load_projection_data(self, directory) -> int:
        """Read a scan's projection files into the tracker arrays (count_histories + read_data_chunk)."""
        n = C.c_int64(0)
        self._chk(self.lib.pct_load_projection_data(self._h, str(directory).encode(), C.byref(n)),
                  "pct_load_projection_data")
        return int(n.value)

    def preprocessing_from_files(self, directory) -> int:
        """preprocessing() from a scan's files; returns the number of reconstruction histories."""
        self._chk(self.lib.pct_preprocessing_from_files(self._h, str(directory).encode()),
                  "pct_preprocessing_from_files")
        return self.reconstruction_histories

    def export_preprocessed(self, directory) -> None:
        """Write histories, MLP paths, chords, image and hull (accumulate_and_export_preprocessed_data)."""
        self._chk(self.lib.pct_export_preprocessed(self._h, str(directory).encode()), "pct_export_preprocessed")

    def import_preprocessed(self, directory) -> int:
        """Load what export_preprocessed wrote; returns the number of reconstruction histories."""
        self._chk(self.lib.pct_import_preprocessed(self._h, str(directory).encode()), "pct_import_preprocessed")
        return self.reconstruction_histories

    def set_history_vectors(self, hist: Mapping[str, object]) -> int:
        arrays = [hist[k] for k in HISTORY_FIELDS[:-1]]
        n = len(arrays[0])
        keep = [_host_array(a, np.float32) for a in arrays] + [np.zeros(1, np.uint32)]
        s = pct_histories(*[C.c_void_p(_ptr(a)) for a in keep])
        self._chk(self.lib.pct_set_history_vectors(self._h, C.byref(s), n, PCT_HOST), "pct_set_history_vectors")
        return n

    def preprocessing(self, tracker: Mapping[str, object], integer_angles: bool = False) -> int:
        """The whole preprocessing chain; returns the number of reconstruction histories."""
        arrays = [tracker[k] for k in TRACKER_FIELDS]
        n = len(arrays[0])
        on_device = _is_cuda_tensor(arrays[0])
        keep = arrays if on_device else [_host_array(a, np.float32) for a in arrays]
        _torch_fence(*keep)
        s = pct_tracker_data(*[C.c_void_p(_ptr(a)) for a in keep])
        self._chk(self.lib.pct_preprocessing(self._h, C.byref(s), n, PCT_DEVICE if on_device else PCT_HOST,
                                             int(bool(integer_angles))), "pct_preprocessing")
        return self.reconstruction_histories

    def stage(self, name: str) -> None:
        """Run one preprocessing stage by its reference name (e.g. "binning", "FBP")."""
        self._chk(getattr(self.lib, "pct_" + name)(self._h), "pct_" + name)

    def get_array(self, name: str) -> np.ndarray:
        n = int(self.lib.pct_array_length(self._h, name.encode()))
        if n < 0:
            raise KeyError(name)
        a = np.empty(n, _ARRAY_DTYPES.get(name, np.float32))
        self._chk(self.lib.pct_get_array(self._h, name.encode(), C.c_void_p(a.ctypes.data), a.nbytes, PCT_HOST),
                  f"pct_get_array({name})")
        return a

    def set_array(self, name: str, values) -> None:
        a = _host_array(values, _ARRAY_DTYPES.get(name, np.float32))
        self._chk(self.lib.pct_set_array(self._h, name.encode(), C.c_void_p(a.ctypes.data), a.nbytes, PCT_HOST),
                  f"pct_set_array({name})")

    # -- diagnostics ----------------------------------------------------------------------
    def counters(self) -> dict:
        arr = (C.c_int64 * 4)()
        self._chk(self.lib.pct_get_counters(self._h, arr), "pct_get_counters")
        return {"voxel_oob": arr[0], "path_overflow": arr[1], "table_range": arr[2], "wait_expired": arr[3]}

    def reset_counters(self):
        self._chk(self.lib.pct_reset_counters(self._h), "pct_reset_counters")

    def s_curve(self, count: int = PCT_MLP_PATH_CAP) -> np.ndarray:
        """The S-curve scale s(k) for k < count (S_CURVE_ON configurations)."""
        out = np.zeros(count, np.float32)
        self._chk(self.lib.pct_get_s_curve(self._h, C.c_void_p(out.ctypes.data), count), "pct_get_s_curve")
        return out

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.pct_kernel_launches(self._h))


class Batch:
    """Several scans' contexts run as one graph per DROP iteration (pct_batch_*)."""

    def __init__(self, contexts):
        self.lib = _abi.load_library()
        self.contexts = list(contexts)  # keeps the contexts alive as long as the batch
        arr = (C.c_void_p * len(self.contexts))(*[c._h for c in self.contexts])
        h = C.c_void_p()
        _check(self.lib.pct_batch_create(arr, len(self.contexts), C.byref(h)), "pct_batch_create")
        self._h = h

    def _chk(self, status, where):
        if status != _abi.PCT_OK:
            raise PCTError(status, where, self.lib.pct_batch_last_error(self._h).decode(errors="replace"))

    def DROP_iteration(self, iteration: int = 1) -> None:
        self._chk(self.lib.pct_batch_drop_iteration(self._h, int(iteration)), "pct_batch_drop_iteration")

    def synchronize(self) -> None:
        self._chk(self.lib.pct_batch_synchronize(self._h), "pct_batch_synchronize")

    @property
    def stream(self) -> int:
        return int(self.lib.pct_batch_stream(self._h) or 0)

    def close(self):
        if getattr(self, "_h", None):
            self.lib.pct_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

