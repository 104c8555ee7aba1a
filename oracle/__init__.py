"""ctypes wrapper of the CPU oracle (oracle/pct_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() (to compare against) and by
bench.py's CPU-baseline leg.  The engine never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "build" / "libpct_oracle.so"


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


class _Tables(C.Structure):
    _fields_ = [("trig_elements", C.c_int), ("coeff_elements", C.c_int), ("poly_elements", C.c_int)] + [
        (n, C.POINTER(C.c_double)) for n in ("sin_table", "cos_table", "scattering_table", "poly_1_2",
                                             "poly_2_3", "poly_3_4", "poly_2_6", "poly_3_12")]


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
        P = C.c_void_p
        _lib.oracle_tables_build.argtypes = [P, C.POINTER(_Tables)]
        _lib.oracle_tables_free.argtypes = [C.POINTER(_Tables)]
        _lib.oracle_a_coefficients.argtypes = [C.POINTER(C.c_double)]
        _lib.oracle_effective_chord_length.argtypes = [P, C.c_double, C.c_double]
        _lib.oracle_effective_chord_length.restype = C.c_double
        _lib.oracle_mlp_paths.argtypes = [P, C.POINTER(_Tables), P, P, C.c_int64, C.c_int64, C.c_int32,
                                          P, P, P, P, P]
        _lib.oracle_drop_iteration.argtypes = [P, C.POINTER(_Tables), P, C.c_int64, P, P, P, P]
        _lib.oracle_s_curve_table.argtypes = [P, C.c_int32, P]
        _lib.oracle_host_drop_iteration.argtypes = [P, P, C.c_int64, P, C.c_int]
        _lib.oracle_host_drop_iteration.restype = C.c_int64
        _lib.oracle_host_effective_chord_length.argtypes = [P, C.c_float, C.c_float]
        _lib.oracle_host_effective_chord_length.restype = C.c_float
        _lib.oracle_host_mlp_paths.argtypes = [P, P, C.c_int64, C.c_int64, C.c_int32, P, P, P]
        _lib.oracle_host_mlp_paths.restype = None
        _lib.oracle_fast_point_check.argtypes = [P, C.POINTER(_Tables), P, C.c_int64, P]
        _lib.oracle_fast_point_check.restype = None
        _lib.oracle_guarded_indices.argtypes = [P, C.c_int64, P, P, P, C.c_double, P, P]
        _lib.oracle_guarded_indices.restype = None
        I64, I32 = C.c_int64, C.c_int
        sigs = {
            "oracle_recon_volume_intersections": [P, I64, P, P, I32, P, P],
            "oracle_binning": [P, I64, P, P, P, P, P, P, P, P],
            "oracle_statistics_and_cuts": [P, I64, P, P, P, P, P, P, P, P, P, P, P, P],
            "oracle_sinogram_filter": [P, P, P, P],
            "oracle_backprojection": [P, P, P],
            "oracle_median_filter": [P, I32, P, P],
            "oracle_initialize_hull": [P, P],
            "oracle_edge_detection": [P, I32, P],
            "oracle_collect_mlp_endpoints": [P, P, I64, P, P],
        }
        for name, args in sigs.items():
            getattr(_lib, name).restype = None
            getattr(_lib, name).argtypes = args
        _lib.oracle_hull_walks.restype = C.c_int64
        _lib.oracle_hull_walks.argtypes = [P, I32, I64, P, P, P, P]
        _lib.oracle_tvs_randi.argtypes = [I32, I32, C.c_uint64, I32]
        _lib.oracle_tvs_eta.argtypes = [P, P, I32]
        _lib.oracle_total_variation.argtypes = [P, P, I32]
        _lib.oracle_total_variation.restype = C.c_double
        _lib.oracle_tvs_direction.argtypes = [P, P, P, P, P, I32]
        _lib.oracle_tvs_direction.restype = None
        _lib.oracle_ntvs_iteration.argtypes = [P, P, P, I32, C.POINTER(C.c_int), I32, P, I32]
        _lib.oracle_trig_table_min.restype = C.c_double
        _lib.oracle_trig_table_step.restype = C.c_double
    return _lib


HISTORY_FIELDS = ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit", "xy_entry_angle",
                  "xz_entry_angle", "xy_exit_angle", "xz_exit_angle", "WEPL", "first_MLP_voxel")


class _Hist(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in HISTORY_FIELDS]


def _host(a, dtype):
    if hasattr(a, "detach"):
        a = a.detach().cpu().numpy()
    return np.ascontiguousarray(a).view(dtype) if np.asarray(a).dtype.itemsize == np.dtype(dtype).itemsize \
        else np.ascontiguousarray(a, dtype=dtype)


class Oracle:
    """CPU restatement of the reference hot path for one configuration (a pct_config struct)."""

    def __init__(self, cfg_struct):
        self.lib = _load()
        self.cfg = cfg_struct
        self.tab = _Tables()
        if self.lib.oracle_tables_build(C.byref(cfg_struct), C.byref(self.tab)) != 0:
            raise MemoryError("oracle tables")
        nv = cfg_struct.NUM_VOXELS
        self.npad = nv + cfg_struct.COLUMNS * cfg_struct.ROWS

    def __del__(self):
        try:
            self.lib.oracle_tables_free(C.byref(self.tab))
        except Exception:
            pass

    def _hist(self, hist):
        arrs = [_host(hist[k], np.uint32 if k == "first_MLP_voxel" else np.float32) for k in HISTORY_FIELDS]
        return arrs, _Hist(*[a.ctypes.data for a in arrs])

    def padded_image(self, x) -> np.ndarray:
        xp = np.zeros(self.npad, np.float32)
        xp[: self.cfg.NUM_VOXELS] = _host(x, np.float32)
        return xp

    def a_coefficients(self):
        a = (C.c_double * 6)()
        self.lib.oracle_a_coefficients(a)
        return list(a)

    def effective_chord_length(self, t, v) -> float:
        return self.lib.oracle_effective_chord_length(C.byref(self.cfg), t, v)

    def mlp_paths(self, hist, x, start=0, n=None, stride=1312):
        arrs, h = self._hist(hist)
        if n is None:
            n = len(arrs[0]) - start
        xp = self.padded_image(x)
        counts = np.zeros(n, np.uint32)
        voxels = np.zeros((n, stride), np.uint32)
        chord = np.zeros(n, np.float64)
        adx = np.zeros(n, np.float64)
        flags = np.zeros(3, np.int64)
        self.lib.oracle_mlp_paths(C.byref(self.cfg), C.byref(self.tab), xp.ctypes.data, C.byref(h), start, n, stride,
                                  counts.ctypes.data, voxels.ctypes.data, chord.ctypes.data, adx.ctypes.data,
                                  flags.ctypes.data)
        return counts, voxels, chord, adx, flags

    def drop_iteration(self, hist, x, iterations=1):
        """Returns the image after `iterations` DROP iterations (input order, float accumulation)."""
        arrs, h = self._hist(hist)
        n = len(arrs[0])
        xp = self.padded_image(x)
        xu = np.zeros(self.npad, np.float32)
        S = np.zeros(self.npad, np.uint32)
        flags = np.zeros(3, np.int64)
        for _ in range(iterations):
            self.lib.oracle_drop_iteration(C.byref(self.cfg), C.byref(self.tab), C.byref(h), n, xp.ctypes.data,
                                           xu.ctypes.data, S.ctypes.data, flags.ctypes.data)
        return xp[: self.cfg.NUM_VOXELS].copy(), flags

    def s_curve_table(self, count=1312) -> np.ndarray:
        """s(k) for k < count, the configured S-curve (B.cu:10606-10626)."""
        out = np.zeros(count, np.float32)
        self.lib.oracle_s_curve_table(C.byref(self.cfg), count, out.ctypes.data)
        return out

    def host_effective_chord_length(self, t, v) -> float:
        """The host code's chord length (the float overload, O.cu:3745-3767)."""
        return self.lib.oracle_host_effective_chord_length(C.byref(self.cfg), t, v)

    def host_mlp_paths(self, hist, start=0, n=None, stride=4096):
        """The host MLP voxel lists (O.cu:4017-4211) and atanf chord lengths (O.cu:6634-6636)."""
        arrs, h = self._hist(hist)
        if n is None:
            n = len(arrs[0]) - start
        counts = np.zeros(n, np.uint32)
        voxels = np.zeros((n, stride), np.uint32)
        chord = np.zeros(n, np.float64)
        self.lib.oracle_host_mlp_paths(C.byref(self.cfg), C.byref(h), start, n, stride, counts.ctypes.data,
                                       voxels.ctypes.data, chord.ctypes.data)
        return counts, voxels, chord

    def fast_point_check(self, hist):
        """(points, points the guarded fast evaluation accepts, accepted points whose voxel differs
        from the reference-order voxel) over every MLP point of the histories."""
        arrs, h = self._hist(hist)
        out = np.zeros(3, np.int64)
        self.lib.oracle_fast_point_check(C.byref(self.cfg), C.byref(self.tab), C.byref(h), len(arrs[0]),
                                         out.ctypes.data)
        return tuple(int(v) for v in out)

    def guarded_indices(self, x, y, z, err):
        """The fast point's voxel guard on positions (cm) with error bound err: (ok, indices[n, 3])."""
        x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
        ok = np.zeros(len(x), np.int32)
        idx = np.zeros((len(x), 3), np.int32)
        self.lib.oracle_guarded_indices(C.byref(self.cfg), len(x), x.ctypes.data, y.ctypes.data, z.ctypes.data,
                                        float(err), ok.ctypes.data, idx.ctypes.data)
        return ok.astype(bool), idx

    def host_drop_iteration(self, hist, x, threads=1, n=None):
        """The reference's host MLP+DROP (O.cu) on `threads` cores; returns (image, path voxels)."""
        arrs, h = self._hist(hist)
        n = len(arrs[0]) if n is None else n
        xp = self.padded_image(x)
        visited = self.lib.oracle_host_drop_iteration(C.byref(self.cfg), C.byref(h), n, xp.ctypes.data, threads)
        return xp[: self.cfg.NUM_VOXELS].copy(), visited


GEOM = ("x_entry", "y_entry", "z_entry", "x_exit", "y_exit", "z_exit", "xy_entry_angle", "xz_entry_angle",
        "xy_exit_angle", "xz_exit_angle")
TRACKER = ("t_in_1", "t_in_2", "t_out_1", "t_out_2", "u_in_1", "u_in_2", "u_out_1", "u_out_2", "v_in_1", "v_in_2",
           "v_out_1", "v_out_2")


def _ptrs(arrays):
    return (C.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])


class PreOracle:
    """CPU restatement of the preprocessing stages (pct_oracle_pre.c) for one configuration."""

    def __init__(self, cfg_struct):
        self.lib = _load()
        self.cfg = cfg_struct
        self.nv = cfg_struct.NUM_VOXELS
        self.nb = cfg_struct.NUM_BINS

    def intersections(self, tracker, gantry_angle, integer_angles):
        tr = [np.ascontiguousarray(tracker[k], np.float32) for k in TRACKER]
        n = len(tr[0])
        ang = np.ascontiguousarray(gantry_angle, np.float32)
        out = [np.zeros(n, np.float32) for _ in GEOM]
        missed = np.zeros(n, np.uint8)
        self.lib.oracle_recon_volume_intersections(C.byref(self.cfg), n, _ptrs(tr), ang.ctypes.data,
                                                   int(integer_angles), _ptrs(out), missed.ctypes.data)
        return dict(zip(GEOM, out)), missed

    def binning(self, geom, wepl, missed):
        g = [np.ascontiguousarray(geom[k], np.float32) for k in GEOM]
        n = len(g[0])
        wepl = np.ascontiguousarray(wepl, np.float32)
        missed = np.ascontiguousarray(missed, np.uint8)
        bin_num = np.zeros(n, np.int32)
        counts = np.zeros(self.nb, np.int32)
        sums = [np.zeros(self.nb, np.float32) for _ in range(3)]
        self.lib.oracle_binning(C.byref(self.cfg), n, _ptrs(g), wepl.ctypes.data, missed.ctypes.data,
                                bin_num.ctypes.data, counts.ctypes.data, sums[0].ctypes.data, sums[1].ctypes.data,
                                sums[2].ctypes.data)
        return bin_num, counts, sums

    def statistics_and_cuts(self, bin_num, wepl, geom, bin_counts, sums):
        g = [np.ascontiguousarray(geom[k], np.float32) for k in GEOM]
        n = len(g[0])
        bin_counts = bin_counts.copy()
        means = [s.copy() for s in sums]
        sds = [np.zeros(self.nb, np.float32) for _ in range(3)]
        sino = np.zeros(self.nb, np.float32)
        keep = np.zeros(n, np.uint8)
        self.lib.oracle_statistics_and_cuts(C.byref(self.cfg), n, np.ascontiguousarray(bin_num, np.int32).ctypes.data,
                                            np.ascontiguousarray(wepl, np.float32).ctypes.data, _ptrs(g),
                                            bin_counts.ctypes.data, *[m.ctypes.data for m in means],
                                            *[s.ctypes.data for s in sds], sino.ctypes.data, keep.ctypes.data)
        return keep, bin_counts, means, sds, sino

    def sinogram_filter(self, bin_counts, sinogram_sums):
        sino = sinogram_sums.copy()
        filt = np.zeros(self.nb, np.float32)
        self.lib.oracle_sinogram_filter(C.byref(self.cfg), np.ascontiguousarray(bin_counts, np.int32).ctypes.data,
                                        sino.ctypes.data, filt.ctypes.data)
        return sino, filt

    def backprojection(self, filtered):
        fbp = np.zeros(self.nv, np.float32)
        self.lib.oracle_backprojection(C.byref(self.cfg), np.ascontiguousarray(filtered, np.float32).ctypes.data,
                                       fbp.ctypes.data)
        return fbp

    def median_filter(self, image, radius):
        out = np.zeros(self.nv, np.float32)
        self.lib.oracle_median_filter(C.byref(self.cfg), int(radius), np.ascontiguousarray(image, np.float32).ctypes.data,
                                      out.ctypes.data)
        return out

    def initialize_hull(self):
        h = np.zeros(self.nv, np.int32)
        self.lib.oracle_initialize_hull(C.byref(self.cfg), h.ctypes.data)
        return h

    def hull_walks(self, kind, geom, wepl, missed, image):
        g = [np.ascontiguousarray(geom[k], np.float32) for k in GEOM]
        image = np.ascontiguousarray(image, np.int32).copy()
        bounded = self.lib.oracle_hull_walks(C.byref(self.cfg), int(kind), len(g[0]), _ptrs(g),
                                             np.ascontiguousarray(wepl, np.float32).ctypes.data,
                                             np.ascontiguousarray(missed, np.uint8).ctypes.data, image.ctypes.data)
        return image, bounded

    def edge_detection(self, kind, counts):
        c = np.ascontiguousarray(counts, np.int32).copy()
        self.lib.oracle_edge_detection(C.byref(self.cfg), int(kind), c.ctypes.data)
        return c

    def collect_endpoints(self, hull, geom):
        g = [np.ascontiguousarray(geom[k], np.float32).copy() for k in GEOM]
        n = len(g[0])
        fv = np.zeros(n, np.uint32)
        self.lib.oracle_collect_mlp_endpoints(C.byref(self.cfg), np.ascontiguousarray(hull, np.uint8).ctypes.data, n,
                                              _ptrs(g), fv.ctypes.data)
        return dict(zip(GEOM, g)), fv


TVS_REFERENCE, TVS_ENGINE = 0, 1


class TvsOracle:
    """CPU restatement of total variation superiorization (pct_oracle_tvs.c)."""

    def __init__(self, cfg_struct, mode=TVS_ENGINE):
        self.lib = _load()
        self.cfg = cfg_struct
        self.nv = cfg_struct.NUM_VOXELS
        self.mode = mode

    def randi(self, lo, hi, k):
        return self.lib.oracle_tvs_randi(lo, hi, self.cfg.TVS_SEED, k)

    def eta(self):
        n = self.lib.oracle_tvs_eta(C.byref(self.cfg), None, 0)
        out = np.zeros(max(n, 1), np.float32)
        self.lib.oracle_tvs_eta(C.byref(self.cfg), out.ctypes.data, n)
        return out[:n]

    def total_variation(self, x):
        x = np.ascontiguousarray(x[:self.nv], np.float32)
        return self.lib.oracle_total_variation(C.byref(self.cfg), x.ctypes.data, self.mode)

    def direction(self, x):
        x = np.ascontiguousarray(x[:self.nv], np.float32)
        G, v, norm = np.zeros(self.nv, np.float32), np.zeros(self.nv, np.float32), C.c_float(0)
        self.lib.oracle_tvs_direction(C.byref(self.cfg), x.ctypes.data, G.ctypes.data, v.ctypes.data,
                                      C.byref(norm), self.mode)
        return G, v, norm.value

    def ntvs_iteration(self, x, hull, k, L):
        """Returns (perturbed image, L after, L after each repetition)."""
        x = np.array(x[:self.nv], np.float32)
        hull = np.ascontiguousarray(hull[:self.nv], np.uint8)
        Lc = C.c_int(L)
        acc = np.zeros(64, np.int32)
        n = self.lib.oracle_ntvs_iteration(C.byref(self.cfg), x.ctypes.data, hull.ctypes.data, k, C.byref(Lc),
                                           self.mode, acc.ctypes.data, len(acc))
        return x, Lc.value, acc[:n].tolist()
