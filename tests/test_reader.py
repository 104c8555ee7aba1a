"""Projection data files (PCTD / PCTN, versions 0 and 1): header parse, data reads, writer, and
the scan loader that feeds the preprocessing stages.

The format follows count_histories_v0 (B.cu:3578) and read_data_chunk_v0 (B.cu:4361): magic,
int32 version, int32 N, float angle, float energy, two int32 dates, three length-prefixed strings,
then N floats each of t0..t3, v0..v3, u0..u3, WEPL (mm) and optionally N per-history angles.
The CPU tests use an independent struct-based writer/parser; they call only the library's host
file functions (no device work).  The GPU tests check that the device mm->cm conversion and
shifts are bit-identical to the reference's `float *= 0.1` / `float += shift` and that a scan
read from files preprocesses exactly like the same data passed as arrays.
"""
import struct

import numpy as np
import pytest

from pct_reconstruction_b200 import Config
from pct_reconstruction_b200 import engine as E
from pct_reconstruction_b200 import phantoms as P

FILE_ORDER = ["t_in_1", "t_in_2", "t_out_1", "t_out_2", "v_in_1", "v_in_2", "v_out_1", "v_out_2",
              "u_in_1", "u_in_2", "u_out_1", "u_out_2", "WEPL"]


def write_raw(path, arrays, *, magic=b"PCTD", version=0, angle=0.0, energy=200.0, dates=(1, 2),
              strings=(b"phantom", b"source", b"me"), n=None, angles=None, truncate=0):
    """Independent writer of the file layout (struct + numpy)."""
    n = len(arrays["WEPL"]) if n is None else n
    blob = magic + struct.pack("<iiffii", version, n, angle, energy, *dates)
    for s in strings:
        blob += struct.pack("<i", len(s)) + s
    for k in FILE_ORDER:
        blob += np.asarray(arrays[k], "<f4").tobytes()
    if angles is not None:
        blob += np.asarray(angles, "<f4").tobytes()
    if truncate:
        blob = blob[:-truncate]
    path.write_bytes(blob)
    return 4 + 7 * 4 + 2 * 4 + sum(len(s) for s in strings)


def parse_raw(path):
    b = path.read_bytes()
    magic = b[:4]
    version, n, angle, energy, d0, d1 = struct.unpack_from("<iiffii", b, 4)
    off = 28
    strings = []
    for _ in range(3):
        (ln,) = struct.unpack_from("<i", b, off)
        strings.append(b[off + 4:off + 4 + ln])
        off += 4 + ln
    data = np.frombuffer(b, "<f4", offset=off)
    arrays = {k: data[i * n:(i + 1) * n] for i, k in enumerate(FILE_ORDER)}
    angles = data[13 * n:14 * n] if len(data) >= 14 * n and n else None
    return dict(magic=magic, version=version, n=n, angle=angle, energy=energy, dates=(d0, d1), strings=strings,
                data_offset=off), arrays, angles


def random_arrays(n, seed):
    rng = np.random.default_rng(seed)
    return {k: (rng.normal(size=n) * 80).astype(np.float32) for k in FILE_ORDER}


# ---------------------------------------------------------------- host file functions -----

def test_read_v0_file_written_independently(tmp_path):
    arr = random_arrays(1001, 1)
    off = write_raw(tmp_path / "p.bin", arr, angle=8.0, strings=(b"CTP404", b"", b"x" * 300))
    h, a = E.read_projection_file(tmp_path / "p.bin")
    assert h["continuous"] == 0 and h["version"] == 0 and h["num_histories"] == 1001
    assert h["projection_angle"] == 8.0 and h["beam_energy"] == 200.0
    assert (h["generation_date"], h["preprocess_date"]) == (1, 2)
    assert h["data_offset"] == off == 4 + 28 + 8 + 6 + 0 + 300
    assert h["phantom_name"] == "CTP404" and h["data_source"] == "" and h["prepared_by"] == "x" * 255
    assert h["has_angles"] == 0 and "projection_angle" not in a
    for k in FILE_ORDER:
        np.testing.assert_array_equal(a[k], arr[k])


def test_pctn_v1_file_with_angles(tmp_path):
    arr = random_arrays(257, 2)
    ang = np.random.default_rng(3).uniform(0, 360, 257).astype(np.float32)
    write_raw(tmp_path / "p.bin", arr, magic=b"PCTN", version=1, angle=92.7, angles=ang)
    h, a = E.read_projection_file(tmp_path / "p.bin")
    assert h["continuous"] == 1 and h["version"] == 1 and h["has_angles"] == 1
    np.testing.assert_array_equal(a["projection_angle"], ang)
    np.testing.assert_array_equal(a["u_out_2"], arr["u_out_2"])


def test_library_writer_matches_independent_parser(tmp_path):
    arr = random_arrays(333, 4)
    ang = np.linspace(0, 359, 333, dtype=np.float32)
    E.write_projection_file(tmp_path / "w.bin", dict(arr, projection_angle=ang), 44.0, continuous=True, version=1,
                            beam_energy=199.5, generation_date=7, preprocess_date=9, phantom_name="head",
                            data_source="sim", prepared_by="b200")
    h, a, angles = parse_raw(tmp_path / "w.bin")
    assert h["magic"] == b"PCTN" and h["version"] == 1 and h["n"] == 333
    assert h["angle"] == 44.0 and h["energy"] == np.float32(199.5) and h["dates"] == (7, 9)
    assert h["strings"] == [b"head", b"sim", b"b200"]
    for k in FILE_ORDER:
        np.testing.assert_array_equal(a[k], arr[k])
    np.testing.assert_array_equal(angles, ang)
    # and the library reads back its own file
    h2, a2 = E.read_projection_file(tmp_path / "w.bin")
    assert h2["data_offset"] == h["data_offset"] and h2["has_angles"] == 1


def test_empty_file(tmp_path):
    write_raw(tmp_path / "e.bin", {k: np.zeros(0, np.float32) for k in FILE_ORDER})
    h, a = E.read_projection_file(tmp_path / "e.bin")
    assert h["num_histories"] == 0 and all(len(v) == 0 for v in a.values())


@pytest.mark.parametrize("case", ["magic", "version", "truncated", "missing", "string_length", "negative_n",
                                  "short_header"])
def test_malformed_files_are_io_errors(tmp_path, case):
    arr = random_arrays(50, 5)
    p = tmp_path / "bad.bin"
    if case == "magic":
        write_raw(p, arr, magic=b"PCTX")
    elif case == "version":
        write_raw(p, arr, version=2)
    elif case == "truncated":
        write_raw(p, arr, truncate=4)
    elif case == "string_length":
        write_raw(p, arr)
        b = bytearray(p.read_bytes())
        b[28:32] = struct.pack("<i", -5)
        p.write_bytes(bytes(b))
    elif case == "negative_n":
        write_raw(p, arr, n=-3)
    elif case == "short_header":
        p.write_bytes(b"PCTD\x00\x00")
    with pytest.raises(E.PCTError) as ei:
        E.read_projection_header(p)
    assert ei.value.status == 7  # PCT_ERR_IO


def test_config_reader_keys():
    cfg = Config(T_SHIFT=2.05, U_SHIFT=-0.16, DATA_IN_MM=0, USE_CONT_ANGLES=1)
    assert cfg.T_SHIFT == 2.05 and cfg.U_SHIFT == -0.16 and cfg.V_SHIFT == 0.0
    assert cfg.DATA_IN_MM == 0 and cfg.USE_CONT_ANGLES == 1
    assert Config().DATA_IN_MM == 1 and Config().USE_CONT_ANGLES == 0


# ---------------------------------------------------------------- scan loader (GPU) -------

def write_scan(directory, td_cm, interval, *, continuous=False, version=0):
    """Split tracker data (cm) by gantry angle into one file per angle, in mm."""
    ang = td_cm["gantry_angle"]
    file_of = np.round(ang / interval).astype(np.int64) % int(round(360 / interval))
    order, firsts = [], []
    for f in range(int(round(360 / interval))):
        idx = np.nonzero(file_of == f)[0]
        arrays = {k: (td_cm[k][idx].astype(np.float64) * 10.0).astype(np.float32) for k in FILE_ORDER}
        if continuous:
            arrays["projection_angle"] = ang[idx]
        E.write_projection_file(directory / E.projection_file_name(f * interval), arrays, float(f * interval),
                                continuous=continuous, version=version)
        order.append(idx)
        firsts.append(float(f * interval))
    return order, firsts


def expected_conversion(values_mm, shift=0.0):
    v = (values_mm.astype(np.float64) * 0.1).astype(np.float32)
    if shift is not None:
        v = (v.astype(np.float64) + shift).astype(np.float32)
    return v


@pytest.fixture(scope="module")
def c1_tracks(c1_params):
    tr = P.simulate_tracks(P.water_cylinder_phantom(6.0), 40000, seed=41, continuous_angles=False,
                           angle_interval_deg=4.0, t_extent=16.0, v_extent=3.5)
    return {k: v.numpy() for k, v in P.tracker_data(tr).items()}


@pytest.mark.gpu
@pytest.mark.parametrize("shifts", [(0.0, 0.0, 0.0), (0.205, -0.016, 0.03)])
def test_scan_load_converts_like_the_reference(tmp_path, c1_params, c1_tracks, shifts):
    from pct_reconstruction_b200 import Context
    cfg = Config(**dict(c1_params, T_SHIFT=shifts[0], U_SHIFT=shifts[1], V_SHIFT=shifts[2]))
    order, angles = write_scan(tmp_path, c1_tracks, 4.0)
    with Context(cfg) as ctx:
        n = ctx.load_projection_data(tmp_path)
        assert n == len(c1_tracks["WEPL"])
        got = {k: ctx.get_array(k) for k in FILE_ORDER[:-1] + ["gantry_angle"]}
        got_wepl = ctx.get_array("WEPL")
    idx = np.concatenate(order)
    apply = any(s != 0.0 for s in shifts)
    for k in FILE_ORDER[:-1]:
        mm = (c1_tracks[k][idx].astype(np.float64) * 10.0).astype(np.float32)
        s = shifts["tuv".index(k[0])] if apply else None
        np.testing.assert_array_equal(got[k], expected_conversion(mm, s), err_msg=k)
    wepl_mm = (c1_tracks["WEPL"][idx].astype(np.float64) * 10.0).astype(np.float32)
    np.testing.assert_array_equal(got_wepl, expected_conversion(wepl_mm, None))
    np.testing.assert_array_equal(got["gantry_angle"], np.repeat(np.float32(angles), [len(o) for o in order]))


@pytest.mark.gpu
def test_scan_from_files_preprocesses_like_arrays(tmp_path, c1_params, c1_tracks):
    """preprocessing() from files == pct_preprocessing on the same converted arrays."""
    from pct_reconstruction_b200 import Context
    cfg = Config(**c1_params)
    order, angles = write_scan(tmp_path, c1_tracks, 4.0)
    idx = np.concatenate(order)
    td = {}
    for k in FILE_ORDER:
        mm = (c1_tracks[k][idx].astype(np.float64) * 10.0).astype(np.float32)
        td[k] = expected_conversion(mm, None)
    td["gantry_angle"] = np.repeat(np.float32(angles), [len(o) for o in order])
    with Context(cfg) as a, Context(cfg) as b:
        na = a.preprocessing_from_files(tmp_path)
        nb = b.preprocessing(td, integer_angles=True)
        assert na == nb and na > 1000
        for k in ("x_entry_vector", "xy_exit_angle_vector", "WEPL_vector", "first_MLP_voxel_vector", "hull"):
            np.testing.assert_array_equal(a.get_array(k), b.get_array(k), err_msg=k)
        # the bin sums behind the FBP start are float atomics: last-bit differences run to run
        np.testing.assert_allclose(a.x_GPU_2_host(), b.x_GPU_2_host(), rtol=1e-5, atol=1e-6)
        a.DROP_full_tx_iteration(1)
        b.DROP_full_tx_iteration(1)
        # float atomics: the scatter order differs run to run (last-bit differences only)
        np.testing.assert_allclose(a.x_GPU_2_host(), b.x_GPU_2_host(), rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
def test_continuous_angle_files(tmp_path, c1_params):
    from pct_reconstruction_b200 import Context
    tr = P.simulate_tracks(P.water_cylinder_phantom(6.0), 20000, seed=43, continuous_angles=True,
                           t_extent=16.0, v_extent=3.5)
    td = {k: v.numpy() for k, v in P.tracker_data(tr).items()}
    order, _ = write_scan(tmp_path, td, 4.0, continuous=True, version=1)
    idx = np.concatenate(order)
    with Context(Config(**dict(c1_params, USE_CONT_ANGLES=1))) as ctx:
        assert ctx.load_projection_data(tmp_path) == len(idx)
        np.testing.assert_array_equal(ctx.get_array("gantry_angle"), td["gantry_angle"][idx])
    with Context(Config(**c1_params)) as ctx:  # USE_CONT_ANGLES off: int(file angle)
        ctx.load_projection_data(tmp_path)
        ga = ctx.get_array("gantry_angle")
        assert np.all(ga == np.floor(ga)) and set(np.unique(ga)) <= set(np.arange(0, 360, 4, dtype=np.float32))


@pytest.mark.gpu
def test_missing_file_in_scan_is_io_error(tmp_path, c1_params, c1_tracks):
    from pct_reconstruction_b200 import Context
    write_scan(tmp_path, c1_tracks, 4.0)
    (tmp_path / E.projection_file_name(88)).unlink()
    with Context(Config(**c1_params)) as ctx:
        with pytest.raises(E.PCTError) as ei:
            ctx.load_projection_data(tmp_path)
        assert ei.value.status == 7 and "projection_088.bin" in str(ei.value)
