"""The C ABI from compiled callers: the reconstruction program and a C translation unit.

pct_reconstruction_b200/pct_recon (cli/pct_recon.cpp) is the C++ program that replaces the
reference's main (B.cu:369-399): settings.cfg -> preprocessing() from projection files ->
DROP_GPU -> image file, through include/pct_api.h only.  The CPU tests build it with g++, check its
usage and configuration errors (no device work), and compile and run a C99 program against the
header, whose view of pct_config (size and field offsets) must match the library's and the Python
binding's.  The GPU test reconstructs a small scan written as projection files and compares the
image with the same steps driven through the Python binding.
"""
import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

from pct_reconstruction_b200 import Config, _abi, build
from pct_reconstruction_b200 import phantoms as P

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def cli():
    build.build()
    return build.build_cli()


def test_cli_usage_and_config_errors(cli, tmp_path):
    r = subprocess.run([str(cli)], capture_output=True, text=True)
    assert r.returncode == 1 and "usage" in r.stderr
    r = subprocess.run([str(cli), str(tmp_path / "missing.cfg"), str(tmp_path), str(tmp_path / "x.bin")],
                       capture_output=True, text=True)
    assert r.returncode == 2 and "pct_config_load" in r.stderr
    r = subprocess.run([str(cli), str(GOLDEN / "settings_c1.cfg"), str(tmp_path), str(tmp_path / "x.bin"), "--set",
                        "NO_SUCH_KEY=1"], capture_output=True, text=True)
    assert r.returncode == 2 and "unknown key NO_SUCH_KEY" in r.stderr
    r = subprocess.run([str(cli), str(GOLDEN / "settings_c1.cfg"), str(tmp_path), str(tmp_path / "x.bin"), "--set",
                        "S_CURVE_ON=1", "--set", "PRECISION=MIXED"], capture_output=True, text=True)
    assert r.returncode == 2 and "S_CURVE_ON needs PRECISION EXACT" in r.stderr


C_PROBE = r"""
#include <stddef.h>
#include <stdio.h>
#include "pct_api.h"
int main(void) {
    pct_config c;
    pct_config_default(&c);
    if (pct_config_finalize(&c) != PCT_OK) return 3;
    printf("%zu %zu %zu %zu %zu %zu %d\n", sizeof(pct_config), pct_config_size(), offsetof(pct_config, LAMBDA),
           offsetof(pct_config, TVS_SEED), offsetof(pct_config, PRIME_OFFSET), offsetof(pct_config, X_N_AIR_THRESHOLD),
           c.NUM_VOXELS);
    return 0;
}
"""


def test_header_is_valid_c_and_matches_the_library_layout(tmp_path):
    build.build()
    src = tmp_path / "probe.c"
    src.write_text(C_PROBE)
    exe = tmp_path / "probe"
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"), str(src),
                        "-L", str(build.PKG), "-lpct_b200", f"-Wl,-rpath,{build.PKG}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    size_c, size_lib, off_lambda, off_seed, off_prime, off_air, nv = map(int, out)
    s = _abi.pct_config
    assert size_c == size_lib == ctypes.sizeof(s)
    assert (off_lambda, off_seed, off_prime, off_air) == (s.LAMBDA.offset, s.TVS_SEED.offset, s.PRIME_OFFSET.offset,
                                                           s.X_N_AIR_THRESHOLD.offset)
    assert nv == Config().NUM_VOXELS


@pytest.mark.gpu
def test_cli_reconstructs_like_the_binding(cli, tmp_path, c1_params):
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    from test_reader import write_scan
    from pct_reconstruction_b200 import Context
    tr = P.simulate_tracks(P.water_cylinder_phantom(6.0), 120000, seed=61, continuous_angles=False,
                           angle_interval_deg=4.0, t_extent=16.0, v_extent=3.5)
    td = {k: v.numpy() for k, v in P.tracker_data(tr).items()}
    scan = tmp_path / "scan"
    scan.mkdir()
    write_scan(scan, td, 4.0)
    settings = GOLDEN / "settings_c1.cfg"
    out = tmp_path / "x.bin"
    over = ["--set", "TVS_ON=0", "--iterations", "2"]
    r = subprocess.run([str(cli), str(settings), str(scan), str(out), *over], capture_output=True, text=True,
                       timeout=600)
    print(r.stdout, r.stderr)
    assert r.returncode == 0, r.stderr
    x_cli = np.fromfile(out, np.float32)
    cfg = Config(str(settings), TVS_ON=0, ITERATIONS=2)
    with Context(cfg) as ctx:
        n = ctx.preprocessing_from_files(scan)
        ctx.DROP_GPU()
        x_api = ctx.x_GPU_2_host()
    assert f"{n} reconstruction histories" in r.stdout and n > 10000
    assert x_cli.shape == x_api.shape
    # float atomics in binning and in the DROP scatter: last-bit differences run to run
    rel = float(np.sqrt(np.mean((x_cli.astype(np.float64) - x_api) ** 2)) / np.sqrt(np.mean(x_api.astype(np.float64) ** 2)))
    print(f"pct_recon vs binding: rel RMSE {rel:.2e}")
    assert rel < 1e-5
