"""Compile the reference's own CUDA program for sm_100a, linked with the fixture harness.

TEST INFRASTRUCTURE ONLY.  Reads the reference source where it lies (it is never copied into this
repository) and writes only into oracle/_ref/ (git-ignored; the built binaries are run on a
machine with a B200).  B.cu's parameters are compile-time macros in B.h, so one harness is built
per configuration:

  builtin   the reference's B.h as it is (256 x 256 x 32 voxels of 0.0625 x 0.0625 x 0.25 cm):
              oracle/_ref/ref_B.o, oracle/_ref/ref_harness
  head      the head-size grid (200 x 200 x 32 voxels of 0.1 x 0.1 x 0.25 cm, R = 10 cm, DROP
            blocks of 60000, HISTORIES_PER_BLOCK 480): a copy of B.h with those macro values
            replaced is written to oracle/_ref/head/include/, next to oracle/_ref/head/src/ which
            holds a symbolic link to the unmodified B.cu, so that B.cu's own
            `#include "../include/..."` picks up the patched copy:
              oracle/_ref/head/ref_B.o, oracle/_ref/head/ref_harness
  scurve    the built-in grid with S_CURVE_ON set to ON (B.h:467), so that DROP_block_update_GPU
            scales each path entry's update by s_curve_scale_GPU:
              oracle/_ref/scurve/ref_B.o, oracle/_ref/scurve/ref_harness
  small     the small workload of bench.py (128 x 128 x 16 voxels of 0.1 x 0.1 x 0.25 cm, R = 6.4 cm,
            SSD_V_SIZE 5 cm, MLP_U_STEP 0.1 cm, DROP blocks of 3200, HISTORIES_PER_BLOCK 640):
              oracle/_ref/small/ref_B.o, oracle/_ref/small/ref_harness

Every B.cu object is compiled unmodified, with relocatable device code; -include oracle/ref_shim.h
supplies the ifstream==NULL comparison the C++11 library lacks, -Dsyncthreads=__syncthreads the
legacy alias, -Dmain renames its main, and -maxrregcount=64 lets its 1024-thread kernels launch on
sm_100a.  The harness (oracle/ref_harness.cu) is compiled with the same grid values (-DPCT_REF_*).

Usage: python oracle/build_reference.py [--reference DIR] [--config builtin|head|scurve|small|all]
The reference checkout is DIR, else $PCT_REFERENCE_DIR, else /root/reference.  Exit status 0
when everything asked for was built or the reference is absent (nothing to build), 1 on a failure.
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
B_CU = Path("src") / "pCT_Reconstruction_Data_Segments_Blake.cu"
B_H = Path("include") / "pCT_Reconstruction_Data_Segments_Blake.h"

# B.h macro values per configuration (B.h:335, 373, 389-390, 421); the derived macros (COLUMNS,
# ROWS, SLICES, MLP_U_STEP = VOXEL_WIDTH / 2, ...) follow from these in B.h itself.
CONFIGS = {
    "builtin": {},
    "head": {"RECON_CYL_RADIUS": "10.0", "VOXEL_WIDTH": "0.1", "VOXEL_HEIGHT": "0.1", "DROP_BLOCK_SIZE": "60000",
             "HISTORIES_PER_BLOCK": "480"},
    "scurve": {"S_CURVE_ON": "ON"},
    "small": {"RECON_CYL_RADIUS": "6.4", "VOXEL_WIDTH": "0.1", "VOXEL_HEIGHT": "0.1", "SSD_V_SIZE": "5.0",
              "DROP_BLOCK_SIZE": "3200", "HISTORIES_PER_BLOCK": "640", "MLP_U_STEP": "0.1"},
}
BUILTIN = {"RECON_CYL_RADIUS": 8.0, "VOXEL_WIDTH": 0.0625, "VOXEL_HEIGHT": 0.0625, "VOXEL_THICKNESS": 0.25,
           "SLICE_THICKNESS": 0.25, "SSD_V_SIZE": 9.0, "HISTORIES_PER_BLOCK": 640}


def reference_dir(arg: str | None) -> Path:
    return Path(arg or os.environ.get("PCT_REFERENCE_DIR") or "/root/reference")


def run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(map(str, cmd)) + "\n" + r.stdout + r.stderr)
        raise SystemExit(1)


def harness_defines(name: str) -> list[str]:
    """The grid B.h derives for `name`, with B.h's own expressions (B.h:373-393)."""
    v = dict(BUILTIN)
    for k, x in CONFIGS[name].items():
        try:
            v[k] = float(x)
        except ValueError:  # a switch such as S_CURVE_ON, which leaves the grid as it is
            pass
    diameter = 2 * v["RECON_CYL_RADIUS"]
    height = v["SSD_V_SIZE"] - 1.0
    d = {"COLUMNS": int(diameter / v["VOXEL_WIDTH"]), "ROWS": int(diameter / v["VOXEL_HEIGHT"]),
         "SLICES": int(height / v["SLICE_THICKNESS"]), "HISTORIES_PER_BLOCK": int(v["HISTORIES_PER_BLOCK"]),
         "RADIUS": repr(v["RECON_CYL_RADIUS"]), "HEIGHT": repr(height), "VOXEL_WIDTH": repr(v["VOXEL_WIDTH"]),
         "VOXEL_HEIGHT": repr(v["VOXEL_HEIGHT"]), "VOXEL_THICKNESS": repr(v["VOXEL_THICKNESS"])}
    return [f"-DPCT_REF_{k}={x}" for k, x in d.items()]


def patched_header(text: str, values: dict[str, str]) -> str:
    """B.h with each named macro's value (everything up to its // comment) replaced."""
    for name, value in values.items():
        pat = re.compile(r"^(#define[ \t]+" + name + r"[ \t]+)(.*?)([ \t]*//.*)?$", re.M)
        text, k = pat.subn(lambda m: m.group(1) + value + (m.group(3) or ""), text)
        if k != 1:
            raise SystemExit(f"B.h: expected one #define {name}, found {k}")
    return text


def stale(target: Path, *sources: Path) -> bool:
    return not target.exists() or any(target.stat().st_mtime < s.stat().st_mtime for s in sources)


def build_config(ref: Path, name: str) -> Path:
    src = ref / B_CU
    if name == "builtin":
        d, cu, hdr = OUT, src, ref / B_H
    else:
        d = OUT / name
        (d / "src").mkdir(parents=True, exist_ok=True)
        (d / "include").mkdir(parents=True, exist_ok=True)
        cu = d / "src" / B_CU.name
        if not cu.is_symlink() or os.readlink(cu) != str(src):
            if cu.exists() or cu.is_symlink():
                cu.unlink()
            cu.symlink_to(src)
        hdr = d / "include" / B_H.name
        text = patched_header((ref / B_H).read_text(errors="surrogateescape"), CONFIGS[name])
        if not hdr.exists() or hdr.read_text(errors="surrogateescape") != text:
            hdr.write_text(text, errors="surrogateescape")
    d.mkdir(parents=True, exist_ok=True)
    ref_o, har_o, exe = d / "ref_B.o", d / "ref_harness.o", d / "ref_harness"
    if stale(ref_o, src, hdr):
        run(["nvcc", *ARCH, "-std=c++11", "-O3", "-rdc=true", "-w", "-maxrregcount=64", "-Dmain=pct_reference_main",
             "-Dsyncthreads=__syncthreads", "-include", str(HERE / "ref_shim.h"), "-Xcompiler", "-fopenmp",
             "-c", str(cu), "-o", str(ref_o)])
    if stale(har_o, HERE / "ref_harness.cu", Path(__file__)):
        run(["nvcc", *ARCH, "-std=c++17", "-O3", "-rdc=true", *harness_defines(name), "-c",
             str(HERE / "ref_harness.cu"), "-o", str(har_o)])
    if stale(exe, ref_o, har_o):
        run(["nvcc", *ARCH, "-rdc=true", str(ref_o), str(har_o), "-o", str(exe)])
    return exe


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None)
    ap.add_argument("--config", choices=[*CONFIGS, "all"], default="all")
    args = ap.parse_args()
    ref = reference_dir(args.reference)
    if not (ref / B_CU).exists():
        print(f"reference source not found under {ref}; nothing built")
        return
    OUT.mkdir(exist_ok=True)
    for name in (CONFIGS if args.config == "all" else [args.config]):
        print(build_config(ref, name))


if __name__ == "__main__":
    main()
