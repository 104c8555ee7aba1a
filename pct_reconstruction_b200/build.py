"""Build libpct_b200.so (the engine) in-tree with nvcc for sm_100a.

Usage: python -m pct_reconstruction_b200.build [--jobs N]

It also builds the reconstruction program pct_reconstruction_b200/pct_recon (cli/pct_recon.cpp, a
C++ caller of include/pct_api.h compiled with g++ and linked against libpct_b200.so).

Each CUDA/C++ source is compiled to an object under pct_reconstruction_b200/_build/ and linked
into pct_reconstruction_b200/libpct_b200.so (static CUDA runtime, so the library only needs the
driver).  Sources that hold the exact-mode MLP are compiled with -fmad=false: their double
arithmetic must round exactly like the reference expressions (no fused multiply-add), see
csrc/pct_mlp.cuh.  Rebuilds only what changed (by mtime of the source and the headers).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libpct_b200.so"
CLI_SRC = PKG / "cli" / "pct_recon.cpp"
CLI = PKG / "pct_recon"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "-I", str(INCLUDE), "-I", str(CSRC)]
# Translation units whose double arithmetic must not be contracted into FMAs.
NO_FMAD = {"pct_drop_exact.cu", "pct_noalloc.cu", "pct_preprocess.cu", "pct_reader.cu", "pct_tables.cpp", "pct_tvs.cu"}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def compile_one(src: Path, force: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, headers_mtime()):
        return obj
    cmd = [nvcc(), *ARCH, *COMMON, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd[len(ARCH) + 1:len(ARCH) + 1] = ["-x", "cu"]
    if src.name in NO_FMAD:
        cmd.insert(1, "-fmad=false")
    if src.suffix == ".cu":
        cmd += ["-Xptxas", "-warn-spills"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    if res.stderr.strip():
        sys.stderr.write(res.stderr)
    return obj


def build(force: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcuda"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, LIB)
    build_cli(force)
    return LIB


def build_cli(force: bool = False) -> Path:
    """g++ build of the reconstruction program against the library (found next to it at run time)."""
    deps = [CLI_SRC, LIB, *INCLUDE.glob("*.h")]
    if force or not CLI.exists() or CLI.stat().st_mtime < max(d.stat().st_mtime for d in deps):
        cmd = [shutil.which("g++") or "g++", "-O2", "-std=c++17", "-Wall", "-Wextra", "-I", str(INCLUDE), str(CLI_SRC),
               "-L", str(PKG), "-lpct_b200", "-Wl,-rpath,$ORIGIN", "-o", str(CLI)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0 or res.stderr.strip():
            raise RuntimeError(f"g++ failed for {CLI_SRC.name}:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    return CLI


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    args = ap.parse_args()
    print(build(force=args.force, jobs=args.jobs))


if __name__ == "__main__":
    main()
