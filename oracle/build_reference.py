"""Compile the reference's own CUDA program for sm_100a, linked with the fixture harness.

TEST INFRASTRUCTURE ONLY.  Reads the reference source where it lies (it is never copied into this
repository) and writes only into oracle/_ref/ (git-ignored; the built binary is run on a machine
with a B200):

  oracle/_ref/ref_B.o          src/pCT_Reconstruction_Data_Segments_Blake.cu, unmodified, with
                               relocatable device code; -include oracle/ref_shim.h supplies the
                               ifstream==NULL comparison the C++11 library lacks,
                               -Dsyncthreads=__syncthreads the legacy alias, -Dmain renames its main,
                               -maxrregcount=64 lets its 1024-thread kernels launch on sm_100a
  oracle/_ref/ref_harness      oracle/ref_harness.cu + ref_B.o

Usage: python oracle/build_reference.py [--reference /path/to/pCT_Reconstruction]
"""
from __future__ import annotations

import argparse
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise SystemExit(r.returncode)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    src = Path(args.reference) / "src" / "pCT_Reconstruction_Data_Segments_Blake.cu"
    if not src.exists():
        print(f"reference source not found at {src}; nothing built")
        return
    OUT.mkdir(exist_ok=True)
    ref_o, har_o, exe = OUT / "ref_B.o", OUT / "ref_harness.o", OUT / "ref_harness"
    if not ref_o.exists() or ref_o.stat().st_mtime < src.stat().st_mtime:
        # -maxrregcount=64: recon_volume_intersections_GPU indexes with THREADS_PER_BLOCK = 1024 and
        # must launch 1024-thread CTAs, but compiles to 70+ registers for sm_100a (more than a
        # 1024-thread CTA can hold), so the stock build cannot launch it on B200.  Capping the
        # register count only changes register allocation (spills), not the arithmetic.
        run(["nvcc", *ARCH, "-std=c++11", "-O3", "-rdc=true", "-w", "-maxrregcount=64", "-Dmain=pct_reference_main",
             "-Dsyncthreads=__syncthreads", "-include", str(HERE / "ref_shim.h"), "-Xcompiler", "-fopenmp",
             "-c", str(src), "-o", str(ref_o)])
    run(["nvcc", *ARCH, "-std=c++17", "-O3", "-rdc=true", "-c", str(HERE / "ref_harness.cu"), "-o", str(har_o)])
    run(["nvcc", *ARCH, "-rdc=true", str(ref_o), str(har_o), "-o", str(exe)])
    print(exe)


if __name__ == "__main__":
    main()
