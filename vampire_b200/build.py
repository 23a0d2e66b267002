"""Build libvgpu.so in-tree with nvcc for sm_100a.

    python -m vampire_b200.build [--force] [--verbose]

Every .cu file under vampire_b200/csrc is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked into
vampire_b200/libvgpu.so (CUDA runtime linked statically), which exports the C
ABI declared in include/vgpu.h.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libvgpu.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", f"-I{REPO / 'include'}", f"-I{CSRC}"]


def sources():
    return sorted(CSRC.glob("*.cu"))


def deps():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h"))
                  + list((REPO / "include").glob("*.h")))


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in deps())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        cmd = [NVCC, "-c", str(src), "-o", str(obj)] + ARCH + FLAGS
        if src.stem.endswith("_fp64"):
            cmd += ["-fmad=false"]  # FP64 rounding as the reference's non-FMA x86-64 build
        if verbose:
            cmd += ["-Xptxas", "-v"]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed = True
            sys.stderr.write(f"nvcc failed on {src.name}:\n{out}\n")
        elif verbose and out:
            sys.stdout.write(out)
    if failed:
        raise RuntimeError("libvgpu build failed")
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC, "-shared", "-o", str(tmp)] + [str(o) for o in objs] + ARCH + ["-Xcompiler", "-fPIC"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
