#!/usr/bin/env python3
"""Build recipe for the reference VAMPIRE CPU code (test infrastructure only).

This script compiles the reference's own C++ sources *where they lie* (the
reference tree is read-only; nothing is copied into this repository) and writes
every output under ``oracle/_ref/``, which is git-ignored:

    oracle/_ref/obj/...            reference object files (serial build)
    oracle/_ref/obj_cuda/...       the few reference files whose code changes
                                   under -DCUDA (src/gpu/*.cpp, sim.cpp, main.cpp)
    oracle/_ref/vampire-serial     the unmodified reference program
    oracle/_ref/vampire-harness    reference objects + oracle/harness.cpp: a
                                   white-box driver that dumps the reference's
                                   own CSR, exchange lists, spins and RNG stream
    oracle/_ref/vampire-harness-b200  the harness on the -DCUDA objects with the
                                   B200 backend: --gpu-mc runs Monte Carlo
                                   through the gpu::mc_step hook
    oracle/_ref/vampire-b200       the unmodified reference program built with
                                   -DCUDA, whose ``vcuda::`` backend is
                                   vampire_b200/host/vcuda_b200.cpp over the
                                   C ABI of libvgpu.so (the drop-in)

The reference's build system is *not* run.  The object list is read from the
reference makefiles' object lists (top-level makefile ``OBJECTS`` plus each
included module's ``<module>_objects``), and each file is compiled with g++
directly, with the compatibility flags the reference needs under g++ 13
(``-include cstdint -include cstdlib -fpermissive -w``).

Usage:  python oracle/build_ref.py [--ref PATH] [--jobs N] [--no-b200]
"""
from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
OUT = HERE / "_ref"

CXX = os.environ.get("CXX", "g++")
BASE_FLAGS = ["-std=c++11", "-O3", "-mtune=native", "-funroll-loops",
              "-include", "cstdint", "-include", "cstdlib", "-fpermissive", "-w",
              "-DCOMP=\"GNU C++ Compiler\""]

# Modules whose object lists the top-level makefile includes (cuda/opencl are
# the reference GPU backends and are not built).
SKIP_MODULES = {"cuda", "opencl"}



# Where this recipe looks for the read-only reference tree when neither
# --ref nor VAMPIRE_REF names one (the container that builds the oracle).
DEFAULT_REF = "/root/reference"


def default_ref() -> str:
    return os.environ.get("VAMPIRE_REF", DEFAULT_REF)

def object_list(ref: Path) -> list[str]:
    """Return reference sources (relative to src/, without extension)."""
    top = (ref / "makefile").read_text()
    # Top-level OBJECTS block
    block = top.split("OBJECTS= \\", 1)[1].split("# Include supplementary makefiles", 1)[0]
    objs = [t.strip().rstrip("\\").strip() for t in block.splitlines()]
    objs = [o for o in objs if o.startswith("obj/") and o.endswith(".o")]
    srcs = [o[len("obj/"):-2] for o in objs]
    for mod in re.findall(r"^include src/(\w+)/makefile", top, re.M):
        if mod in SKIP_MODULES:
            continue
        mtext = (ref / "src" / mod / "makefile").read_text()
        pm = re.search(r"OBJECTS\+=\$\(addprefix obj/(\w+)/,\$\((\w+)\)\)", mtext)
        if not pm:
            continue
        subdir, var = pm.group(1), pm.group(2)
        # collect the list assigned to var (continuation lines)
        lines = mtext.splitlines()
        collecting = False
        for ln in lines:
            s = ln.strip()
            if re.match(rf"^{var}\s*=", s):
                collecting = True
                s = s.split("=", 1)[1]
            if collecting:
                for t in s.replace("\\", " ").split():
                    if t.endswith(".o"):
                        srcs.append(f"{subdir}/{t[:-2]}")
                collecting = ln.rstrip().endswith("\\")
    # unique, keep order
    seen, out = set(), []
    for s in srcs:
        if s not in seen:
            seen.add(s)
            out.append(s)
    return out


def _compile(args):
    src, obj, flags = args
    obj.parent.mkdir(parents=True, exist_ok=True)
    if obj.exists() and obj.stat().st_mtime >= src.stat().st_mtime:
        return None
    cmd = [CXX, "-c", str(src), "-o", str(obj)] + flags
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return f"FAILED {' '.join(cmd)}\n{r.stderr[-4000:]}"
    return None


def build(ref: Path, jobs: int, with_b200: bool) -> None:
    inc = ["-I", str(ref / "hdr"), "-I", str(ref / "src" / "qvoronoi")]
    srcs = object_list(ref)
    tasks = []
    for s in srcs:
        src = ref / "src" / f"{s}.cpp"
        if not src.exists():
            src = ref / "src" / f"{s}.c"
        extra = ["-DGHASH=\"reference\""] if s == "main/githash" else []
        tasks.append((src, OUT / "obj" / f"{s}.o", BASE_FLAGS + inc + extra))
    # -DCUDA variants of the files whose code depends on it
    cuda_files = [s for s in srcs if s.startswith("gpu/") or s in ("simulate/sim", "main/main")]
    for s in cuda_files:
        tasks.append((ref / "src" / f"{s}.cpp", OUT / "obj_cuda" / f"{s}.o",
                      BASE_FLAGS + inc + ["-DCUDA"]))
    with ThreadPoolExecutor(jobs) as ex:
        errs = [e for e in ex.map(_compile, tasks) if e]
    if errs:
        sys.stderr.write("\n".join(errs) + "\n")
        raise SystemExit(1)

    serial_objs = [str(OUT / "obj" / f"{s}.o") for s in srcs]
    lib_objs = [o for s, o in zip(srcs, serial_objs) if s != "main/main"]

    def link(out: Path, objs: list[str], extra: list[str]) -> None:
        cmd = [CXX, "-o", str(out)] + objs + extra
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stderr[-4000:])
            raise SystemExit(1)

    link(OUT / "vampire-serial", serial_objs, [])

    harness_o = OUT / "harness.o"
    err = _compile((HERE / "harness.cpp", harness_o,
                    BASE_FLAGS + inc + ["-I", str(ref / "src")]))
    if err:
        sys.stderr.write(err)
        raise SystemExit(1)
    link(OUT / "vampire-harness", lib_objs + [str(harness_o)], [])

    if with_b200:
        lib = REPO / "vampire_b200" / "libvgpu.so"
        if not lib.exists():
            print("build_ref: libvgpu.so not built yet; skipping vampire-b200")
            return
        shim_o = OUT / "vcuda_b200.o"
        err = _compile((REPO / "vampire_b200" / "host" / "vcuda_b200.cpp", shim_o,
                        BASE_FLAGS + inc + ["-DCUDA", "-I", str(ref / "src"),
                                            "-I", str(REPO / "include")]))
        if err:
            sys.stderr.write(err)
            raise SystemExit(1)
        cuda_set = set(cuda_files)
        objs = [str(OUT / ("obj_cuda" if s in cuda_set else "obj") / f"{s}.o") for s in srcs]
        link(OUT / "vampire-b200", objs + [str(shim_o)],
             ["-L", str(lib.parent), "-lvgpu", f"-Wl,-rpath,$ORIGIN/../../vampire_b200"])
        # the harness on the same -DCUDA objects, with the gpu::mc_step hook
        hook_o = OUT / "harness_b200.o"
        err = _compile((HERE / "harness.cpp", hook_o,
                        BASE_FLAGS + inc + ["-DCUDA", "-DVGPU_MC_HOOK", "-I", str(ref / "src")]))
        if err:
            sys.stderr.write(err)
            raise SystemExit(1)
        lib_cuda = [o for s, o in zip(srcs, objs) if s != "main/main"]
        link(OUT / "vampire-harness-b200", lib_cuda + [str(shim_o), str(hook_o)],
             ["-L", str(lib.parent), "-lvgpu", f"-Wl,-rpath,$ORIGIN/../../vampire_b200"])


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=default_ref())
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--no-b200", action="store_true")
    a = ap.parse_args()
    ref = Path(a.ref)
    if not (ref / "src" / "simulate" / "LLGHeun.cpp").exists():
        raise SystemExit(f"reference tree not found at {ref}")
    build(ref, a.jobs, not a.no_b200)
    print("build_ref: ok ->", OUT)


if __name__ == "__main__":
    main()
