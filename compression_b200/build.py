"""Build libgd.so (CUDA kernels for sm_100a + host C++) in-tree.

    python -m compression_b200.build            # incremental
    python -m compression_b200.build --clean

Objects go to compression_b200/_build/ (git-ignored); the shared library is
written to compression_b200/libgd.so next to this file so that it travels
with the source tree.
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
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libgd.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                  "-I", str(ROOT / "include"), "-I", str(CSRC)]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function", "-I", str(ROOT / "include"),
            "-I", "/usr/local/cuda/include"]


def sources():
    cu = sorted(CSRC.glob("*.cu"))
    cpp = sorted((CSRC / "host").glob("*.cpp"))
    return cu, cpp


def headers():
    return sorted(list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h")) + list(CSRC.glob("*.h")))


def _newer(src: Path, obj: Path, deps) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(d.stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    cu, cpp = sources()
    deps = headers()
    jobs = []
    objs = []
    for s in cu:
        o = BUILD / (s.stem + ".cu.o")
        objs.append(o)
        if _newer(s, o, deps) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([NVCC] + NVFLAGS + extra + ["-c", str(s), "-o", str(o)])
    for s in cpp:
        o = BUILD / (s.stem + ".cpp.o")
        objs.append(o)
        if _newer(s, o, deps):
            jobs.append(["g++"] + CXXFLAGS + ["-c", str(s), "-o", str(o)])
    with cf.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 4)) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    if jobs or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-cudart", "static"] + [str(o) for o in objs]
             + ["-lz", "-lpthread", "-o", str(tmp)])
        os.replace(tmp, LIB)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v register/smem usage")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args(argv)
    if a.clean and BUILD.exists():
        shutil.rmtree(BUILD)
    p = build(verbose=a.v or a.ptxas, ptxas_info=a.ptxas)
    print(p)


if __name__ == "__main__":
    sys.exit(main())
