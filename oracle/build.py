"""Build the oracle (test infrastructure only).

    python oracle/build.py          # liboracle.so from gd_oracle.c (gcc)
    python oracle/build.py --ref    # also oracle/_ref/ from the reference sources

liboracle.so is the CPU checker that tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py load; nothing in the compression_b200 package
links or imports it.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"


# liboracle.so: the C restatement of the decoders (gd_oracle.c), the input
# builders of the CPU baselines (gd_inputs.cpp, with the lane encoder header
# it includes) and the seeded column generators, compiled from the product's
# generator source so that a seed gives the same column in both libraries.
GEN = HERE.parent / "compression_b200" / "csrc" / "host" / "gd_gen.cpp"
DEPS = [HERE / "gd_oracle.c", HERE / "gd_inputs.cpp", GEN, HERE.parent / "compression_b200" / "csrc" / "lane_enc.h"]


def build_oracle() -> Path:
    if LIB.exists() and all(LIB.stat().st_mtime >= d.stat().st_mtime for d in DEPS):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    obj = HERE / "_ref" / "obj"
    obj.mkdir(parents=True, exist_ok=True)
    inc = str(HERE.parent / "include")
    subprocess.run(["gcc", "-O2", "-fPIC", "-std=c11", "-Wall", "-c", str(HERE / "gd_oracle.c"), "-o",
                    str(obj / "gd_oracle.o")], check=True)
    for src in (HERE / "gd_inputs.cpp", GEN):
        subprocess.run(["g++", "-O2", "-fPIC", "-std=c++17", "-Wall", "-I", inc, "-I", "/usr/local/cuda/include",
                        "-c", str(src), "-o", str(obj / (src.stem + ".o"))], check=True)
    subprocess.run(["g++", "-shared", "-o", str(tmp), str(obj / "gd_oracle.o"), str(obj / "gd_inputs.o"),
                    str(obj / "gd_gen.o"), "-lz", "-pthread"], check=True)
    tmp.replace(LIB)
    return LIB


def build_ref() -> bool:
    """Compile the reference's own host-callable codec sources into oracle/_ref.

    Needs the reference checkout (present only where the sources are); returns
    False when it is absent so the GPU box, which only uses prebuilt files,
    skips this step.
    """
    ref = reference_dir()
    if ref is None:
        return False
    subprocess.run(["make", "-s", "-C", str(HERE / "ref"), f"REF={ref}"], check=True)
    return True


def reference_dir() -> Path | None:
    """The reference checkout: $GD_REFERENCE_DIR, else a directory named
    "reference" beside the repository; None when neither holds include/."""
    import os
    cand = [os.environ.get("GD_REFERENCE_DIR"), str(HERE.parent.parent / "reference")]
    for c in cand:
        if c and (Path(c) / "include").is_dir():
            return Path(c).resolve()
    return None


if __name__ == "__main__":
    print(build_oracle())
    if "--ref" in sys.argv:
        print("ref:", build_ref())
