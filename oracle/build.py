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


def build_oracle() -> Path:
    src = HERE / "gd_oracle.c"
    if LIB.exists() and LIB.stat().st_mtime >= src.stat().st_mtime:
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-std=c11", "-Wall", str(src), "-lz", "-o", str(tmp)],
                   check=True)
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
