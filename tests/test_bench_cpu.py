"""bench.py's reference arm on CPU: it runs the reference's own CPU decoders
on inputs built without the product library (no libgd.so in the process),
and reports the same metric and config as the GPU arm's line."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_reference_arm_loads_no_product_library():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--scale", "0.01",
                        "--steps", "1", "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    import bench
    assert line["impl"] == "reference"
    assert line["metric"] == bench.HEADLINE_METRIC
    assert line["config"] == bench.run_config(bench.HEADLINE, 1)
    assert line["native_libs"] == ["oracle/liboracle.so"], line["native_libs"]
    assert {k["kernel"] for k in line["kernels"]} == {"brle", "rlev2", "rlev1", "lzss", "deflate"}
    assert all(k["value"] > 0 for k in line["kernels"])
    assert line["e2e"]["value"] == line["value"] > 0
