"""bench.py's reference arm, on the CPU: it prints one JSON line with the own arm's workload
object, times the reference's redzone_CPU and std::remove(par_unseq) beside it, and loads no
library of this package (only the reference's code compiled into oracle/_ref)."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

_RUNNER = r"""
import runpy, sys, json
sys.argv = ["bench.py", "--impl", "reference", "--steps", "3", "--warmup", "1"]
try:
    runpy.run_path("bench.py", run_name="__main__")
finally:
    maps = open("/proc/self/maps").read()
    print(json.dumps({"package_lib_loaded": "libredzone_b200" in maps,
                      "reference_lib_loaded": "librz_ref_cpu" in maps,
                      "package_imported": any(m == "redzone_b200" or m.startswith("redzone_b200.") for m in sys.modules)}))
"""


def test_reference_arm_loads_only_the_reference():
    if not (ROOT / "oracle" / "_ref" / "librz_ref_cpu.so").exists():
        pytest.skip("the reference's CPU path was not built on this machine")
    r = subprocess.run([sys.executable, "-c", _RUNNER], cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.strip().splitlines() if x.startswith("{")]
    line, probe = lines[-2], lines[-1]
    assert probe == {"package_lib_loaded": False, "reference_lib_loaded": True, "package_imported": False}
    sys.path.insert(0, str(ROOT))
    import bench
    assert line["impl"] == "reference" and line["config"] == bench.config(1)
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT and line["higher_is_better"] is True
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == line["value"] > 0
    assert cb["std_remove_par"]["calls"] >= 1 and cb["std_remove_par"]["pstl_parallel_backend"] in (True, False)
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
