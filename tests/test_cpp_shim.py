"""The C++ half of the boundary: a host program compiled against include/redzone.hpp (the
reference-shaped redzone::RemoveFromList) and linked with the library. The CPU test builds it; the
GPU test runs it and checks both of its removals against the oracle."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from redzone_b200 import _native, workloads

ROOT = Path(__file__).resolve().parents[1]
CUDA = Path("/usr/local/cuda")


def _build(tmp_path: Path) -> Path:
    exe = tmp_path / "shim_main"
    cmd = ["g++", "-std=c++17", "-O2", str(ROOT / "tests" / "cpp" / "shim_main.cpp"), "-o", str(exe),
           f"-I{ROOT / 'include'}", f"-I{CUDA / 'include'}", f"-L{_native.LIB_PATH.parent}", "-lredzone_b200",
           f"-Wl,-rpath,{_native.LIB_PATH.parent}", f"-L{CUDA / 'lib64'}", "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_shim_program_builds(tmp_path):
    if not (CUDA / "include" / "cuda_runtime.h").exists():
        pytest.skip("CUDA headers not available")
    assert _build(tmp_path).exists()


@pytest.mark.gpu
@pytest.mark.parametrize("n,k,dist", [(1 << 18, 1 << 12, "uniform"), (1 << 20, 1 << 16, "red40"),
                                      (100003, 30011, "clustered")])
def test_cpp_shim_matches_oracle(tmp_path, n, k, dist):
    exe = _build(tmp_path)
    idx = workloads.make(dist, n, k, seed=11)
    (tmp_path / "idx.bin").write_bytes(idx.astype(np.uint32).tobytes())
    out = tmp_path / "out.bin"
    r = subprocess.run([str(exe), str(tmp_path / "idx.bin"), str(n), str(out)], capture_output=True, text=True,
                       timeout=120, env=dict(os.environ))
    assert r.returncode == 0, r.stderr
    raw = out.read_bytes()
    code = int(np.frombuffer(raw[:4], dtype=np.int32)[0])
    assert code == _native.RZ_ERR_DUPLICATE
    got_int = np.frombuffer(raw[4: 4 + 4 * (n - k)], dtype=np.uint32)
    got_rec = np.frombuffer(raw[4 + 4 * (n - k):], dtype=np.uint32).reshape(n - k, 4)
    i = np.arange(n, dtype=np.uint32)
    exp_int = i.copy()
    oracle.remove(exp_int, idx)
    rec = np.stack([i, i ^ np.uint32(0xA5A5A5A5), (3 * i.astype(np.uint64)).astype(np.uint32), ~i], axis=1)
    exp_rec = np.ascontiguousarray(rec)
    oracle.remove(exp_rec, idx)
    assert np.array_equal(got_int, exp_int[: n - k])
    assert np.array_equal(got_rec, exp_rec[: n - k])
