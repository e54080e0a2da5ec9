"""Host-side checks of the native library that need no GPU: it loads, exports every function
include/*.h declares, and its status strings are defined. No compute calls here."""
import ctypes
import subprocess

import numpy as np

from redzone_b200 import _native, workloads


def test_library_loads_and_exports_every_declared_symbol():
    names = _native.declared_symbols()
    assert "rz_remove" in names and "rz_create" in names
    missing = [nm for nm in names if not hasattr(_native.lib, nm)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(_native.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    assert set(names) <= exported


def test_status_strings():
    for code in range(9):
        s = _native.status_string(code)
        assert s and s != "unknown status"
    assert _native.status_string(99) == "unknown status"


def test_library_is_built_for_sm100a_only():
    """The build compiles and links every source for sm_100a and for nothing else (checked on the
    build recipe, not on the binary)."""
    import importlib.util
    from pathlib import Path

    spec = importlib.util.spec_from_file_location("_rz_build_check", Path(_native.PKG) / "build.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    assert b.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "-lineinfo" in b.COMMON
    assert not any("gencode" in f or "arch" in f for f in b.COMMON)


def test_item_bytes():
    import torch
    from redzone_b200 import item_bytes
    assert item_bytes(torch.zeros(10, dtype=torch.int32)) == 4
    assert item_bytes(torch.zeros(10, 4, dtype=torch.int32)) == 16
    assert item_bytes(torch.zeros(10, 4, dtype=torch.int64)) == 32


def test_workload_distributions():
    n = 1 << 16
    u = workloads.uniform(n, 5000, 1)
    assert u.dtype == np.uint32 and np.unique(u).size == 5000 and u.max() < n
    c = workloads.clustered(n, 256 * 20, 2)
    s = np.sort(c.astype(np.int64))
    assert np.unique(s).size == s.size
    starts = np.flatnonzero(np.diff(np.concatenate([[-10], s])) != 1)
    runs = np.diff(np.concatenate([starts, [s.size]]))
    assert (runs % 256 == 0).all()  # adjacent runs may touch, never overlap
    t = workloads.tail(n, 3000, 3)
    assert t.min() >= n - n // 10 and np.unique(t).size == 3000
    r = workloads.red_split(n, 1000, 4, 25)
    assert (r >= n - 1000).sum() == 250
    nn, kk = workloads.batched_lists(4096, seed=0)
    assert nn.min() >= 256 and nn.max() <= 1 << 22 and (kk <= nn // 2 + 1).all()


def test_device_producer_header_compiles_in_a_caller_kernel(tmp_path):
    """include/redzone_device.cuh is usable from a caller's own CUDA file (compiled for sm_100a
    here; running it is the GPU tests' job)."""
    import os
    import pytest
    nvcc = "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "caller.cu"
    src.write_text(
        '#include "redzone_device.cuh"\n'
        "__global__ void delete_small(rz_producer_view v, const float* score, uint32_t n) {\n"
        "    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ((n + 31u) & ~31u);\n"
        "         i += gridDim.x * blockDim.x)\n"
        "        rz_emit(v, i, i < n && score[i] < 0.5f);\n"
        "}\n")
    r = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-c", str(src), "-o",
                        str(tmp_path / "caller.o"), "-I", os.path.join(root, "include")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_predictor_space_matches_the_library():
    """The predictor's class index is a position in the library's configuration space: the Python
    mirror used for training and evaluation must list the same configurations in the same order."""
    from redzone_b200 import learn
    n = _native.lib.rz_config_space(None, 0)
    out = (_native.LaunchCfg * n)()
    assert _native.lib.rz_config_space(out, n) == n == learn.N_CFG
    lib = [(c.block, c.items, c.ctas_per_sm, c.schedule) for c in out]
    assert lib == learn.config_space()
    assert all(c.use_partition == 0 for c in out)


def test_batched_queue_order_keeps_every_wait_behind_its_target(tmp_path):
    """The batched kernel's work-queue order (both orders, several lags), compiled from its header
    and checked on random list mixes: a permutation in which every item follows what it waits for."""
    import os
    import pytest
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cuda_inc = "/usr/local/cuda/include"
    if not os.path.exists(os.path.join(cuda_inc, "vector_types.h")):
        pytest.skip("CUDA headers not available")
    exe = tmp_path / "order_check"
    r = subprocess.run(["g++", "-std=c++17", "-O1", os.path.join(root, "tests", "cpp", "order_check.cpp"), "-o", str(exe),
                        "-I", os.path.join(root, "redzone_b200", "csrc"), "-I", cuda_inc], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def test_e2e_driver_is_built_and_checks_its_arguments():
    """build() also links the C++ end-to-end timing program next to the library; with bad
    arguments it reports the error before touching a GPU."""
    exe = _native.LIB_PATH.parent / "rz_e2e"
    assert exe.exists()
    r = subprocess.run([str(exe), "10", "10", "5", "4"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and '"error": "bad arguments"' in r.stdout
