"""CPU oracle for Redzone removal -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this
package, and only as a checker or a timed CPU baseline; the library in ``redzone_b200`` never
calls it.

* ``remove`` / ``stable_remove`` / ``validate`` / ``remove_batched``: the C restatement in
  ``oracle/canonical.c`` (built to ``oracle/_build/librz_oracle.so``), payload-agnostic.
* ``ref_redzone_cpu`` / ``ref_par_remove``: the reference's own ``redzone_CPU``
  (Redzone_CPU.hxx:150) and ``par_remove_phase1/2`` (std_parallel_remove.hxx:13-36), compiled
  from its sources by ``oracle/Makefile`` into ``oracle/_ref/librz_ref_cpu.so``.
* ``remove_numpy``: a vectorised numpy statement of the same rule, for tiny cross-checks.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "librz_oracle.so"
REF_SO = HERE / "_ref" / "librz_ref_cpu.so"

_oracle = None
_ref = None


# Where the reference checkout is read from when oracle/_ref is built (environment variable
# RZ_REFERENCE_DIR overrides it); machines without it keep a prebuilt oracle/_ref.
REFERENCE_DIR = os.environ.get("RZ_REFERENCE_DIR", "/root/reference")


def build(ref: bool = True) -> None:
    """Compile the oracle (and the reference CPU path when its sources are present)."""
    args = ["make", "-s", "-C", str(HERE), "oracle"]
    if ref:
        args += ["ref", f"REF={REFERENCE_DIR}"]
    subprocess.run(args, check=True)


def _vp(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def lib() -> ctypes.CDLL:
    global _oracle
    if _oracle is None:
        if not ORACLE_SO.exists():
            build(ref=False)
        L = ctypes.CDLL(str(ORACLE_SO))
        u64, vp = ctypes.c_uint64, ctypes.c_void_p
        L.rz_oracle_remove.argtypes = [vp, u64, ctypes.c_uint32, vp, u64]
        L.rz_oracle_stable_remove.argtypes = [vp, u64, ctypes.c_uint32, vp, u64]
        L.rz_oracle_validate.argtypes = [u64, vp, u64]
        L.rz_oracle_remove_batched.argtypes = [vp, ctypes.c_uint32, vp, ctypes.c_int64, vp, vp, vp, vp]
        _oracle = L
    return _oracle


def ref_lib() -> ctypes.CDLL | None:
    """The reference's compiled CPU path, or None when it was never built on this machine."""
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            return None
        L = ctypes.CDLL(str(REF_SO))
        vp, i = ctypes.c_void_p, ctypes.c_int
        L.ref_redzone_cpu.argtypes = [vp, i, vp, i]
        L.ref_par_remove.argtypes = [vp, i, vp, i]
        L.ref_redzone_threads.restype = i
        L.ref_pool_threads.restype = i
        L.ref_pstl_parallel.restype = i
        _ref = L
    return _ref


def _items(data: np.ndarray) -> tuple[int, int]:
    """(n, item bytes) of a C-contiguous array whose first axis enumerates the items."""
    assert data.flags.c_contiguous
    n = data.shape[0]
    w = data.itemsize * (int(np.prod(data.shape[1:])) if data.ndim > 1 else 1)
    return n, w


def remove(data: np.ndarray, idx: np.ndarray) -> int:
    """Redzone removal in place (tail left as is). Returns the new length; raises on bad input."""
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    n, w = _items(data)
    rc = lib().rz_oracle_remove(_vp(data), n, w, _vp(idx), idx.size)
    if rc:
        raise ValueError(f"oracle rejected input (code {rc})")
    return n - idx.size


def stable_remove(data: np.ndarray, idx: np.ndarray) -> int:
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    n, w = _items(data)
    rc = lib().rz_oracle_stable_remove(_vp(data), n, w, _vp(idx), idx.size)
    if rc:
        raise ValueError(f"oracle rejected input (code {rc})")
    return n - idx.size


def validate(n: int, idx: np.ndarray) -> int:
    """0 ok, 2 duplicate, 3 out of range (rz_status codes)."""
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    return int(lib().rz_oracle_validate(n, _vp(idx), idx.size))


def remove_batched(data: np.ndarray, w: int, idx: np.ndarray, data_off, n, idx_off, k) -> None:
    arrs = [np.ascontiguousarray(a, dtype=np.uint64) for a in (data_off, n, idx_off, k)]
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    rc = lib().rz_oracle_remove_batched(_vp(data), w, _vp(idx), len(arrs[0]), *[_vp(a) for a in arrs])
    if rc:
        raise ValueError(f"oracle rejected input (code {rc})")


def remove_numpy(data: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """Vectorised restatement of the same rule; returns the new prefix (copy)."""
    a = data.copy()
    n, k = a.shape[0], idx.size
    cut = n - k
    if k == 0 or k == n:
        return a[:cut]
    idx = idx.astype(np.int64)
    red = np.zeros(k, dtype=bool)
    red[idx[idx >= cut] - cut] = True
    sv, dv = ~red, idx < cut
    src = a[cut:].copy()
    both = sv & dv
    a[idx[both]] = src[both]
    a[idx[dv & ~sv]] = src[sv & ~dv]
    return a[:cut]


def ref_redzone_cpu(data: np.ndarray, idx: np.ndarray) -> int:
    """Run the reference's redzone_CPU in place on int32 data (clobbers a copy of idx)."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("reference CPU library not built (oracle/_ref/librz_ref_cpu.so)")
    assert data.dtype == np.int32 and data.flags.c_contiguous
    r = np.ascontiguousarray(idx, dtype=np.int32).copy()
    L.ref_redzone_cpu(_vp(data), data.size, _vp(r), r.size)
    return data.size - r.size
