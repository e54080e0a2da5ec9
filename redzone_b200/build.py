"""Build the native library ``redzone_b200/_lib/libredzone_b200.so`` with nvcc for sm_100a.

Every ``.cu`` / ``.cpp`` file under ``redzone_b200/csrc`` is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked into one shared library
exposing the C-ABI of ``include/redzone.h``. Objects are rebuilt only when a source or header
is newer than its object. The build runs on a machine without a GPU (nvcc cross-compiles).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
OBJ_DIR = PKG / "_lib" / "obj"
LIB = OUT_DIR / "libredzone_b200.so"
E2E = OUT_DIR / "rz_e2e"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", f"-I{ROOT / 'include'}", f"-I{CSRC}"]


def _sources():
    return sorted([p for p in CSRC.iterdir() if p.suffix in (".cu", ".cpp")])


def _headers():
    return sorted([p for p in CSRC.iterdir() if p.suffix in (".h", ".cuh", ".hpp")]) + sorted(
        (ROOT / "include").glob("*.h*"))


def _compile(src: Path, verbose: bool) -> tuple[Path, bool]:
    """Compile one source; returns (object, whether it was rebuilt)."""
    obj = OBJ_DIR / (src.name + ".o")
    newest_dep = max([src.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    if obj.exists() and obj.stat().st_mtime >= newest_dep:
        return obj, False
    cmd = [NVCC, *ARCH, *COMMON, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd[1:1] = ["-x", "cu"]
    if verbose:
        cmd.append("-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        sys.stderr.write(res.stderr)
    return obj, True


def build(verbose: bool = False, quiet: bool = False) -> Path:
    """Compile what is out of date and link; prints which sources were rebuilt and whether the
    library was relinked (unless quiet)."""
    OBJ_DIR.mkdir(parents=True, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        done = list(ex.map(lambda s: _compile(s, verbose), srcs))
    objs = [o for o, _ in done]
    rebuilt = [s.name for s, (_, r) in zip(srcs, done) if r]
    if LIB.exists() and LIB.stat().st_mtime >= max(o.stat().st_mtime for o in objs):
        if not quiet:
            print(f"redzone_b200: {LIB.name} up to date ({len(srcs)} sources, none rebuilt)")
        build_e2e_driver(quiet)
        return LIB
    cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcuda"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    if not quiet:
        print(f"redzone_b200: rebuilt {len(rebuilt)} of {len(srcs)} sources "
              f"({', '.join(rebuilt) if rebuilt else 'objects newer than the library'}); linked {LIB.name}")
    build_e2e_driver(quiet)
    return LIB


def build_e2e_driver(quiet: bool = False) -> Path:
    """The C++ end-to-end timing program (redzone_b200/e2e_driver.cpp), linked against the library
    it sits next to."""
    src = PKG / "e2e_driver.cpp"
    if E2E.exists() and E2E.stat().st_mtime >= max(src.stat().st_mtime, LIB.stat().st_mtime,
                                                    (ROOT / "include" / "redzone.h").stat().st_mtime):
        return E2E
    cuda = Path(NVCC).resolve().parent.parent
    cmd = ["g++", "-std=c++17", "-O2", str(src), "-o", str(E2E), f"-I{ROOT / 'include'}", f"-I{cuda / 'include'}",
           f"-L{OUT_DIR}", "-lredzone_b200", "-Wl,-rpath,$ORIGIN", f"-L{cuda / 'lib64'}", "-lcudart_static",
           "-ldl", "-lpthread", "-lrt"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"e2e driver build failed:\n{res.stdout}\n{res.stderr}")
    if not quiet:
        print(f"redzone_b200: built {E2E.name}")
    return E2E


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
