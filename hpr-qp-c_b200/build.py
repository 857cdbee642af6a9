"""Build recipe of the engine library: nvcc, sm_100a only, in-tree.

    python hpr-qp-c_b200/build.py          # -> hpr-qp-c_b200/lib/libhprqp.so
    python hpr-qp-c_b200/build.py --sanitize
        # -> hpr-qp-c_b200/_build_san/libhprqp.so: the host code built with
        #    AddressSanitizer + UndefinedBehaviorSanitizer (-O1 -g), for CPU
        #    test runs of the builders, readers and bindings:
        #    LD_PRELOAD="$(gcc -print-file-name=libasan.so) $(gcc -print-file-name=libubsan.so)"
        #    ASAN_OPTIONS=detect_leaks=0 HPRQP_LIBRARY_PATH=<that .so> python -m pytest tests -m "not gpu"

Compiles every source under csrc/ with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` into one shared
library whose exported symbols are exactly the C ABI declared in
include/*.h.  Objects are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
OBJ = PKG / "_build"
LIB = PKG / "lib" / "libhprqp.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers():
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.rglob("*.h"))


def _compile(src: Path, verbose_ptxas: bool) -> Path:
    obj = OBJ / (src.name + ".o")
    newest_dep = max([src.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    if obj.exists() and obj.stat().st_mtime >= newest_dep and not verbose_ptxas:
        return obj
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
           f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(src), "-o", str(obj)]
    if verbose_ptxas and src.suffix == ".cu":
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return obj


def build(verbose_ptxas: bool = False) -> Path:
    OBJ.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    srcs = _sources()
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"], check=True)
    return LIB


def build_sanitized() -> Path:
    """Every source with host-side ASan + UBSan into _build_san/libhprqp.so
    (always rebuilt; not used by the package unless HPRQP_LIBRARY_PATH
    points at it)."""
    out = PKG / "_build_san"
    out.mkdir(parents=True, exist_ok=True)
    flags = ["-Xcompiler", "-fPIC,-fsanitize=address,-fsanitize=undefined,-fno-omit-frame-pointer"]

    def one(src: Path) -> Path:
        obj = out / (src.name + ".o")
        subprocess.run([nvcc(), *ARCH, "-O1", "-g", "-std=c++17", *flags, f"-I{INCLUDE}", f"-I{CSRC}", "-c",
                        str(src), "-o", str(obj)], check=True)
        return obj

    srcs = _sources()
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(one, srcs))
    lib = out / "libhprqp.so"
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(lib), *map(str, objs), "-lcudart", "-Xcompiler",
                    "-fsanitize=address,-fsanitize=undefined"], check=True)
    return lib


if __name__ == "__main__":
    print(build_sanitized() if "--sanitize" in sys.argv else build(verbose_ptxas="-v" in sys.argv))
