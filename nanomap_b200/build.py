"""Build step of the library: compiles nanomap_b200/csrc into nanomap_b200/libnanomap_b200.so.

Every CUDA translation unit is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``).  Host code is compiled with
``-frounding-math -ffp-contract=off`` because the per-frame constants are evaluated under an
explicit rounding mode.  Objects are rebuilt only when a source or header is newer.

Usage: ``python -m nanomap_b200.build [--force] [--verbose-ptxas]``
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
SRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libnanomap_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_FLAGS = ["-Xcompiler", "-fPIC", "-Xcompiler", "-frounding-math", "-Xcompiler", "-ffp-contract=off"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", f"-I{INCLUDE}", f"-I{SRC}"] + HOST_FLAGS


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; set NVCC or install the CUDA toolkit")


def _sources():
    return sorted(list(SRC.glob("*.cu")) + list(SRC.glob("*.cpp")))


def _headers():
    return sorted(list(SRC.glob("*.h")) + list(SRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


def _compile(src: Path, force: bool, ptxas_v: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    newest_dep = max([src.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    if not force and obj.exists() and obj.stat().st_mtime >= newest_dep:
        return obj
    cmd = [nvcc()] + COMMON + ARCH + ["-c", str(src), "-o", str(obj)]
    if src.suffix == ".cu":
        cmd += ["--expt-relaxed-constexpr"]
        if ptxas_v:
            cmd += ["-Xptxas", "-v"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
    if ptxas_v and proc.stderr:
        sys.stderr.write(proc.stderr)
    return obj


def build(force: bool = False, ptxas_v: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, ptxas_v), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc()] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in objs] + ["-lpthread"]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
        os.replace(tmp, LIB)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_v=a.verbose_ptxas))


if __name__ == "__main__":
    main()
