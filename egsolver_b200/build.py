"""Builds the solver's shared library in-tree for sm_100a.

    python -m egsolver_b200.build        (or build() from Python)

Host C sources are compiled with gcc, CUDA sources with nvcc
(-gencode arch=compute_100a,code=sm_100a), and everything is linked into
egsolver_b200/libegsolver_b200.so next to this file.  The reference-ABI
shim (eg_refabi.c, which binds to the globals of the reference's own
driver) is archived separately as egsolver_b200/libegrefabi.a.  Objects go
to egsolver_b200/_build/; a source is recompiled only when it or a header
changed.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libegsolver_b200.so"
REFABI = PKG / "libegrefabi.a"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I", str(INCLUDE), "-I", str(CSRC)] + ARCH
CC_FLAGS = ["-O3", "-fPIC", "-std=gnu11", "-Wall", "-Wno-unused-function", "-I", str(INCLUDE), "-I", str(CSRC),
            "-I", str(CUDA_HOME / "include")]

C_SOURCES = ["eg_host.c", "eg_reader.c", "eg_fixtures.c"]
CU_SOURCES = ["eg_prep.cu", "eg_lift.cu", "eg_dense.cu", "eg_api.cu", "eg_batch.cu", "eg_serve.cu", "eg_noalloc.cu"]
REFABI_SOURCES = ["eg_refabi.c"]


def _headers() -> list[Path]:
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ... (exit {res.returncode})")
    if verbose and (res.stdout or res.stderr):
        sys.stderr.write(res.stdout + res.stderr)


def build(verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compiles every source that changed and links the library; returns its path."""
    BUILD.mkdir(exist_ok=True)
    hdrs = _headers()
    objs: list[Path] = []
    changed = False
    for src in C_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        if _stale(o, [s] + hdrs):
            _run(["gcc", *CC_FLAGS, "-c", str(s), "-o", str(o)], verbose)
            changed = True
        objs.append(o)
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        if _stale(o, [s] + hdrs) or ptxas_verbose:
            extra = ["-Xptxas", "-v"] if ptxas_verbose else []
            _run([NVCC, *NVCC_FLAGS, *extra, "-c", str(s), "-o", str(o)], verbose or ptxas_verbose)
            changed = True
        objs.append(o)
    if changed or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC, "-shared", *ARCH, "-o", str(tmp), *map(str, objs), "-lz"], verbose)
        tmp.replace(LIB)
    # reference-ABI shim: a static archive linked into the reference's driver
    robjs = []
    for src in REFABI_SOURCES:
        s = CSRC / src
        if not s.exists():
            continue
        o = BUILD / (s.stem + ".o")
        if _stale(o, [s] + hdrs):
            _run(["gcc", *CC_FLAGS, "-c", str(s), "-o", str(o)], verbose)
        robjs.append(o)
    if robjs and _stale(REFABI, robjs):
        if REFABI.exists():
            REFABI.unlink()
        _run(["ar", "rcs", str(REFABI), *map(str, robjs)], verbose)
    return LIB


def clean() -> None:
    shutil.rmtree(BUILD, ignore_errors=True)
    for p in (LIB, REFABI):
        if p.exists():
            p.unlink()


if __name__ == "__main__":
    if "--clean" in sys.argv:
        clean()
    build(verbose=True, ptxas_verbose="--ptxas" in sys.argv)
    print(LIB)
