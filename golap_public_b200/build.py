"""In-tree build of libgx.so (the C-ABI library) for sm_100a.

Compiles golap_public_b200/csrc/*.cu and *.cpp with nvcc
(-gencode arch=compute_100a,code=sm_100a) and links them, with the static
CUDA runtime, into golap_public_b200/libgx.so.  Rebuilds only when a source
or header is newer than the library.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libgx.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include")]


def _sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _deps():
    return _sources() + sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted((ROOT / "include").glob("*.h"))


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:4])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)
    return r


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> Path:
    """Compile every CUDA/C++ source and link libgx.so; returns its path."""
    if not force and not ptxas_info and not _stale(LIB, _deps()):
        return LIB
    BUILD.mkdir(exist_ok=True)
    objs = []
    headers = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted((ROOT / "include").glob("*.h"))
    for src in _sources():
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if not force and not ptxas_info and not _stale(obj, [src] + headers):
            continue
        cmd = [NVCC] + COMMON + ARCH + ["-c", str(src), "-o", str(obj)]
        if src.suffix == ".cu":
            cmd += ["-lineinfo"]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
        _run(cmd, verbose or ptxas_info)
    tmp = LIB.with_suffix(".so.tmp")
    _run([NVCC] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in objs] + ["-lpthread"], verbose)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
