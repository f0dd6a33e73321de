"""Build recipe for libvt_b200.so (the CUDA kernels and the C ABI of include/vt.h).

Compiles every ``csrc/*.cu`` for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``) with
nvcc and links them into ``metal_vibe_tracer_b200/lib/libvt_b200.so``, in tree, so the library
travels with the repository. Objects are rebuilt when their source or any header is newer.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import time
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OBJ = PKG / "lib" / "obj"
LIB = PKG / "lib" / "libvt_b200.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
    "-Xptxas", "-warn-spills",
]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libvt_b200.so")
    return exe


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compile and link libvt_b200.so; returns its path."""
    OBJ.mkdir(parents=True, exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    if not sources:
        raise RuntimeError(f"no CUDA sources under {CSRC}")
    newest_header = max((h.stat().st_mtime for h in _headers()), default=0.0)
    objs = []
    compiled = False
    for src in sources:
        obj = OBJ / (src.stem + ".o")
        objs.append(obj)
        if (not force and obj.exists() and obj.stat().st_mtime >= src.stat().st_mtime
                and obj.stat().st_mtime >= newest_header):
            continue
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *(extra or []), "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        started = time.time()
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}\n{res.stderr}")
        # The object carries the time its compile began, so a source or header edited while it
        # compiled stays newer and is compiled again next time.
        os.utime(obj, (started, started))
        compiled = True
        if verbose and (res.stdout or res.stderr):
            print(res.stdout + res.stderr, file=sys.stderr)
    if force or compiled or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "--cudart", "static", "-o", str(tmp), *map(str, objs)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
