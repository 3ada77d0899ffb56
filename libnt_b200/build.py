"""Builds the CUDA library ``libnt_b200/liblnt_cuda.so`` in-tree with nvcc.

Every ``csrc/*.cu`` is compiled for sm_100a only and linked into one shared
library exporting the C ABI of ``include/lnt.h``.  Objects go to
``libnt_b200/_build/``; a source is recompiled when it, or any header under
``csrc/`` or ``include/``, is newer than its object.

Run ``python -m libnt_b200.build`` (or call :func:`build`).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "liblnt_cuda.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr", "-I", str(ROOT / "include"), "-I", str(CSRC),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the LNT CUDA library cannot be built")


def cuda_lib_dir() -> str:
    return str(Path(nvcc()).resolve().parent.parent / "lib64")


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, obj: Path, extra: list[str]) -> tuple[Path, str]:
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stderr}")
    return obj, r.stderr


def build(verbose: bool = False, extra: list[str] | None = None, force: bool = False) -> Path:
    """Compile all kernels and link liblnt_cuda.so; returns its path."""
    extra = list(extra or [])
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    hdr = _headers_mtime()
    todo = []
    objs = []
    for s in srcs:
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if force or not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, hdr):
            todo.append((s, o))
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(len(todo), os.cpu_count() or 4)) as ex:
            for obj, log in ex.map(lambda t: _compile(t[0], t[1], extra), todo):
                if verbose and log.strip():
                    print(f"[{obj.name}]\n{log}", file=sys.stderr)
    if force or todo or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart_static", "-lcublasLt",
               "-lrt", "-ldl", "-lpthread", "-Xlinker", f"-rpath={cuda_lib_dir()}"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    v = "-v" in sys.argv
    ex = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(verbose=v or bool(ex), extra=ex, force="--force" in sys.argv))
