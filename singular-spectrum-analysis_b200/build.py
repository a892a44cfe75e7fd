"""Builds libssa.so (the drop-in SSA library) in this directory.

C host sources are compiled with gcc, the CUDA kernels with nvcc for sm_100a only, and
everything is linked with the static CUDA runtime, so the library depends on the NVIDIA driver
alone. Usage: ``python build.py`` (from anywhere) or ``build.build()``.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
OUT = HERE / "libssa.so"
BUILD = HERE / "_build"

C_SOURCES = ["ssa_engine.c", "ssa_api.c", "ssa_batch.c", "ssa_mssa.c", "ssa_ragged.c", "ssa_server.c",
             "ssa_mbatch.c"]
CU_SOURCES = ["ssa_kernels.cu"]

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC,-fvisibility=hidden",
]


def _cuda_home() -> Path:
    for c in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if c and (Path(c) / "bin" / "nvcc").exists():
            return Path(c)
    nv = shutil.which("nvcc")
    if nv:
        return Path(nv).resolve().parent.parent
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def _stale(target: Path, deps: list[Path], cmd: list[str] | None = None) -> bool:
    """True when `target` is missing or was built from other contents of `deps` (or another
    command): a content digest is kept beside each target, so clock skew between file systems
    cannot leave a stale object in place."""
    h = hashlib.sha256()
    for d in sorted(deps):
        h.update(str(d).encode())
        h.update(d.read_bytes())
    h.update(" ".join(cmd or []).encode())
    digest = h.hexdigest()
    stamp = target.with_name(target.name + ".sha256")
    if target.exists() and stamp.exists() and stamp.read_text() == digest:
        return False
    _pending[target] = (stamp, digest)
    return True


_pending: dict = {}


def _done(target: Path) -> None:
    if target in _pending:
        stamp, digest = _pending.pop(target)
        stamp.write_text(digest)


def build(force: bool = False, verbose: bool = False) -> Path:
    cuda = _cuda_home()
    nvcc = str(cuda / "bin" / "nvcc")
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    objs = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".cu.o")
        cmd = [nvcc, *NVCC_FLAGS, "-I", str(CSRC), "-I", str(INCLUDE), "-c", str(s), "-o", str(o)]
        if _stale(o, [s] + headers, cmd) or force:
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
            _done(o)
        objs.append(o)
    for src in C_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".c.o")
        cmd = ["gcc", "-std=gnu11", "-O2", "-fPIC", "-Wall", "-Wextra", "-Wno-unused-parameter",
               "-I", str(cuda / "include"), "-I", str(CSRC), "-I", str(INCLUDE), "-c", str(s), "-o", str(o)]
        if _stale(o, [s] + headers, cmd) or force:
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
            _done(o)
        objs.append(o)
    cmd = [nvcc, "-shared", "-cudart", "static", "-gencode", "arch=compute_100a,code=sm_100a",
           "-o", str(OUT), *map(str, objs), "-lm", "-lpthread"]
    if _stale(OUT, objs, cmd) or force:
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
        _done(OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(OUT)
