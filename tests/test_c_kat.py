"""The drop-in C API as a C caller sees it: tests/c/kat_drop_in.c is compiled against
include/ssa_opt.h and linked with libssa.so (CPU: it builds and links; GPU: its known-answer
checks, modelled on the reference's C tests, all pass)."""
import os
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "singular-spectrum-analysis_b200"
SRC = Path(__file__).resolve().parent / "c" / "kat_drop_in.c"


def _build(out_dir: Path) -> Path:
    exe = out_dir / "kat_drop_in"
    cmd = ["gcc", "-std=gnu11", "-O2", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(SRC),
           "-L", str(PKG), "-l:libssa.so", f"-Wl,-rpath,{PKG}", "-lm", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.fixture(scope="module")
def kat_exe(tmp_path_factory):
    if not (PKG / "libssa.so").exists():
        import importlib.util
        spec = importlib.util.spec_from_file_location("ssabuild", PKG / "build.py")
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
        m.build()
    return _build(tmp_path_factory.mktemp("kat"))


def test_c_caller_builds_and_links(kat_exe):
    assert kat_exe.exists()


@pytest.mark.gpu
def test_c_known_answers_on_gpu(kat_exe):
    env = dict(os.environ, LD_LIBRARY_PATH=str(PKG))
    r = subprocess.run([str(kat_exe)], capture_output=True, text=True, env=env, timeout=300)
    print(r.stdout)
    assert r.returncode == 0 and "ALL PASSED" in r.stdout, r.stdout + r.stderr
