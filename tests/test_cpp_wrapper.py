"""The C++20 host mirror compiles against the ABI header and library (CPU),
and drives the step on the GPU (gpu)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "wrapper_smoke.cpp")
LIBDIR = os.path.join(ROOT, "frehg_b200")


def build(tmp_path):
    exe = str(tmp_path / "wrapper_smoke")
    cmd = ["g++", "-std=c++20", "-O1", SRC, "-o", exe, f"-L{LIBDIR}", "-lfrehg_gw",
           f"-Wl,-rpath,{LIBDIR}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


@pytest.mark.skipif(not os.path.exists(os.path.join(LIBDIR, "libfrehg_gw.so")),
                    reason="libfrehg_gw.so not built")
def test_wrapper_compiles(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_wrapper_runs_on_gpu(tmp_path):
    exe = build(tmp_path)
    res = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
