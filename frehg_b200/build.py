"""Builds ``libfrehg_gw.so`` in-tree for sm_100a with nvcc.

Usage: ``python -m frehg_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libfrehg_gw.so")
SOURCES = ["gw_api.cu", "gw_kernels.cu", "gw_cg.cu", "gw_cg_mixed.cu", "gw_cg_line64.cu",
           "gw_batch.cu", "gw_serve.cu",
           "gw_couple.cu", "gw_density.cu",
           "gw_setup.cpp"]
HEADERS = ["gw_device.cuh", "gw_internal.h", "gw_setup.h", "gw_coop.cuh", "gw_handle.h",
           "gw_linefactor.cuh", "gw_linesolve.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_compiler() -> str:
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "frehg_gw.h"))
    deps.append(os.path.abspath(__file__))
    return all(os.path.getmtime(p) <= t for p in deps if os.path.exists(p))


def _compile(src: str, obj: str, ptxas_info: bool) -> subprocess.CompletedProcess:
    cmd = [nvcc_path(), "-ccbin", host_compiler(), *ARCH, "-lineinfo", "-O3", "-std=c++17",
           "-Xcompiler", "-fPIC", "-c", "-o", obj, src]
    if ptxas_info:
        cmd[1:1] = ["-Xptxas", "-v"]
    return subprocess.run(cmd, capture_output=True, text=True)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> str:
    """Compiles every source to an object in parallel (no cross-file device
    code, so no device link), then links the shared library."""
    if not force and up_to_date():
        return OUT
    import concurrent.futures
    import tempfile

    with tempfile.TemporaryDirectory(prefix="frehg_build_") as tmp:
        objs = [os.path.join(tmp, os.path.splitext(s)[0] + ".o") for s in SOURCES]
        jobs = max(1, min(len(SOURCES), os.cpu_count() or 1))
        with concurrent.futures.ThreadPoolExecutor(jobs) as ex:
            results = list(ex.map(lambda so: _compile(os.path.join(CSRC, so[0]), so[1], ptxas_info),
                                  zip(SOURCES, objs)))
        for src, res in zip(SOURCES, results):
            if res.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src}:\n" + res.stdout + res.stderr)
            if verbose or ptxas_info:
                sys.stderr.write(res.stderr)
        cmd = [nvcc_path(), "-ccbin", host_compiler(), *ARCH, "-shared", "-o", OUT + ".tmp", *objs]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError("nvcc link failed:\n" + res.stdout + res.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv, ptxas_info="-v" in sys.argv))
