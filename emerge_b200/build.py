"""Build ``libemfem.so`` (sm_100a) in-tree with nvcc.

    python -m emerge_b200.build [--force] [--verbose]

The library is a plain C-ABI shared object (``include/emfem.h``); it links only the CUDA runtime.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libemfem.so")
SOURCES = ["emfem_core.cu", "ned2_tet.cu", "robin.cu", "sweep_solve.cu", "sparam.cu", "mesh_conn.cu", "aux_space.cu", "bma.cu", "freq_csr.cu", "multifrontal.cu"]
HEADERS = ["emfem_internal.cuh", "ned2_math.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "emfem.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, obj: str, ptxas_info: bool) -> subprocess.CompletedProcess:
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-c",
           "-I", os.path.join(os.path.dirname(HERE), "include"), "-o", obj, src]
    if ptxas_info:
        cmd += ["-Xptxas", "-v"]
    return subprocess.run(cmd, capture_output=True, text=True)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile every source to an object in parallel (a temporary folder), then link the library."""
    if not force and not _stale():
        return LIB
    import concurrent.futures
    import tempfile
    tmp = LIB + ".tmp"
    with tempfile.TemporaryDirectory(prefix="emfem_build_") as td:
        objs = [os.path.join(td, f.replace(".cu", ".o")) for f in SOURCES]
        with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
            results = list(ex.map(lambda so: _compile(os.path.join(CSRC, so[0]), so[1], ptxas_info),
                                  zip(SOURCES, objs)))
        for f, res in zip(SOURCES, results):
            if res.returncode != 0:
                raise RuntimeError(f"nvcc failed on {f} ({res.returncode}):\n{res.stdout}\n{res.stderr}")
            if verbose or ptxas_info:
                print(f"== {f}\n{res.stderr}", file=sys.stderr)
        link = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs]
        if verbose:
            print(" ".join(link), file=sys.stderr)
        res = subprocess.run(link, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc link failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_info=a.ptxas))
