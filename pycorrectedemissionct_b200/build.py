"""Build ``libcorrct_b200.so`` (sm_100a) in-tree with nvcc.

Usage: ``python -m pycorrectedemissionct_b200.build`` (also called by
``__graft_entry__.build()``).  The library is written next to this file so it
ships with the source tree; nvcc cross-compiles without a GPU.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB_NAME = "libcorrct_b200.so"
LIB_PATH = os.path.join(HERE, LIB_NAME)

SOURCES = ["cct_api.cu", "cct_project.cu", "cct_maps.cu", "cct_solver.cu", "cct_noalloc.cu", "cct_net.cu", "cct_noise.cu"]
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def build(verbose: bool = False, ptxas_verbose: bool = False, force: bool = False) -> str:
    """Compile the CUDA sources into the in-tree shared library; returns its path."""
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    deps.append(os.path.join(ROOT, "include", "corrct_b200.h"))
    if not force and os.path.exists(LIB_PATH):
        lib_t = os.path.getmtime(LIB_PATH)
        if all(os.path.getmtime(d) <= lib_t for d in deps):
            return LIB_PATH
    cmd = [
        nvcc_path(),
        *ARCH_FLAGS,
        "-O3",
        "-lineinfo",
        "-std=c++17",
        "-Xcompiler",
        "-fPIC",
        "-shared",
        "-cudart",
        "static",
        "-I",
        os.path.join(ROOT, "include"),
        "-o",
        LIB_PATH + ".tmp",
        *srcs,
    ]
    if ptxas_verbose:
        cmd[1:1] = ["-Xptxas", "-v"]
    if verbose:
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{res.stdout}\n{res.stderr}")
    if verbose or ptxas_verbose:
        print(res.stdout + res.stderr)
    os.replace(LIB_PATH + ".tmp", LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(verbose=True, ptxas_verbose="-v" in sys.argv, force="-f" in sys.argv))
