"""Compile the CUDA library in-tree: surfmol_b200/_lib/libsurfmol_b200.so (sm_100a)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libsurfmol_b200.so")
SOURCES = ["relax.cu", "grid.cu", "raff.cu", "topology.cpp", "abi.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = os.path.join(home, "bin", "nvcc")
    return p if os.path.exists(p) else "nvcc"


def host_cxx() -> list:
    # nvcc's host compiler: the system g++ (the image's CXX wrapper lacks OpenMP/spec files)
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def build(verbose: bool = False, extra: list | None = None) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OUT_DIR, src + ".o")
        cmd = [nvcc(), *host_cxx(), "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-O3",
               "-c", path, "-o", obj]
        if src.endswith(".cu"):
            cmd += ["--expt-relaxed-constexpr"]
            if src in ("relax.cu", "raff.cu"):
                cmd += ["-use_fast_math"]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        if extra:
            cmd += extra
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src}")
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(obj)
    cmd = [nvcc(), *host_cxx(), "-shared", *ARCH, "-cudart", "static", "-o", LIB, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
