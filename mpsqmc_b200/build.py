"""Build the CUDA engine (libmpsqmc_b200.so) in-tree for sm_100a.

The library is compiled by nvcc directly (no JIT cache), so the built file sits next to this
module and travels with the repository snapshot.
"""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmpsqmc_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh")))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(INCLUDE, "mpsqmc_gpu.h")]
    return all(os.path.getmtime(s) <= t for s in deps)


HOST = os.path.join(HERE, "host")
HOST_LIB = os.path.join(HERE, "libmpsqmc_host.so")


def host_sources() -> list[str]:
    src = os.path.join(HOST, "src")
    return sorted(os.path.join(src, f) for f in os.listdir(src) if f.endswith(".cpp"))


def build_host(force: bool = False) -> str:
    """The reference-compatible C++ classes (host/include) over the engine, as libmpsqmc_host.so."""
    deps = host_sources() + [os.path.join(HOST, "include", f) for f in os.listdir(os.path.join(HOST, "include"))]
    if not force and os.path.exists(HOST_LIB) and all(os.path.getmtime(d) <= os.path.getmtime(HOST_LIB) for d in deps):
        return HOST_LIB
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-I", os.path.join(HOST, "include"), *host_sources(),
           "-L", HERE, "-lmpsqmc_b200", "-Wl,-rpath,$ORIGIN", "-o", HOST_LIB + ".tmp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"host library build failed:\n{r.stdout}\n{r.stderr}")
    os.replace(HOST_LIB + ".tmp", HOST_LIB)
    return HOST_LIB


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        build_host()
        return LIB
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    units = [os.path.join(CSRC, f) for f in ("capi.cu", "noalloc.cu", "batched.cu")]
    cmd = [nvcc, *NVCC_FLAGS, *units, "-o", LIB + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{r.stdout}\n{r.stderr}")
    os.replace(LIB + ".tmp", LIB)
    if verbose:
        print(r.stderr)
    build_host(force=True)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
