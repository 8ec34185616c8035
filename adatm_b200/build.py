"""Build libadatm_b200.so in-tree: nvcc for sm_100a, static CUDA runtime.

Usage: python -m adatm_b200.build [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libadatm_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                "-I", os.path.join(ROOT, "include"), "-I", CSRC, "--expt-relaxed-constexpr",
                "-ccbin", "/usr/bin/g++"]
SOURCES = ["scan.cu", "csf_build.cu", "mttkrp.cu", "als.cu", "mlp.cu", "engine.cu", "planner.cpp", "api.cu"]


def _headers_mtime() -> float:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    hs += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    return max(os.path.getmtime(h) for h in hs)


def _compile(src: str, force: bool, hmt: float) -> str:
    s = os.path.join(CSRC, src)
    o = os.path.join(OBJ, src + ".o")
    if (not force and os.path.exists(o) and os.path.getmtime(o) >= os.path.getmtime(s)
            and os.path.getmtime(o) >= hmt):
        return o
    cmd = [NVCC] + FLAGS + ["-x", "cu" if src.endswith(".cu") else "c++", "-c", s, "-o", o]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return o


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hmt = _headers_mtime()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, hmt), SOURCES))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-ccbin", "/usr/bin/g++", "-o", LIB] + objs + [
            "-lrt", "-ldl", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    _build_cli(force)
    if verbose:
        print(LIB)
    return LIB


CLI_SRC = os.path.join(HERE, "cli", "splatt_cli.c")
CLI = os.path.join(HERE, "splatt")


def _build_cli(force: bool = False) -> str:
    """The `splatt` command (cpd, bench -a adatm), linked to the library with
    an $ORIGIN run path so it finds libadatm_b200.so beside itself."""
    if (not force and os.path.exists(CLI) and os.path.getmtime(CLI) >= os.path.getmtime(CLI_SRC)
            and os.path.getmtime(CLI) >= os.path.getmtime(LIB)):
        return CLI
    cmd = ["gcc", "-O2", "-std=gnu99", "-Wall", "-I", os.path.join(ROOT, "include"), CLI_SRC,
           "-o", CLI, "-L", HERE, "-ladatm_b200", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building the splatt command failed:\n{r.stdout}\n{r.stderr}")
    return CLI


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
