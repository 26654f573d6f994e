"""Builds libgpl_b200.so (the CUDA library behind include/gpl.h) and the ggplvm CLI in-tree.

Every kernel is compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
there is no other architecture and no fallback. Objects are cached under
``gaspacho2_b200/_build/`` and rebuilt when a source or header is newer.

    python -m gaspacho2_b200.build            # library + CLI
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libgpl_b200.so")
CLI = os.path.join(PKG, "bin", "ggplvm")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, headers, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if _newer(obj, [src] + headers):
        cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if r.stderr.strip() and verbose:
            print(r.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False, jobs: int = 8) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    lib_srcs = [s for s in srcs if not os.path.basename(s).startswith("cli_")]
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, headers, verbose), lib_srcs))
    if _newer(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    # the command-line drop-ins: csrc/cli_<name>.cpp -> bin/<name> (host C++ over the C ABI)
    for cli_src in sorted(glob.glob(os.path.join(CSRC, "cli_*.cpp"))):
        exe = os.path.join(PKG, "bin", os.path.basename(cli_src)[4:-4])
        if _newer(exe, [cli_src, LIB] + headers):
            os.makedirs(os.path.dirname(exe), exist_ok=True)
            cmd = ["/usr/bin/g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", CSRC, cli_src,
                   "-o", exe, "-L", PKG, "-lgpl_b200", "-Wl,-rpath,$ORIGIN/..", "-lz"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"CLI build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
