"""Build libcpsfdtd.so (sm_100a) in-tree with nvcc.

    python -m cpsfdtd_b200.build [--jobs N]

Sources are compiled separately (in parallel) and linked into
cpsfdtd_b200/libcpsfdtd.so; objects go to cpsfdtd_b200/_build/.  The plain
per-routine kernels are compiled with --fmad=false and the host code with
-ffp-contract=off so that FP64 arithmetic keeps the reference's roundings.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libcpsfdtd.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
          "-I" + os.path.join(ROOT, "include"), "-ccbin", "g++"]

SOURCES = {
    "capi.cpp": ["-x", "cu"],
    "host_setup.cpp": ["-x", "cu"],
    "kernels_plain.cu": ["--fmad=false"],
    "kernels_fused.cu": [],
    "kernels_tma.cu": [],
    "kernels_ports.cu": [],
    "kernels_batch.cu": [],
    "kernels_step.cu": [],
    "kernels_three.cu": ["--fmad=false"],
    "raster.cu": ["--fmad=false"],
    "deck_load.cpp": [],
    "image.cu": [],
    "batch.cpp": ["-x", "cu"],
    "server.cpp": ["-x", "cu"],
    "noalloc.cu": [],
}


def _compile(src: str, extra: list, verbose: bool) -> str:
    obj = os.path.join(BUILD, src + ".o")
    cmd = [NVCC] + ARCH + COMMON + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd.append("-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(jobs: int = 8, verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "cps_capi.h")]
    newest = max(os.path.getmtime(p) for p in deps)
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= newest:
        return OUT
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda kv: _compile(kv[0], kv[1], verbose), SOURCES.items()))
    cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart_static", "-ldl", "-lrt", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=8)
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.jobs, a.verbose, a.force))
