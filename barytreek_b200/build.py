"""Builds libbarytreek_b200.so in-tree with nvcc for sm_100a.

Objects go to barytreek_b200/_build/; the shared library lands next to this
file so it travels with the source tree. Rebuilds only stale objects.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbarytreek_b200.so")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include")]
# Host tree code must evaluate every expression exactly as written (bit-identical
# trees and lists): no contraction into fused multiply-adds.
PER_FILE = {"host_tree.cpp": ["-Xcompiler", "-ffp-contract=off"], "tree_device.cu": ["-Xcompiler", "-ffp-contract=off"],
            "traverse_device.cu": ["-Xcompiler", "-ffp-contract=off"]}
SOURCES = ["host_tree.cpp", "plan.cu", "kernels_updown.cu", "kernels_interact.cu", "kernels_direct.cu",
           "kernels_probe.cu", "kernels_degree.cu", "selector.cu", "direct_noalloc.cu", "batch.cpp", "tree_device.cu", "traverse_device.cu",
           "cc_operators.cu"]
HEADERS = ["btk_internal.h", "kernels.cuh", "device_math.cuh"]


def _host_compiler() -> list[str]:
    # The image's CXX wrapper lacks some runtime pieces; nvcc's default (g++ on
    # PATH) is used unless NVCC_CCBIN is set.
    cc = os.environ.get("NVCC_CCBIN")
    return ["-ccbin", cc] if cc else []


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str) -> tuple[str, str]:
    obj = os.path.join(BUILD, src + ".o")
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(ROOT, "include", "barytreek_b200.h"), __file__]
    if not _stale(obj, deps):
        return obj, ""
    cmd = [NVCC, *_host_compiler(), *ARCH, *COMMON, *PER_FILE.get(src, []), "-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        results = list(ex.map(_compile, SOURCES))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                print(log, file=sys.stderr)
    if _stale(LIB, objs):
        cmd = [NVCC, *_host_compiler(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
