"""Builds libwarpmd_rmsd.so for sm_100a with nvcc, in-tree.

    python warp-md_b200/build_native.py [--force] [--debug]

Output: warp-md_b200/warp_md/_native/libwarpmd_rmsd.so (git-ignored; it ships
with the source tree).  Objects go to warp-md_b200/_build/.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT_DIR = os.path.join(HERE, "warp_md", "_native")
LIB = os.path.join(OUT_DIR, "libwarpmd_rmsd.so")
SOURCES = ["wmd_api.cu", "rmsd_frames.cu", "rmsd_lanes.cu", "rmsd_vg.cu", "pairwise.cu", "pairwise_tc.cu", "pairwise_dme.cu", "noalloc.cu", "batched.cu", "superpose.cu", "fluct.cu", "cluster.cu", "dcd.cu"]
HEADERS = ["device_util.cuh", "qcp.cuh", "wmd_internal.h", "pairwise.h", "pairwise_tc.h", "pairwise_dme.h", "batched.h", "superpose.h", "fluct.h", "cluster.h", "dcd.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, debug: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(OUT_DIR, exist_ok=True)
    inc = os.path.join(os.path.dirname(HERE), "include")
    common = [nvcc(), *ARCH, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
              "-I", CSRC, "-I", inc, "--expt-relaxed-constexpr", "-ccbin", shutil.which("g++") or "g++"]
    if debug:
        common += ["-DWMD_DEBUG"]
    if verbose:
        common += ["-Xptxas", "-v"]
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(inc, "warpmd_rmsd.h")]
    objs, cmds = [], []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [path, *hdrs]):
            cmds.append(common + ["-c", path, "-o", obj])
    # translation units compile independently: one nvcc per core
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as pool:
        for cmd in cmds:
            print(" ".join(cmd), flush=True)
        for cmd, rc in zip(cmds, pool.map(lambda c: subprocess.run(c).returncode, cmds)):
            if rc != 0:
                raise subprocess.CalledProcessError(rc, cmd)
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "--cudart", "static", "-o", LIB, *objs, "-Xcompiler", "-fvisibility=hidden"]
        print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.debug, a.verbose))
    sys.exit(0)
