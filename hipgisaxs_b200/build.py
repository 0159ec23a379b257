"""Builds the hgx CUDA library (hipgisaxs_b200/libhgx.so) for sm_100a with nvcc.

Objects go to hipgisaxs_b200/_build/; the shared library is written in-tree next to this
file so that it travels with the source tree.  Usage:  python -m hipgisaxs_b200.build
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
LIB = os.path.join(HERE, "libhgx.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
                     "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


# per-file extra flags.  ff_exact.cu, sf_liquid.cu and postproc.cu follow the reference's FP64
# arithmetic without fused multiply-adds: the exact triangle form factor's edge and vertex
# terms and the Percus-Yevick function's terms cancel and amplify any difference in rounding,
# and the smearing sums then round as the reference's do (those kernels are memory-bound).
# qgrid.cu likewise: QGrid::create's 2theta is acos(t) with t just below 1 near qy = 0, where
# a one-ulp change of t (a contracted cos_af^2 + cos_ai^2) moves 2theta by up to ~1e-9
# relative; the grid is built once per description.
FILE_FLAGS = {"ff_exact.cu": ["-fmad=false"], "sf_liquid.cu": ["-fmad=false"],
              "postproc.cu": ["-fmad=false"], "qgrid.cu": ["-fmad=false"]}


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith(".cu") or f.endswith(".cpp"))


def _needs(obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, extra_flags=None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h", ".hpp"))]
    headers.append(os.path.join(ROOT, "include", "hgx.h"))
    flags = NVCC_FLAGS + list(extra_flags or [])
    env = dict(os.environ)
    # the system host compiler (the image's default CC/CXX may point at a reduced toolchain)
    env.pop("CC", None)
    env.pop("CXX", None)
    jobs = []
    objs = []
    for src in _sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _needs(obj, [src] + headers):
            cmd = [nvcc(), "-ccbin", "g++"] + flags + FILE_FLAGS.get(os.path.basename(src), []) + \
                ["-c", src, "-o", obj]
            jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        futs = {ex.submit(subprocess.run, cmd, capture_output=True, text=True, env=env): cmd
                for cmd in jobs}
        for f in cf.as_completed(futs):
            r = f.result()
            if verbose or r.returncode != 0:
                sys.stderr.write(" ".join(futs[f]) + "\n" + r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError("nvcc failed: " + " ".join(futs[f]))
    if force or jobs or not os.path.exists(LIB):
        cmd = [nvcc(), "-ccbin", "g++"] + ARCH + ["-shared", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True, env=env)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
