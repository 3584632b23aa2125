"""Build libfastgpu.so in-tree with nvcc for sm_100a.

    python -m fast_b200.build        (or fast_b200.build.build())

The library is written next to this file (fast_b200/libfastgpu.so) so it
travels with the source tree; nothing is installed elsewhere.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libfastgpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    s = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")) + glob.glob(os.path.join(HERE, "csrc", "*.cpp")))
    h = sorted(glob.glob(os.path.join(HERE, "csrc", "*.h")) + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) +
               glob.glob(os.path.join(ROOT, "include", "*.h")))
    return s, h


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    s, h = sources()
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in s + h)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    s, _ = sources()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    common = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp", "-I", os.path.join(ROOT, "include"),
              "-I", os.path.join(HERE, "csrc")]
    procs = []
    for src in s:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        cmd = [nvcc(), *ARCH, *common, "-c", src, "-o", obj]
        if src.endswith(".cu"):
            cmd += ["--expt-relaxed-constexpr", "-Xptxas", "-v"] if verbose else ["--expt-relaxed-constexpr"]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out)
            raise RuntimeError("nvcc failed: " + " ".join(cmd))
        if verbose and out:
            sys.stderr.write(out)
    tmp = LIB + ".tmp"
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-Xcompiler", "-fopenmp", "-lgomp"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
