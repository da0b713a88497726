"""Builds liblpm_b200.so (the CUDA library behind include/lpm_b200.h) for sm_100a with nvcc, in the source tree.

    python lpm-solver-trained-coarse-graining_b200/build.py [--force] [--jobs N]

Objects go to _build/ next to this file; the shared library lands beside this file so that it travels with the tree.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblpm_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "--expt-relaxed-constexpr",
         "-I", CSRC, "-I", INCLUDE]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build liblpm_b200.so")
    return exe


def _deps():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(force=False, jobs=None, verbose=True, extra_flags=()):
    """Compile every csrc/*.cu to an object (in parallel) and link the shared library; returns its path."""
    os.makedirs(OBJ, exist_ok=True)
    cus = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    deps = _deps()
    cmds = []
    objs = []
    for cu in cus:
        o = os.path.join(OBJ, os.path.splitext(os.path.basename(cu))[0] + ".o")
        objs.append(o)
        if force or _stale(o, [cu] + deps):
            cmds.append([nvcc()] + ARCH + FLAGS + list(extra_flags) + ["-c", cu, "-o", o])
    jobs = jobs or min(8, os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        for cmd, r in zip(cmds, ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds)):
            if verbose:
                print(" ".join(cmd[-3:]), flush=True)
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError("nvcc failed on %s" % cmd[-3])
    if force or cmds or _stale(LIB, objs):
        link = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print("link", LIB, flush=True)
        subprocess.run(link, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args()
    build(force=a.force, jobs=a.jobs)
