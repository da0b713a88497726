"""Builds the CPU oracle library (oracle/_build/liblpm_oracle.so) from oracle/lpm_oracle.c with gcc + OpenMP.

TEST INFRASTRUCTURE: the oracle is the checker for the CUDA library and the CPU baseline of bench.py; nothing on the
product path links it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "lpm_oracle.c")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liblpm_oracle.so")


def build(force=False, quiet=False):
    """Compile the oracle if the library is missing or older than its source; returns the library path."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c99", "-Wall", "-o", LIB, SRC, "-lm"]
    if not quiet:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
