"""Build recipe for the CPU oracle (test infrastructure only).

    python -m oracle.build          # -> oracle/_build/liboracle.so

The flags target x86-64-v3 (AVX2 + FMA) rather than -march=native so that the
library built here also runs on the GPU host; a*b+c is never contracted into
a fused multiply-add (-ffp-contract=off, which ISO C mode already implies),
as in the reference's default x86-64 build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")
CFLAGS = ["-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-std=c11", "-Wall"]


def build(force=False, verbose=False):
    src = [os.path.join(HERE, "oracle.c")]
    deps = src + [os.path.join(HERE, "oracle.h")]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["gcc", *CFLAGS, *src, "-o", LIB, "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
