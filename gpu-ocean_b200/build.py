"""Build the in-tree CUDA library ``lib/libgocean.so`` for sm_100a.

    python gpu-ocean_b200/build.py [--force]

The floating-point flags are the reference's own (gpu_ocean/SWESimulators/
CDKLM16.py:196-200): --ftz=true --prec-div=false --prec-sqrt=false
--fmad=false.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib", "libgocean.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC_FLAGS = [
    "-O3", "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "--ftz=true", "--prec-div=false", "--prec-sqrt=false", "--fmad=false",
    "-Xcompiler", "-fPIC", "-shared",
]


def sources():
    out = [os.path.join(INCLUDE, "gocean.h")]
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cuh", ".h")):
            out.append(os.path.join(CSRC, f))
    return out


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-I", INCLUDE, os.path.join(CSRC, "gocean.cu"), "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
