"""Build the in-tree CUDA library ``lib/libgocean.so`` for sm_100a, and its
checked-index twin ``lib/libgocean_debug.so`` (the stage-kernel units again
with -DGO_DEBUG_BOUNDS: every global access and shared ring read of the
stage kernels tests its index and flags GO_STATUS_BOUNDS instead of going
outside its array).

    python gpu-ocean_b200/build.py [--force]

The floating-point flags are the reference's own (gpu_ocean/SWESimulators/
CDKLM16.py:196-200): --ftz=true --prec-div=false --prec-sqrt=false
--fmad=false (the adjoint unit contracts FMAs and the drifter unit uses
nvcc's defaults as the reference's drifter kernels do, see UNIT_FLAGS).
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib", "libgocean.so")
# the checked-index build: the units that instantiate the stage kernels are
# compiled again with -DGO_DEBUG_BOUNDS and linked with the other objects
DEBUG_LIB = os.path.join(HERE, "lib", "libgocean_debug.so")
DEBUG_UNITS = ("batch.cu", "pair_batch_frame.cu", "pair_batch_int_f0.cu", "pair_batch_int_f1.cu",
               "pair_batch_int_f2.cu", "pair_single_frame.cu", "pair_single_int_f0.cu", "pair_single_int_f1.cu",
               "pair_single_int_f2.cu", "stage_launch.cu")
INCLUDE = os.path.join(ROOT, "include")

NVCC_FLAGS = [
    "-O3", "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "--ftz=true", "--prec-div=false", "--prec-sqrt=false", "--fmad=false",
    "-Xcompiler", "-fPIC",
]


# Units whose flags differ: the adjoint is not bit-compared with the
# reference and keeps the forward's rounding only where a branch depends on
# it (written out with __fmul_rn in the source), so it may contract FMAs.
UNIT_FLAGS = {"adjoint.cu": {"--fmad=false": "--fmad=true"},
              # the reference builds its drifter kernels with nvcc's defaults
              "drifters.cu": {"--ftz=true": "--ftz=false", "--prec-div=false": "--prec-div=true",
                              "--prec-sqrt=false": "--prec-sqrt=true", "--fmad=false": "--fmad=true"}}
# ... and its boundary kernels (open boundaries) the same way
UNIT_FLAGS["open_boundaries.cu"] = UNIT_FLAGS["drifters.cu"]
# the model-error kernels with --use_fast_math (OceanStateNoise.py:222-227):
# flush to zero, approximate division and square root (already set), FMA
# contraction and the fast intrinsics for logf, expf, sinf, cosf
UNIT_FLAGS["ocean_noise.cu"] = {"--fmad=false": "--use_fast_math"}
# Flags added for some units.  The single-domain column-pair region kernel is
# allocated at ptxas register-usage level 10 (the same arithmetic, so the same
# bits): measured on a B200 at 4096^2, 579-584 us per RK2 step against 588-589
# at the default level, and 623-629 at levels 0 and 2; the batched kernel was
# 0.2% slower at level 10 and stays at the default.
UNIT_EXTRA = {u: ["-Xptxas", "--register-usage-level=10"]
              for u in ("pair_single_int_f0.cu", "pair_single_int_f1.cu", "pair_single_int_f2.cu")}


def flags_for(unit):
    """nvcc flags of one source unit; GOCEAN_NVCC_FLAGS appends more (e.g.
    -DGO_PACKED_PAIRS for the packed-sum build of the stage kernel)."""
    sub = UNIT_FLAGS.get(unit, {})
    return ([sub.get(f, f) for f in NVCC_FLAGS] + UNIT_EXTRA.get(unit, [])
            + os.environ.get("GOCEAN_NVCC_FLAGS", "").split())


def sources():
    # this file too: its flags are part of what the libraries are built from
    out = [os.path.join(INCLUDE, "gocean.h"), os.path.abspath(__file__)]
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cuh", ".h")):
            out.append(os.path.join(CSRC, f))
    return out


def up_to_date():
    if not os.path.exists(LIB) or not os.path.exists(DEBUG_LIB):
        return False
    t = min(os.path.getmtime(LIB), os.path.getmtime(DEBUG_LIB))
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force=False, verbose=False):
    """Compile each csrc/*.cu to an object in parallel, then link."""
    if not force and up_to_date():
        return LIB
    import shutil
    import tempfile
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    units = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    work = tempfile.mkdtemp(prefix="gocean_build_")
    try:
        def compile_one(job):
            u, debug = job
            obj = os.path.join(work, u + (".debug.o" if debug else ".o"))
            extra = ["-DGO_DEBUG_BOUNDS"] if debug else []
            cmd = [nvcc] + flags_for(u) + extra + ["-I", INCLUDE, "-c", os.path.join(CSRC, u), "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
            return obj
        jobs = [(u, False) for u in units] + [(u, True) for u in units if u in DEBUG_UNITS]
        with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
            objs = dict(zip(jobs, ex.map(compile_one, jobs)))
        for out, pick in ((LIB, lambda u: objs[(u, False)]),
                          (DEBUG_LIB, lambda u: objs[(u, u in DEBUG_UNITS)])):
            cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a"] + [pick(u) for u in units]
            subprocess.run(cmd + ["-o", out + ".tmp"], check=True)
            os.replace(out + ".tmp", out)
    finally:
        shutil.rmtree(work, ignore_errors=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
