"""Build the reference's own CDKLM16 kernels into oracle/_ref/ (test oracle).

    python oracle/build_ref.py [REFERENCE_ROOT]

The reference (metno/gpu-ocean) JIT-compiles gpu_ocean/SWESimulators/
gpu_kernels/*.cu with PyCUDA.  Those files use legacy texture references
(``texture<float, cudaTextureType2D> x;`` / ``tex2D(x, s, t)``), which CUDA 12
removed.  This recipe copies CDKLM16_kernel.cu, common.cu, max_dt.cu,
boundary_kernels.cu, initBm_kernel.cu, driftKernels.cu,
observationKernels.cu and ocean_noise.cu into a temporary directory,
rewrites each texture reference into a ``__constant__ cudaTextureObject_t``
read with ``tex2D<T>``, and compiles them with the wrapper translation units
in oracle/ref_driver/ into one shared library per compile-time
configuration (the reference bakes NX, NY, DX, DY, GRAV, FRIC into each JIT
module, CDKLM16.py:179-191).  Only the .so files are kept, in oracle/_ref/
(git-ignored).  Nothing else of the reference is modified.
"""

import os
import re
import shutil
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
DRIVER = os.path.join(HERE, "ref_driver")
KERNEL_FILES = ["CDKLM16_kernel.cu", "common.cu", "max_dt.cu", "boundary_kernels.cu", "initBm_kernel.cu",
                "driftKernels.cu", "observationKernels.cu", "ocean_noise.cu"]

# Compile flags of the CDKLM16 module (CDKLM16.py:196-200); the other
# modules are compiled with PyCUDA's defaults.
CDKLM_FLAGS = ["--ftz=true", "--prec-div=false", "--prec-sqrt=false", "--fmad=false"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# (nx, ny, dx, dy, g, r) configurations used by the tests and the bench.
CONFIGS = {
    "golden": dict(nx=50, ny=70, dx=200.0, dy=200.0, g=9.81, r=0.0),
    "bump256": dict(nx=256, ny=256, dx=200.0, dy=200.0, g=9.81, r=0.0),
    "small_beta": dict(nx=96, ny=80, dx=500.0, dy=500.0, g=9.81, r=3e-3),
    "grf4096": dict(nx=4096, ny=4096, dx=500.0, dy=500.0, g=9.81, r=3e-3),
    # the kernel's linear friction branch (CDKLM16_kernel.cu:884-886), which
    # the reference host never enables, built with use_linear_friction
    "small_linear": dict(nx=96, ny=80, dx=500.0, dy=500.0, g=9.81, r=3e-3, linear=True),
}


def _fmt(x):
    # CDKLM16.py:180-190 formats every float define as "{:.12f}f" of the
    # float32 value held by the simulator
    return "{:.12f}f".format(np.float32(x))


def lib_name(cfg, fmad=False):
    tag = "nx%d_ny%d_dx%g_dy%g_g%g_r%g" % (cfg["nx"], cfg["ny"], cfg["dx"], cfg["dy"], cfg["g"], cfg["r"])
    if cfg.get("linear"):
        tag += "_linear"
    return os.path.join(OUT, "libref_cdklm16_%s%s.so" % (tag, "_fmad" if fmad else ""))


_TEX_DECL = re.compile(r"texture<\s*(float4|float)\s*,\s*cudaTextureType2D\s*>\s*(\w+)\s*;")


def rewrite(src):
    """Texture references -> texture objects (the only change made)."""
    names = {}

    def decl(m):
        names[m.group(2)] = m.group(1)
        return "__constant__ cudaTextureObject_t %s;" % m.group(2)

    out = _TEX_DECL.sub(decl, src)
    for name, typ in names.items():
        out = re.sub(r"tex2D\(\s*%s\s*," % name, "tex2D<%s>(%s," % (typ, name), out)
    return out


def stage_sources(ref_root, dst):
    kdir = os.path.join(ref_root, "gpu_ocean", "SWESimulators", "gpu_kernels")
    for f in KERNEL_FILES:
        with open(os.path.join(kdir, f)) as fh:
            s = fh.read()
        with open(os.path.join(dst, f), "w") as fh:
            fh.write(rewrite(s))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s" % (" ".join(cmd), r.stderr[-4000:]))


def build_one(src_dir, cfg, fmad=False):
    target = lib_name(cfg, fmad)
    work = tempfile.mkdtemp(prefix="gocean_ref_obj_")
    try:
        common = ["nvcc", "-O3", "-std=c++14"] + ARCH + ["-Xcompiler", "-fPIC", "-I", src_dir, "-w"]
        cdefs = ["-Dblock_width=12", "-Dblock_height=32",
                 "-DKPSIMULATOR_DESING_EPS=" + _fmt(0.1), "-DKPSIMULATOR_FLUX_SLOPE_EPS=" + _fmt(0.1),
                 "-DKPSIMULATOR_DEPTH_CUTOFF=" + _fmt(1e-5), "-DTHETA=" + _fmt(1.3), "-DRK_ORDER=2",
                 "-DNX=%d" % cfg["nx"], "-DNY=%d" % cfg["ny"], "-DDX=" + _fmt(cfg["dx"]),
                 "-DDY=" + _fmt(cfg["dy"]), "-DGRAV=" + _fmt(cfg["g"]), "-DFRIC=" + _fmt(cfg["r"])]
        if cfg.get("linear"):
            cdefs.append("-Duse_linear_friction")
        flags = list(CDKLM_FLAGS)
        if fmad:
            flags[-1] = "--fmad=true"
        objs = []
        jobs = [
            ("tu_cdklm.cu", cdefs + flags),
            ("tu_bc.cu", ["-Dblock_width=16", "-Dblock_height=16"]),
            ("tu_maxdt.cu", ["-Dblock_width=12", "-Dblock_height=32", "-DNUM_THREADS=256"]),
            ("tu_drift.cu", ["-Dblock_width=64", "-Dblock_height=1"]),
            # OceanStateNoise.py:222-227
            ("tu_noise.cu", ["-Dblock_width=16", "-Dblock_height=16", "--use_fast_math", "--maxrregcount=32"]),
            ("driver.cu", cdefs),
        ]
        for src, extra in jobs:
            obj = os.path.join(work, src + ".o")
            _run(common + extra + ["-c", os.path.join(DRIVER, src), "-o", obj])
            objs.append(obj)
        os.makedirs(OUT, exist_ok=True)
        _run(["nvcc", "-shared"] + ARCH + objs + ["-o", target + ".tmp"])
        os.replace(target + ".tmp", target)
    finally:
        shutil.rmtree(work, ignore_errors=True)
    return target


def up_to_date(cfg, fmad=False):
    t = lib_name(cfg, fmad)
    if not os.path.exists(t):
        return False
    mt = os.path.getmtime(t)
    deps = [os.path.join(DRIVER, f) for f in os.listdir(DRIVER)] + [os.path.abspath(__file__)]
    return all(os.path.getmtime(d) <= mt for d in deps)


def reference_root(argv=None):
    """The gpu-ocean source tree: the first command-line argument, else the
    GOCEAN_REFERENCE environment variable; fails clearly when neither is set."""
    args = [a for a in (sys.argv[1:] if argv is None else argv) if not a.startswith("--")]
    root = args[0] if args else os.environ.get("GOCEAN_REFERENCE")
    if not root:
        raise SystemExit("name the gpu-ocean source tree: build_ref.py <tree> or GOCEAN_REFERENCE=<tree>")
    return root


def build(ref_root, names=None, force=False):
    names = list(CONFIGS) if names is None else names
    todo = []
    for n in names:
        for fmad in ((False, True) if n == "bump256" else (False,)):
            if force or not up_to_date(CONFIGS[n], fmad):
                todo.append((CONFIGS[n], fmad))
    if not todo:
        return []
    if not os.path.isdir(os.path.join(ref_root, "gpu_ocean")):
        raise FileNotFoundError("reference tree not found at %s" % ref_root)
    src_dir = tempfile.mkdtemp(prefix="gocean_ref_src_")
    try:
        stage_sources(ref_root, src_dir)
        with ThreadPoolExecutor(max_workers=min(4, len(todo))) as ex:
            return list(ex.map(lambda a: build_one(src_dir, *a), todo))
    finally:
        shutil.rmtree(src_dir, ignore_errors=True)


if __name__ == "__main__":
    for p in build(reference_root(), force="--force" in sys.argv):
        print(p)
