"""Builds the CUDA library ``ecogen_b200/libecg.so`` (sm_100a) and the ``ecogen-b200`` driver.

nvcc compiles every translation unit for ``-gencode arch=compute_100a,code=sm_100a`` with
``--fmad=false`` (no multiply-add contraction, as in the reference's x86-64 build) and links them
into one shared library with a plain C ABI (``include/ecogen_b200.h``).  Objects are rebuilt only
when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.environ.get("ECG_BUILD_DIR", os.path.join(HERE, "_build"))
LIB = os.environ.get("ECG_LIB_OUT", os.path.join(HERE, "libecg.so"))
DRIVER = os.path.join(HERE, "ecogen-b200")
PROBE_LIB = os.path.join(HERE, "libecg_probe.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
           "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")] + os.environ.get("ECG_NVCC_EXTRA", "").split()
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I" + os.path.join(ROOT, "include")]


def _nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return p


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(f) > t for f in [src] + _headers())


def _compile(src: str, extra=None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not _stale(obj, src):
        return obj
    if src.endswith(".cu"):
        cmd = [_nvcc()] + ARCH + NVFLAGS + (extra or []) + ["-c", src, "-o", obj]
    else:
        cmd = ["g++"] + CXXFLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False, jobs: int = 8, lib_only: bool = False) -> str:
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    lib_srcs = [s for s in srcs if not os.path.basename(s).startswith("ecogen_main")]

    def cost(src):  # the kernel-heavy units first (largest previous object), so the jobs finish together
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        return os.path.getsize(obj) if os.path.exists(obj) else (1 << 40 if src.endswith(".cu") else 0)

    order = sorted(lib_srcs, key=cost, reverse=True)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        built = dict(zip(order, ex.map(_compile, order)))
    objs = [built[s] for s in lib_srcs]
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if lib_only:
        return LIB
    # measurement and check probes (FP64 pipe peak for the bench's FP64 roofline; the branch-free
    # division / square root against CUDA's), their own library
    probe_srcs = sorted(glob.glob(os.path.join(HERE, "probe", "*.cu")))
    if probe_srcs:
        pobjs = [_compile(src) for src in probe_srcs]
        if not os.path.exists(PROBE_LIB) or any(os.path.getmtime(o) > os.path.getmtime(PROBE_LIB) for o in pobjs):
            cmd = [_nvcc()] + ARCH + ["-shared", "-o", PROBE_LIB] + pobjs + ["-lcudart"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    main_src = os.path.join(CSRC, "ecogen_main.cpp")
    if os.path.exists(main_src):
        mobj = _compile(main_src)
        if not os.path.exists(DRIVER) or os.path.getmtime(mobj) > os.path.getmtime(DRIVER) or \
                os.path.getmtime(LIB) > os.path.getmtime(DRIVER):
            cmd = ["g++", "-o", DRIVER, mobj, "-L" + HERE, "-lecg", "-Wl,-rpath,$ORIGIN"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print("built", LIB)
    return LIB


BOUNDS_LIB = os.path.join(HERE, "libecg_bounds.so")


def build_bounds(verbose: bool = False, jobs: int = 8) -> str:
    """The bounds-checked library (libecg_bounds.so): every state, face-array and output index of the
    step kernels is checked, counted in ecg_step_stats.bounds_violations and the access skipped when
    outside its buffer.  Built with the generic-EOS kernels only (-DECG_NO_EOS_SPECIALIZATION): the
    EOS-specialised kernels index exactly as the generic ones, and the build is a fraction of the size."""
    env = dict(os.environ, ECG_BUILD_DIR=os.path.join(HERE, "_build_bounds"), ECG_LIB_OUT=BOUNDS_LIB,
               ECG_NVCC_EXTRA="-DECG_BOUNDS_CHECK -DECG_NO_EOS_SPECIALIZATION")
    r = subprocess.run([sys.executable, "-m", "ecogen_b200.build", "--lib-only"], env=env, cwd=ROOT,
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("bounds-checked build failed:\n" + r.stdout[-3000:] + r.stderr[-3000:])
    if verbose:
        print("built", BOUNDS_LIB)
    return BOUNDS_LIB


def ptxas_report(src: str) -> str:
    """Register / shared-memory / spill report of one .cu file (nvcc -Xptxas -v)."""
    cmd = [_nvcc()] + ARCH + NVFLAGS + ["-Xptxas", "-v", "-c", src, "-o", os.devnull]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return r.stdout + r.stderr


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "ptxas":
        print(ptxas_report(sys.argv[2]))
    elif len(sys.argv) > 1 and sys.argv[1] == "bounds":
        build_bounds(verbose=True)
    else:
        build(verbose=True, lib_only="--lib-only" in sys.argv)
