"""Build step of libshtcuda: nvcc cross-compiles the sm_100a kernels into an
in-tree shared library, shtools_b200/lib/libshtcuda.so.

    python -m shtools_b200.build [--force]

No GPU is needed to build.  The library exports only the C ABI declared in
include/shtcuda.h.
"""
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIBPATH = os.path.join(LIBDIR, "libshtcuda.so")
PROBE_SRC = os.path.join(CSRC, "probe", "fp64_probe.cu")
PROBE_LIB = os.path.join(LIBDIR, "libshtc_probe.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc",
                 shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA extension cannot be built")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def deps():
    return sources() + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [
        os.path.join(ROOT, "include", "shtcuda.h"), os.path.abspath(__file__)]


def flags(extra=()):
    return ["-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC",
            "-Xcompiler", "-O2", "-Xcompiler", "-fvisibility=hidden", "--shared",
            "-I" + os.path.join(ROOT, "include"), *extra]


def _stale(target, inputs):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in inputs)


def _compile_objects(extra, verbose):
    """One nvcc per translation unit, run in parallel; returns the objects."""
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    hdrs = sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [
        os.path.join(ROOT, "include", "shtcuda.h"), os.path.abspath(__file__)]
    objs, procs = [], []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if _stale(obj, [src] + hdrs):
            cmd = [nvcc(), *flags(extra), "-c", "-o", obj + ".tmp", src]
            cmd.remove("--shared")
            if verbose:
                print(" ".join(cmd))
            procs.append((subprocess.Popen(cmd), obj))
    failed = []
    for pr, obj in procs:
        if pr.wait() != 0:
            failed.append(obj)
        else:
            os.replace(obj + ".tmp", obj)
    if failed:
        raise subprocess.CalledProcessError(1, "nvcc -c " + " ".join(failed))
    return objs


def build(force=False, verbose=False, extra=()):
    """Compile libshtcuda.so (translation units in parallel, then one link)
    and the FP64 probe library; returns the path of libshtcuda.so."""
    os.makedirs(LIBDIR, exist_ok=True)
    if force or _stale(LIBPATH, deps()):
        if force:
            for o in glob.glob(os.path.join(LIBDIR, "obj", "*.o")):
                os.remove(o)
        objs = _compile_objects(extra, verbose)
        tmp = LIBPATH + ".tmp"
        cmd = [nvcc(), *ARCH, "--shared", "-Xcompiler", "-fPIC", "-o", tmp, *objs]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        os.replace(tmp, LIBPATH)
    if force or _stale(PROBE_LIB, [PROBE_SRC, os.path.abspath(__file__)]):
        tmp = PROBE_LIB + ".tmp"
        cmd = [nvcc(), "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC",
               "-Xcompiler", "-fvisibility=hidden", "--shared", "-o", tmp,
               PROBE_SRC]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        os.replace(tmp, PROBE_LIB)
    return LIBPATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
