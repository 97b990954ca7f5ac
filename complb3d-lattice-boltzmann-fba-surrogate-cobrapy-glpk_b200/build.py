"""Build libcomplab_gpu.so in place with nvcc for sm_100a.

Every translation unit under csrc/ is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked into one
shared library next to this file.  Object files go to _build/ (git-ignored);
a unit is recompiled only when it or a header it includes changed.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcomplab_gpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
HOST = os.path.join(HERE, "host")
DRIVER = os.path.join(HERE, "complab_b200")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
    "-I" + INCLUDE,
]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(INCLUDE, "complab_gpu.h"))
    return hs


def _compile(src, extra):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest = max(os.path.getmtime(p) for p in [src] + _headers())
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj, None
    cmd = [_nvcc(), "-c", src, "-o", obj] + NVCC_FLAGS + extra
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, "nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr)
    return obj, None


def build(verbose=False, extra=None):
    extra = list(extra or [])
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, extra), srcs))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("\n".join(errs))
    objs = [o for o, _ in results]
    newest_obj = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest_obj:
        cmd = [_nvcc(), "-shared", "-o", LIB] + objs + [
            "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    build_driver()
    if verbose:
        print("built", LIB)
        print("built", DRIVER)
    return LIB


def build_driver():
    """The host driver (host/*.cpp): CompLaB.xml in, the time loop over the C
    ABI, fields out.  Plain g++, linked against libcomplab_gpu.so next to it."""
    srcs = sorted(os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".cpp"))
    hdrs = [os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".h")]
    newest = max(os.path.getmtime(p) for p in srcs + hdrs + [LIB, os.path.join(INCLUDE, "complab_gpu.h")])
    if os.path.exists(DRIVER) and os.path.getmtime(DRIVER) >= newest:
        return DRIVER
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-o", DRIVER] + srcs + [
        "-I" + INCLUDE, "-L" + HERE, "-lcomplab_gpu", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("host driver build failed:\n%s\n%s" % (r.stdout, r.stderr))
    return DRIVER


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
