"""Builds video-to-3d_b200/lib/libv3d_dense.so for sm_100a.

Every .cu and .cpp under csrc/ is compiled in parallel with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` (host code with
-ffp-contract=off, so f64 host arithmetic is never fused) and linked with the
static CUDA runtime, so the library loads on machines without a GPU and fails
at context creation instead.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libv3d_dense.so")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
          "-I", os.path.join(HERE, "..", "include")]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _headers_mtime():
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    paths.append(os.path.join(HERE, "..", "include", "v3d_dense.h"))
    return max(os.path.getmtime(p) for p in paths)


def _compile(src, verbose):
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    if os.path.exists(obj) and os.path.getmtime(obj) > max(os.path.getmtime(path), _headers_mtime()):
        return obj
    cmd = [NVCC] + ARCH + COMMON + ["-c", path, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-x", "c++"] + COMMON + ["-c", path, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s%s" % (src, r.stdout, r.stderr))
    return obj


def build(verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(len(srcs), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if os.path.exists(LIB) and os.path.getmtime(LIB) > max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [NVCC, "-shared"] + ARCH + ["-cudart", "static", "-o", LIB] + objs
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
