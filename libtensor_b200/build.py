"""Builds the CUDA/C++ library of the B200 block-tensor path in-tree.

    python -m libtensor_b200.build        # -> libtensor_b200/_lib/libltg.so

All device code is compiled for sm_100a only.  Objects go to
libtensor_b200/_build/ (not committed); the shared library lands next to the
package so it travels with the source tree.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libltg.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]

SOURCES = [
    "ltg_host.cpp",
    "ltg_capi.cu",
    "contract_fp64.cu",
    "elementwise.cu",
    "ozaki.cu",
    "noalloc.cu",
    "crt.cu",
    "group.cu",
]
OPTIONAL_SOURCES = []


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _compile(src, obj, verbose):
    path = os.path.join(CSRC, src)
    t_src = os.path.getmtime(path)
    if src.endswith(".cpp"):
        cmd = [os.environ.get("CXX", "g++"), *CXX_FLAGS, "-I/usr/local/cuda/include", "-c", path, "-o", obj]
    else:
        cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, "-c", path, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src}\n{r.stdout}\n{r.stderr}")
    if os.path.getmtime(path) != t_src:          # edited while compiling: not up to date
        os.utime(obj, (t_src, t_src))
    return obj


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "ltg.h"))
    srcs = SOURCES + [s for s in OPTIONAL_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    jobs = []
    objs = []
    for s in srcs:
        obj = os.path.join(BUILD, s.rsplit(".", 1)[0] + ".o")
        objs.append(obj)
        if force or _stale(obj, [os.path.join(CSRC, s), *headers]):
            jobs.append((s, obj))
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for f in [ex.submit(_compile, s, o, verbose) for s, o in jobs]:
            f.result()
    if jobs or not os.path.exists(LIB):
        # --no-undefined: an object compiled from an older source (a changed
        # launcher signature) fails the link instead of loading with a hole
        cmd = [_nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart", "-Xlinker", "--no-undefined"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
