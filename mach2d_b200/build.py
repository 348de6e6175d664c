"""Builds libmach2d_b200.so in-tree for sm_100a with nvcc.

The library is plain CUDA C++ behind a C ABI (include/mach2d_b200.h); it does
not link against torch.  FP64 kernels are compiled with -fmad=false so that
every a*b+c is rounded twice, as the reference's x86-64 build evaluates it.
Each source compiles to its own object (in parallel, into _build/), then one
link step makes the shared library.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmach2d_b200.so")
OBJ = os.path.join(HERE, "..", "_build", "objs")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", *ARCH, "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                  if f.endswith(".cu") or f.endswith(".cpp"))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(HERE, "..", "include", "mach2d_b200.h"))
    hs.append(os.path.abspath(__file__))
    return [h for h in hs if os.path.exists(h)]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in sources() + headers())


def _obj(src):
    return os.path.join(OBJ, os.path.basename(src) + ".o")


def build(force=False, verbose=False, jobs=None):
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    nvcc = nvcc_path()
    hdr_t = max(os.path.getmtime(h) for h in headers())

    def compile_one(src):
        o = _obj(src)
        if not force and os.path.exists(o) and os.path.getmtime(o) >= max(hdr_t, os.path.getmtime(src)):
            return o
        cmd = [nvcc, *FLAGS, "-c", "-o", o, src]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        return o

    srcs = sources()
    # the largest translation units first, so they do not finish last
    srcs.sort(key=lambda s: -os.path.getsize(s))
    with ThreadPoolExecutor(max_workers=jobs or min(len(srcs), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, srcs))
    cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
