"""Build the CUDA library in-tree: lblrtm_b200/_lib/liblblgpu.so (sm_100a).

Host planning code is compiled by g++ without FMA contraction (its FP64
schedule arithmetic must round exactly as the reference's); the kernels and
the C ABI are compiled by nvcc for sm_100a.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
BUILD = os.path.join(HERE, "_lib", "obj")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SRCS = ["lbl_kernels.cu", "lbl_capi.cu", "lbl_noalloc.cu"]
CPP_SRCS = ["lbl_plan.cpp", "lbl_tape3.cpp"]
HEADERS = ["lbl_kernels.cuh", "lbl_plan.h", "../../include/lblgpu.h", "../data/ref_tables.h",
           "../data/cont_tables.h"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd))
    return r


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS]
    objs = []
    for s in CPP_SRCS:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        if _newer(obj, [src] + hdrs):
            _run(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall",
                  "-c", src, "-o", obj])
        objs.append(obj)
    for s in CUDA_SRCS:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        if _newer(obj, [src] + hdrs):
            _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                  "-Xptxas", "-v" if verbose else "-O3", "-c", src, "-o", obj])
        objs.append(obj)
    lib = os.path.join(OUT, "liblblgpu.so")
    if _newer(lib, objs):
        _run([NVCC, *ARCH, "-shared", "-o", lib, *objs, "-lcudart", "-lpthread"])
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
