"""Build libcpipe_b200.so in-tree (cpipe_b200/_lib/) for sm_100a.

Every .cu file is compiled by nvcc with `-gencode arch=compute_100a,code=sm_100a`
and -fmad=false (the node math is specified without fused multiply-add); the C++
host files are compiled by nvcc's host compiler with -ffp-contract=off for the
same reason.  The CUDA runtime is linked statically so the library does not
depend on which libcudart the embedding process loads.

    python -m cpipe_b200.build          # incremental
    python -m cpipe_b200.build --clean  # from scratch
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIB = os.path.join(OUT_DIR, "libcpipe_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "nvcc")
QUIET = ["-Wno-deprecated-gpu-targets"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
                   "-I", INCLUDE, "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-Wall", "-I", INCLUDE]


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _headers_mtime():
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    paths += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return max(os.path.getmtime(p) for p in paths)


def _compile(src):
    path = os.path.join(CSRC, src)
    obj = os.path.join(OBJ_DIR, src + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(path), _headers_mtime()):
        return obj
    flags = CU_FLAGS if src.endswith(".cu") else CXX_FLAGS
    cmd = [NVCC] + QUIET + flags + ["-c", path, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-x", "c++"] + QUIET + flags + ["-c", path, "-o", obj]
    subprocess.check_call(cmd)
    return obj


def build(clean=False, verbose=True):
    if clean and os.path.isdir(OUT_DIR):
        shutil.rmtree(OUT_DIR)
    os.makedirs(OBJ_DIR, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(_compile, sources()))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        subprocess.check_call([NVCC] + QUIET + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs +
                              ["-Xlinker", "--no-undefined", "-lpthread", "-ldl", "-lrt"])
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(clean="--clean" in sys.argv)
