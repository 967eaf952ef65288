"""Builds libbielcc_gpu.so in-tree for sm_100a with nvcc (no JIT, no torch
extension machinery): every csrc/*.cu is compiled in parallel, then linked
into bielcc_b200/libbielcc_gpu.so, which travels with the source tree."""
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbielcc_gpu.so")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fvisibility=hidden"]
# the C ABI symbols carry default visibility via extern "C" + this define
DEFS = ["-DBIELCC_BUILDING"]
HOST_CC = ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []
# FP32 kernels: flush FP32 denormals (values here are O(1e-10..1e3), far from
# the denormal range), so rsqrt / reciprocal need no subnormal fix-ups. FP64
# arithmetic is unaffected by this flag.
PER_FILE = {"field.cu": ["-ftz=true"], "assemble.cu": ["-ftz=true"], "batch.cu": ["-ftz=true"]}


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        [os.path.join(HERE, "..", "include", "bielcc_gpu.h")]
    procs, objs = [], []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [NVCC] + HOST_CC + ARCH + FLAGS + DEFS + PER_FILE.get(os.path.basename(s), []) + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for s, p in procs:
        out = p.communicate()[0].decode()
        if p.returncode != 0:
            failed.append((s, out))
        elif verbose and out.strip():
            print(out)
    if failed:
        for s, out in failed:
            sys.stderr.write(f"--- {s}\n{out}\n")
        raise RuntimeError("nvcc failed on " + ", ".join(os.path.basename(s) for s, _ in failed))
    if force or _stale(LIB, objs):
        cmd = [NVCC] + HOST_CC + ARCH + ["-shared", "-o", LIB] + objs + ["-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
