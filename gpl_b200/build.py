"""Builds the engine's shared library, gpl_b200/libgpl_b200.so, for sm_100a (nvcc + g++).

The reference-ordered kernels are compiled with --fmad=false (no fused multiply-add on the
paths whose float results must equal the reference's); the solver's GEMMs are not.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
SO = os.path.join(HERE, "libgpl_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fno-fast-math",
          "-I", os.path.join(CSRC, "kernels"), "-I", os.path.join(CSRC, "host")]
# (source, exact float order?)
CU = [("kernels/nesterov_kernels.cu", True), ("kernels/bicgstab.cu", True), ("kernels/rudy.cu", True),
      ("kernels/poisson.cu", False), ("kernels/b2b.cu", True), ("kernels/adjoint.cu", False), ("kernels/poisson_tc.cu", False), ("kernels/cell_order.cu", True), ("host/engine.cu", True),
      ("host/capi_kernels.cu", True), ("host/bicgstab_noalloc.cu", True)]
CPP = ["host/place.cpp", "host/nesterov.cpp", "host/tune.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def sources():
    out = []
    for root, _, files in os.walk(CSRC):
        out += [os.path.join(root, f) for f in files]
    return out + [os.path.join(os.path.dirname(HERE), "include", "gpl.h"), __file__]


def build(force=False, verbose=False):
    if not force and os.path.exists(SO) and max(os.path.getmtime(s) for s in sources()) < os.path.getmtime(SO):
        return SO
    os.makedirs(OUT, exist_ok=True)
    jobs = []
    for src, exact in CU:
        obj = os.path.join(OUT, src.replace("/", "_") + ".o")
        flags = ["--fmad=false"] if exact else []
        jobs.append([NVCC] + ARCH + COMMON + flags + ["-c", os.path.join(CSRC, src), "-o", obj])
    for src in CPP:
        obj = os.path.join(OUT, src.replace("/", "_") + ".o")
        jobs.append(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
                     "-Wno-unused-function", "-I/usr/local/cuda/include", "-I", os.path.join(CSRC, "host"),
                     "-c", os.path.join(CSRC, src), "-o", obj])
    with ThreadPoolExecutor(max_workers=8) as ex:
        logs = list(ex.map(_run, jobs))
    if verbose:
        print("\n".join(l for l in logs if l.strip()))
    objs = [j[j.index("-o") + 1] for j in jobs]
    _run([NVCC] + ARCH + ["-shared", "-o", SO] + objs + ["-lcudart"])
    return SO


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(SO)
