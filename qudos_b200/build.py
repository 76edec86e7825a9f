"""Build libqdgpu.so (CUDA sm_100a kernels + C host code) in-tree.

    python qudos_b200/build.py

nvcc cross-compiles for sm_100a without a GPU.  Everything is built with the
per-thread default stream, so that solves driven from several host threads
(the batched entry point) overlap instead of serialising on one stream.  cuBLAS is linked from the CUDA
toolkit (12.9) with an RPATH to it; the CUDA runtime is linked statically.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libqdgpu.so")
OBJ = os.path.join(HERE, "_build")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

CU_SOURCES = ["tables.cu", "assemble.cu", "eig_stage1.cu", "eig_stage2.cu", "eig_driver.cu", "eig_refine.cu",
              "panel_ops.cu", "envelope.cu", "coulomb.cu", "tc_gemm.cu"]
C_SOURCES = ["host_inputs.c", "qd_api.c", "batch.c"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("command failed: " + " ".join(cmd))
    return r.stdout


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "qudos_b200.h"))
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or _stale(o, [s] + headers):
            cmd = [NVCC, "-std=c++17", "-O3", "-lineinfo", "--default-stream", "per-thread", *ARCH, "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include"),
                   "-c", s, "-o", o]
            out = _run(cmd)
            if verbose:
                print(out)
        objs.append(o)
    for src in C_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        if force or _stale(o, [s] + headers):
            _run(["gcc", "-std=gnu11", "-O2", "-fPIC", "-Wall", "-DCUDA_API_PER_THREAD_DEFAULT_STREAM=1", "-I" + os.path.join(ROOT, "include"),
                  "-I" + os.path.join(CUDA, "include"), "-c", s, "-o", o])
        objs.append(o)
    if force or _stale(OUT, objs):
        _run([NVCC, "-shared", *ARCH, "-cudart", "static", "-o", OUT, *objs, "-L" + os.path.join(CUDA, "lib64"),
              "-lcublas", "-Xlinker", "-rpath=" + os.path.join(CUDA, "lib64")])
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
