"""Compile the CUDA sources into the in-tree shared library
umagnus_b200/libumagnus_b200.so (sm_100a only)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libumagnus_b200.so")
BUILD = os.path.join(HERE, "_build")
SOURCES = ["ops.cu", "demag.cu", "demag_fast.cu", "engine.cu", "capi.cu", "noalloc.cu", "ovf.cu", "brute.cu", "adjoint.cu"]
# per-file flags: the brute-force kernel keeps the reference's FP64 operation
# order (no fused multiply-adds)
FILE_FLAGS = {"brute.cu": ["-fmad=false"]}
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-rdc=false"]


def _needs(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "umagnus_b200.h"))
    objs, cmds = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _needs(o, [s] + headers):
            cmd = [NVCC] + ARCH + FLAGS + FILE_FLAGS.get(src, []) + ["-c", s, "-o", o]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), flush=True)
            cmds.append(cmd)
    # translation units compile in parallel
    procs = [subprocess.Popen(c) for c in cmds]
    codes = [p.wait() for p in procs]
    if any(codes):
        raise subprocess.CalledProcessError(max(codes), "nvcc")
    if force or _needs(OUT, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose=True, force="-f" in sys.argv, ptxas_info="-v" in sys.argv))
