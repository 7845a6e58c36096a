"""Builds libgalic_cuda.so in-tree for sm_100a (B200).

Every .cu/.cpp file in csrc/ is compiled with nvcc
(`-gencode arch=compute_100a,code=sm_100a -lineinfo`).  The FP64 files are
compiled with `--fmad=false` and the host side with `-ffp-contract=off`: no
multiply-add contraction, so each operation rounds like the reference's
scalar C (the CPU restatement is built the same way).  Files named *_fp32.cu
keep contraction on.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libgalic_cuda.so")
OBJ = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _needs(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "galic_gpu.h"))
    objs = []
    for f in sorted(os.listdir(CSRC)):
        if not f.endswith((".cu", ".cpp")):
            continue
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if not _needs(obj, [src] + headers + [__file__]):
            continue
        fp32 = f.endswith("_fp32.cu")
        fmad = ["--fmad=true", "-ftz=true", "-prec-div=false", "-prec-sqrt=false"] if fp32 else ["--fmad=false"]
        cmd = [NVCC, "-O3", "-std=c++17", *ARCH, "-lineinfo", *fmad, "-Xcompiler", "-fPIC,-ffp-contract=off",
               "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-c", src, "-o", obj]
        if f.endswith(".cu"):
            cmd += ["-Xptxas", "-warn-spills"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if _needs(OUT, objs):
        cmd = [NVCC, "-shared", *ARCH, "-o", OUT, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
