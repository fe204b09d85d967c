"""Builds the CUDA library librhgpu.so in-tree for sm_100a (B200).

FP64 kernels are compiled with --fmad=false (no fused multiply-add
contraction) and IEEE-rounded division and square root, so that they
evaluate the reference's expressions with the same rounding as its CPU build.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "librhgpu.so")
SOURCES = ["rhgpu.cu"]
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "--fmad=false",
         "-prec-div=true", "-prec-sqrt=true", "-ftz=false", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-shared"]


def deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(HERE, "..", "include", "rhgpu.h")]


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in deps())


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> str:
    if up_to_date() and not force and not ptxas_info:
        return OUT
    cmd = [NVCC] + FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + \
        [os.path.join(CSRC, s) for s in SOURCES] + ["-o", OUT]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    if ptxas_info:
        sys.stderr.write(r.stderr)
    return OUT


if __name__ == "__main__":
    build(verbose=True, force=True, ptxas_info="-v" in sys.argv)
