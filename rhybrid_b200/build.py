"""Builds the CUDA library librhgpu.so in-tree for sm_100a (B200).

Every translation unit under csrc/ (the host side of the C ABI, rhgpu*.cu, and
the kernel definitions of each family, k_*.cu) is compiled to an object in
_build/, in parallel, and linked into one shared library that exports only
the C ABI (rhgpu_* symbols).

FP64 kernels are compiled with --fmad=false (no fused multiply-add
contraction) and IEEE-rounded division and square root, so that they
evaluate the reference's expressions with the same rounding as its CPU build.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "librhgpu.so")
EXPORTS = os.path.join(CSRC, "exports.map")
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "--fmad=false",
         "-prec-div=true", "-prec-sqrt=true", "-ftz=false", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-Xfatbin=-compress-all"]


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(HERE, "..", "include", "rhgpu.h")]


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in deps())


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    return subprocess.run(cmd, capture_output=True, text=True)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> str:
    if up_to_date() and not force and not ptxas_info:
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    jobs = [(s, os.path.join(OBJ, s[:-3] + ".o")) for s in sources()]
    cmds = [[NVCC] + FLAGS + extra + ["-c", os.path.join(CSRC, s), "-o", o] for s, o in jobs]
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda c: _run(c, verbose), cmds))
    failed = [r for r in results if r.returncode != 0]
    if ptxas_info:
        for r in results:
            sys.stderr.write(r.stderr)
    if failed:
        for r in failed:
            sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    link = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xlinker", f"--version-script={EXPORTS}"] + \
        [o for _, o in jobs] + ["-o", OUT]
    r = _run(link, verbose)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc link failed")
    return OUT


if __name__ == "__main__":
    build(verbose=True, force=True, ptxas_info="-v" in sys.argv)
