"""Build recipe for libiclblas_b200.so (sm_100a) and its checkers.

The library is compiled in-tree with nvcc for sm_100a only and links the
CUDA runtime statically, so the shared object has no dependency besides the
driver.  `build()` also builds the CPU oracle (oracle/Makefile) and, when the
clGPU reference tree is present, the reference's C-API suite linked against
this library (oracle/_ref/ref_capi_tests_b200).
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libiclblas_b200.so")
CSRC = os.path.join(HERE, "csrc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-fvisibility=hidden",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force: bool = False, verbose: bool = False) -> str:
    """Compile every .cu under csrc/ into objects and link the shared library."""
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + [
        os.path.join(ROOT, "include", "iclBLAS.h")]
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    nvcc = _nvcc()
    objs = []
    procs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc, *NVCC_FLAGS, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for s, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {s}:\n{out.decode()}")
    if force or _stale(LIB, objs):
        cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB, *objs,
               "-cudart", "static", "-Xlinker", "--no-undefined"]
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout.decode()}")
    return LIB


def build_oracle(verbose: bool = False) -> None:
    """Build the CPU oracle and, with the reference tree present, its checkers."""
    r = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-j8"], stdout=subprocess.PIPE,
                       stderr=subprocess.STDOUT)
    if verbose or r.returncode != 0:
        print(r.stdout.decode(), file=sys.stderr)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed")
    ref = os.environ.get("ICLB_REFERENCE", "/root/reference")
    if os.path.exists(os.path.join(ref, "tests", "iclBLAS", "test_Sgemm.cpp")):
        r = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-j8", "b200-tests", f"REF={ref}"],
                           stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
        if r.returncode != 0:
            print(r.stdout.decode(), file=sys.stderr)
            raise RuntimeError("reference C-API suite link against the GPU library failed")


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True)
    build_oracle(verbose=True)
    print(LIB)
