"""Build libhyqmom_b200.so in-tree for sm_100a (nvcc cross-compiles without a GPU).

Strict FP64 semantics for parity with the oracle: no FMA contraction
(-fmad=false); division and square root are IEEE-rounded in FP64 by default.
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
SOURCES = ["hyq_b200.cu", "k_phase_A.cu", "k_phase_EF.cu", "k_cells.cu", "hyq_noalloc.cu", "k_mlp.cu"]
HEADERS = ["hyq_cell.cuh", "hyq_closure.cuh", "hyq_eigen.cuh", "hyq_eig6.cuh", "hyq_charpoly.cuh", "hyq_umma.cuh", "hyq_step.cuh",
           "gen_jacobian6.inc"]
OBJ_DIR = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libhyqmom_b200.so")
INCLUDE = os.path.join(os.path.dirname(PKG), "include", "hyqmom.h")

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-fmad=false", "-std=c++17",
              "-Xcompiler", "-fPIC"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.exists(c) or c == "nvcc"):
            return c
    return "nvcc"


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = [os.path.join(PKG, "csrc", f) for f in SOURCES + HEADERS] + [INCLUDE]
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force=False, verbose=False):
    """Compile the translation units in parallel, then link the shared library."""
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    nvcc = _nvcc()
    procs = []
    for f in SOURCES:
        obj = os.path.join(OBJ_DIR, f.replace(".cu", ".o"))
        cmd = [nvcc] + NVCC_FLAGS + (["-Xptxas=-v"] if verbose else []) + ["-c", "-o", obj, os.path.join(PKG, "csrc", f)]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((f, subprocess.Popen(cmd)))
    bad = [f for f, p in procs if p.wait() != 0]
    if bad:
        raise RuntimeError("nvcc failed for " + ", ".join(bad))
    objs = [os.path.join(OBJ_DIR, f.replace(".cu", ".o")) for f in SOURCES]
    subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB + ".tmp"] + objs)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
