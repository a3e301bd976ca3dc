"""Build libncs_b200.so in-tree with nvcc for sm_100a (B200).

Usage: ``python ncs_b200/build.py [--force] [-v]`` (also called by
``__graft_entry__.build``).  Run it as a script: importing the package loads
the library, which must exist first.
The library is a plain C-ABI shared object (include/ncs_b200.h) loaded with
ctypes; it links only the CUDA runtime.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libncs_b200.so")
SOURCES = ["ncs_capi.cu", "ncs_plain.cu", "ncs_warp.cu", "ncs_spectral.cu", "ncs_noalloc.cu",
           "ncs_net.cu", "ncs_masks.cu", "ncs_sim.cu",
           "ncs_norm.cu", "ncs_net_tc.cu", "ncs_adu.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(ROOT, "include", "ncs_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-Wall", "-I", os.path.join(ROOT, "include"), "-o", LIB + ".tmp"]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
