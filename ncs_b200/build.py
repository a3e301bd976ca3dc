"""Build libncs_b200.so in-tree with nvcc for sm_100a (B200).

Usage: ``python ncs_b200/build.py [--force] [-v]`` (also called by
``__graft_entry__.build``).  Run it as a script: importing the package
requires the library, which must exist first.
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
           "ncs_norm.cu", "ncs_net_tc.cu", "ncs_adu.cu", "ncs_tc.cu"]
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
    """Compile each source to an object in parallel (objects under _build/),
    then link the shared library."""
    if not force and not needs_build():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    obj_dir = os.path.join(ROOT, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    common = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-Wall", "-I", os.path.join(ROOT, "include")]
    if verbose:
        common += ["-Xptxas", "-v"]

    def compile_one(src):
        obj = os.path.join(obj_dir, os.path.splitext(src)[0] + ".o")
        subprocess.run(common + ["-c", os.path.join(CSRC, src), "-o", obj], check=True)
        return obj

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs], check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
