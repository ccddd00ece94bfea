"""Builds libccstep.so (the sm_100a step library) in place, beside this file.

nvcc cross-compiles for sm_100a without a GPU.  Device code that decides an
integer outcome uses non-fusing _rn intrinsics (see csrc/ccs_device.cuh); the
rest may fuse.  Host code is compiled with -ffp-contract=off so the binary64
routines round once per operation, as the reference's JavaScript does.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libccstep.so")
SOURCES = ["ccs_step.cu", "ccs_contact.cu", "ccs_mesh.cu", "ccs_pp.cu", "ccs_nn.cu", "ccs_fof.cu", "ccs_order.cu", "ccs_api.cu",
           "ccs_build.cu", "ccs_host.cpp"]
HEADERS = ["ccs_device.cuh", "ccs_internal.h", "ccs_umma.cuh", os.path.join("..", "..", "include", "ccstep.h")]

NVCC_FLAGS = [
    "-O3", "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-shared",
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    """Compile the library if any source is newer than it (or force)."""
    if not force and not stale():
        return LIB
    cmd = [_nvcc()] + NVCC_FLAGS + [os.path.join(CSRC, s) for s in SOURCES] + ["-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
