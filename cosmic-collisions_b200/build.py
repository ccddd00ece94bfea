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
SOURCES = ["ccs_step.cu", "ccs_contact.cu", "ccs_mesh.cu", "ccs_pp.cu", "ccs_split.cu", "ccs_nn.cu", "ccs_fof.cu",
           "ccs_order.cu", "ccs_api.cu", "ccs_build.cu", "ccs_host.cpp"]
HEADERS = ["ccs_device.cuh", "ccs_grid.cuh", "ccs_internal.h", "ccs_umma.cuh",
           os.path.join("..", "..", "include", "ccstep.h")]

NVCC_FLAGS = [
    "-O3", "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
]
OBJ = os.path.join(HERE, "_build")


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _newest_header():
    return max(os.path.getmtime(os.path.join(CSRC, h)) for h in HEADERS if os.path.exists(os.path.join(CSRC, h)))


def _obj(src):
    return os.path.join(OBJ, os.path.splitext(src)[0] + ".o")


def _obj_stale(src, hdr_t):
    o = _obj(src)
    return not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(os.path.join(CSRC, src)), hdr_t)


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    """Compile the library if any source is newer than it (or force): one object per source, compiled in
    parallel (only the stale ones), then linked into libccstep.so."""
    if not force and not stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(OBJ, exist_ok=True)
    hdr_t = _newest_header()
    todo = [s for s in SOURCES if force or _obj_stale(s, hdr_t)]

    def compile_one(src):
        cmd = [_nvcc()] + NVCC_FLAGS + ["-c", os.path.join(CSRC, src), "-o", _obj(src) + ".tmp"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError("nvcc failed on %s:\n%s%s" % (src, r.stdout, r.stderr))
        if r.stderr.strip() and verbose:
            print(r.stderr, file=sys.stderr)
        os.replace(_obj(src) + ".tmp", _obj(src))

    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 4))) as ex:
        for f in [ex.submit(compile_one, s) for s in todo]:
            f.result()
    cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a"] + [_obj(s) for s in SOURCES] + \
        ["-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
