"""Build libpyfwi_b200.so (the sm_100a kernels and the C ABI of
include/pyfwi_b200.h) in-tree with nvcc.

    python -m pyfwi_b200.build
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libpyfwi_b200.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("pyfwi_b200.cu", "static_scratch.cu", "lowpass.cu")]
DEPS = SOURCES + [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))] + \
    [os.path.join(ROOT, "include", "pyfwi_b200.h")]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC,-O3", "-shared", "-I" + os.path.join(ROOT, "include"),
              "-I" + os.path.join(HERE, "csrc")]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in DEPS if os.path.exists(d))


def build(force=False, verbose=False):
    """Compile the library unless it is newer than every source."""
    if not force and up_to_date():
        return LIB
    tmp = LIB + ".tmp%d" % os.getpid()
    cmd = [nvcc()] + NVCC_FLAGS + SOURCES + ["-o", tmp]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
