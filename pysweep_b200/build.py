"""Build the CUDA library in-tree with nvcc (sm_100a).

``python -m pysweep_b200.build`` (or ``build()``) compiles
``csrc/pysweep_b200.cu`` into ``libpysweep_b200.so`` next to this file.  The
library is built with ``--fmad=false`` so that every floating-point operation
is rounded separately, as numpy rounds it; the kernels use fma() only where
it is exactly equal to the separate operations.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpysweep_b200.so")
SOURCES = ["pysweep_b200.cu", "noalloc.cu", "adjoint.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
         "-shared"]


def nvcc():
    home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    exe = os.path.join(home, "bin", "nvcc")
    return exe if os.path.exists(exe) else "nvcc"


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "pysweep_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    cmd = [nvcc()] + ARCH + FLAGS + ["-o", LIB + ".tmp"] + srcs + ["-ldl"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
