"""Builds liblux.so (sm_100a CUDA kernels + C ABI) in-tree with nvcc."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liblux.so")

SOURCES = ["context.cpp", "scene_pack.cpp", "scene.cu", "view.cu", "cache.cu", "screen.cu", "pathtrace.cu", "rate.cu"]
HEADERS = ["lux_internal.h", "lux_math.cuh", "traverse.cuh", "shade.cuh",
           os.path.join("..", "..", "include", "lux.h")]

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    # IEEE binary32 without contraction: the evaluation contract shared with
    # the CPU oracle (bit-identical hit distances and interval radiance).
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
    "-Xcompiler", "-fPIC,-ffp-contract=off",
    "-shared",
]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    built = os.path.getmtime(LIB)
    for name in SOURCES + HEADERS:
        if os.path.getmtime(os.path.join(CSRC, name)) > built:
            return True
    return False


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles liblux.so when a source is newer than the library."""
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
