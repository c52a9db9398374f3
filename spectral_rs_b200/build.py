"""Build libspectral_gpu.so in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs=3):
    subprocess.check_call(["make", "-C", os.path.join(HERE, "csrc"), f"-j{jobs}"])
    return os.path.join(HERE, "libspectral_gpu.so")


if __name__ == "__main__":
    print(build(int(sys.argv[1]) if len(sys.argv) > 1 else 3))
