"""Build libtn_cuda.so for sm_100a in-tree (nvcc cross-compiles without a GPU)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8) -> str:
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", os.path.join(HERE, "csrc")], check=True)
    lib = os.path.join(HERE, "lib", "libtn_cuda.so")
    if not os.path.exists(lib):
        raise RuntimeError("libtn_cuda.so was not produced")
    return lib


if __name__ == "__main__":
    print(build(int(sys.argv[1]) if len(sys.argv) > 1 else 8))
