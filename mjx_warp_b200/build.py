"""Builds libmjb200.so in-tree with nvcc for sm_100a.

  python -m mjx_warp_b200.build [--force]

The CUDA runtime is linked statically so the library does not depend on the runtime version that
ships with torch; the stream handed in through the C ABI is a driver-level handle shared by both.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC_DIR = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmjb200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "mjb200.h")

# No -split-compile: its partitioning of the module changes the generated code from one build of
# the same kernels to the next (one such build ran the small-model solver 17 % slower).
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared", "-cudart", "static"]


def _sources():
  return [os.path.join(SRC_DIR, f) for f in sorted(os.listdir(SRC_DIR))
          if f.endswith((".cu", ".cuh"))] + [HEADER]


def build(force: bool = False, verbose: bool = False) -> str:
  """Compiles csrc/mjb200.cu into libmjb200.so unless it is newer than every source."""
  if not force and os.path.exists(LIB):
    newest = max(os.path.getmtime(s) for s in _sources())
    if os.path.getmtime(LIB) >= newest:
      return LIB
  nvcc = os.environ.get("NVCC", "nvcc")
  cmd = [nvcc, *NVCC_FLAGS, "-o", LIB + ".tmp", os.path.join(SRC_DIR, "mjb200.cu")]
  if verbose:
    cmd.insert(1, "-Xptxas=-v")
  subprocess.check_call(cmd)
  os.replace(LIB + ".tmp", LIB)
  return LIB


if __name__ == "__main__":
  print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
