"""Build recipe of ``librbim_sm100.so`` (the CUDA engine behind the C ABI).

The library is compiled in-tree for sm_100a only, with ``nvcc`` directly; it
links the CUDA runtime statically so that it carries no runtime dependency of
its own beyond the driver.
"""

from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "librbim_sm100.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-O2",
    "--expt-relaxed-constexpr",
    "-shared", "-cudart", "static",
]


def sources() -> list:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _newest_input() -> float:
    files = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    files += glob.glob(os.path.join(INCLUDE, "*.h"))
    return max(os.path.getmtime(f) for f in files)


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found; the CUDA engine cannot be built")
    return path


def build(force: bool = False, verbose: bool = False, extra_flags=None) -> str:
    """Compile every ``csrc/*.cu`` into ``librbim_sm100.so`` if it is stale."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest_input():
        return LIB
    tmp = LIB + f".tmp{os.getpid()}"
    cmd = [nvcc(), *NVCC_FLAGS, *(extra_flags or []), "-I", INCLUDE, "-o", tmp, *sources()]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    flags = [a for a in sys.argv[1:] if a.startswith("-")]
    print(build(force=True, verbose=True, extra_flags=flags))
