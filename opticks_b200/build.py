"""Build the in-tree shared library ``opticks_b200/libphox.so`` for sm_100a.

The library holds every CUDA kernel of the engine plus its C ABI (``include/phox.h``).  It is
compiled with ``--use_fast_math`` like the reference's CUDA code
(cmake/Modules/OpticksCUDAFlags.cmake:95), which the bit-exact seqhis comparison depends on.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libphox.so")

SOURCES = ["phx_engine.cu", "phx_bvh.cc"]
HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith((".h", ".cuh")))

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "--use_fast_math", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "-Xptxas", "-warn-spills",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "phox.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, defines=(), out: str | None = None) -> str:
    """compile libphox.so; `defines` (e.g. ["PHX_OUTLINE=0"]) and `out` build variants elsewhere"""
    target = out or LIB
    if not force and not defines and out is None and not needs_build():
        return LIB
    cmd = [_nvcc(), *NVCC_FLAGS, *[f"-D{d}" for d in defines], "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           *[os.path.join(CSRC, s) for s in SOURCES], "-o", target + ".tmp", "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc build of libphox.so failed")
    os.replace(target + ".tmp", target)
    return target


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
