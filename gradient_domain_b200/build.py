"""Build the sm_100a shared library ``libgd_poisson.so`` in-tree with nvcc.

    python -m gradient_domain_b200.build            # build if sources changed
    python -m gradient_domain_b200.build --force    # rebuild

The library is the C ABI declared in ``include/gd_poisson.h``; the Python
package loads it with ctypes from this directory.
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgd_poisson.so")

# the library links only the CUDA runtime (every kernel, the DCT's FFTs included, is its own)
LINK: list[str] = []

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3",
    "--expt-relaxed-constexpr",
    "-shared",
]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    built = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + [
        os.path.join(ROOT, "include", "gd_poisson.h"), os.path.abspath(__file__)]
    return any(os.path.getmtime(p) > built for p in deps)


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    """Compile every ``csrc/*.cu`` into ``libgd_poisson.so``; returns its path."""
    if not force and not _stale():
        return LIB
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *NVCC_FLAGS, *(extra or []), "-I", os.path.join(ROOT, "include"),
           "-o", tmp, *sources(), *LINK]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    args = sys.argv[1:]
    extra = [a for a in args if a.startswith("-X") or a.startswith("--resource")]
    print(build(force="--force" in args, verbose=True, extra=extra))
