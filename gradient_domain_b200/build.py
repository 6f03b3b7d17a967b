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
from concurrent.futures import ThreadPoolExecutor

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
    """Compile every ``csrc/*.cu`` into ``libgd_poisson.so``; returns its path.

    The translation units share no device code, so each compiles to its own
    object in parallel (under ``_build/``) and one nvcc call links them.
    """
    if not force and not _stale():
        return LIB
    objdir = os.path.join(ROOT, "_build")
    os.makedirs(objdir, exist_ok=True)
    srcs = sources()
    objs = [os.path.join(objdir, os.path.basename(src)[:-3] + ".o") for src in srcs]
    cmds = [[nvcc(), *NVCC_FLAGS, *(extra or []), "-I", os.path.join(ROOT, "include"),
             "-c", "-o", obj, src] for src, obj in zip(srcs, objs)]
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd), flush=True)
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds))
    for cmd, res in zip(cmds, results):
        if res.stdout or res.stderr:
            sys.stdout.write(res.stdout)
            sys.stderr.write(res.stderr)
        if res.returncode != 0:
            raise subprocess.CalledProcessError(res.returncode, cmd)
    tmp = LIB + ".tmp"
    link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
            "-o", tmp, *objs, *LINK]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.run(link, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    args = sys.argv[1:]
    extra = [a for a in args if a.startswith("-X") or a.startswith("--resource")]
    print(build(force="--force" in args, verbose=True, extra=extra))
