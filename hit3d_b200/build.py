"""Build the sm_100a shared library libhit3d_gpu.so in-tree with nvcc.

The library is the product: the C-ABI declared in include/hit3d_gpu.h.  It is
built beside this file so that it travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libhit3d_gpu.so")
SOURCES = ["hit3d.cu", "xpass_f64.cu", "xpass_f32.cu", "noalloc.cu", "mlp.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
OBJDIR = os.path.join(HERE, "_build")


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "hit3d_gpu.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    """Compile every translation unit in parallel (nvcc -c), then link the library."""
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(OBJDIR, exist_ok=True)
    flags = ["-O3", "-std=c++17", *ARCH, "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC"]
    if verbose:
        flags += ["-Xptxas", "-v"]
    flags += list(extra or [])

    def compile_one(src):
        obj = os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")
        res = subprocess.run([nvcc(), *flags, "-c", "-o", obj, os.path.join(CSRC, src)], capture_output=True, text=True)
        return src, obj, res

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    failed = False
    for src, _, res in results:
        if res.returncode != 0 or verbose:
            sys.stderr.write(res.stdout + res.stderr)
        failed |= res.returncode != 0
    if failed:
        raise RuntimeError("nvcc failed building libhit3d_gpu.so")
    res = subprocess.run([nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *[o for _, o, _ in results]],
                         capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed linking libhit3d_gpu.so")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
