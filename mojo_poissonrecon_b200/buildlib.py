"""Compile the sm_100a CUDA library `libpoisson_b200.so` in-tree with nvcc.

Every translation unit is compiled with `-gencode arch=compute_100a,code=sm_100a`
and `-lineinfo`.  Units whose FP64 results must match the serial reference bit
for bit are compiled with `-fmad=false` (no fused multiply-add); the FP32
solver units keep FMA.  The CUDA runtime is linked statically, so the library
needs only the driver at run time.

    python -m mojo_poissonrecon_b200.buildlib [--force] [--verbose]
"""

from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIBRARY = os.path.join(HERE, "libpoisson_b200.so")
OBJDIR = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "--expt-relaxed-constexpr"]
# Units that restate the reference's FP64 arithmetic exactly.
EXACT_FP64 = {"octree.cu", "splat.cu", "stencil64.cu", "iso.cu", "dual.cu", "prep.cu", "mesh.cu"}


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libpoisson_b200.so")
    return path


def sources() -> list[str]:
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps_mtime() -> float:
    newest = 0.0
    for root in (CSRC, INCLUDE):
        for name in os.listdir(root):
            newest = max(newest, os.path.getmtime(os.path.join(root, name)))
    return max(newest, os.path.getmtime(__file__))


def _compile(src: str, verbose: bool) -> tuple[str, str]:
    obj = os.path.join(OBJDIR, src[:-3] + ".o")
    flags = ARCH + COMMON + ["-I", INCLUDE]
    if src in EXACT_FP64:
        flags += ["-fmad=false"]
    if verbose:
        flags += ["-Xptxas", "-v"]
    cmd = [nvcc(), "-c", os.path.join(CSRC, src), "-o", obj] + flags
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode:
        raise RuntimeError(f"nvcc failed on {src}:\n{proc.stderr[-6000:]}")
    return obj, proc.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    """Build (if stale) and return the path of libpoisson_b200.so."""
    if not force and os.path.exists(LIBRARY) and os.path.getmtime(LIBRARY) >= _deps_mtime():
        return LIBRARY
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = sources()
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as pool:
        results = list(pool.map(lambda s: _compile(s, verbose), srcs))
    if verbose:
        for (_, log), src in zip(results, srcs):
            if log.strip():
                print(f"== {src}\n{log}", file=sys.stderr)
    tmp = LIBRARY + ".tmp"
    cmd = [nvcc(), "-shared", "-o", tmp] + ARCH + [obj for obj, _ in results]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode:
        raise RuntimeError(f"nvcc link failed:\n{proc.stderr[-6000:]}")
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    parser = argparse.ArgumentParser()
    parser.add_argument("--force", action="store_true")
    parser.add_argument("--verbose", action="store_true")
    args = parser.parse_args()
    print(build(force=args.force, verbose=args.verbose))
