"""Compile the sm_100a CUDA library `libpoisson_b200.so` in-tree with nvcc.

Every translation unit is compiled with `-gencode arch=compute_100a,code=sm_100a`
and `-lineinfo`.  Units whose FP64 results must match the serial reference bit
for bit are compiled with `-fmad=false` (no fused multiply-add); the FP32
solver units keep FMA.  The CUDA runtime is linked statically, so the library
needs only the driver at run time.

`--checked` builds `libpoisson_b200_checked.so` instead: the same sources with
`-DPB_CHECKED` and relocatable device code (one device error word shared by
every unit), whose index helpers and guarded stores report out-of-range
indices to that word instead of touching memory (`csrc/checked.cuh`).

    python -m mojo_poissonrecon_b200.buildlib [--force] [--verbose] [--checked]
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
CHECKED_LIBRARY = os.path.join(HERE, "libpoisson_b200_checked.so")
OBJDIR = os.path.join(HERE, "_build")
CHECKED_OBJDIR = os.path.join(HERE, "_build_checked")
CHECKED_FLAGS = ["-DPB_CHECKED", "-rdc=true"]
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


def _compile(src: str, verbose: bool, checked: bool = False) -> tuple[str, str]:
    obj = os.path.join(CHECKED_OBJDIR if checked else OBJDIR, src[:-3] + ".o")
    flags = ARCH + COMMON + ["-I", INCLUDE] + (CHECKED_FLAGS if checked else [])
    if src in EXACT_FP64:
        flags += ["-fmad=false"]
    if verbose:
        flags += ["-Xptxas", "-v"]
    cmd = [nvcc(), "-c", os.path.join(CSRC, src), "-o", obj] + flags
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode:
        raise RuntimeError(f"nvcc failed on {src}:\n{proc.stderr[-6000:]}")
    return obj, proc.stderr


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> str:
    """Build (if stale) and return the path of libpoisson_b200.so (checked=True:
    libpoisson_b200_checked.so)."""
    library = CHECKED_LIBRARY if checked else LIBRARY
    if not force and os.path.exists(library) and os.path.getmtime(library) >= _deps_mtime():
        return library
    os.makedirs(CHECKED_OBJDIR if checked else OBJDIR, exist_ok=True)
    srcs = sources()
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as pool:
        results = list(pool.map(lambda s: _compile(s, verbose, checked), srcs))
    if verbose:
        for (_, log), src in zip(results, srcs):
            if log.strip():
                print(f"== {src}\n{log}", file=sys.stderr)
    tmp = library + ".tmp"
    cmd = [nvcc(), "-shared", "-o", tmp] + ARCH + (["-rdc=true"] if checked else []) + [obj for obj, _ in results]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode:
        raise RuntimeError(f"nvcc link failed:\n{proc.stderr[-6000:]}")
    os.replace(tmp, library)
    return library


if __name__ == "__main__":
    parser = argparse.ArgumentParser()
    parser.add_argument("--force", action="store_true")
    parser.add_argument("--verbose", action="store_true")
    parser.add_argument("--checked", action="store_true")
    args = parser.parse_args()
    print(build(force=args.force, verbose=args.verbose, checked=args.checked))
