"""NVTX ranges around the reconstruction's stages, for profiler timelines.

MPR_B200_NVTX=1 (read at import) makes `stage(name)` push an NVTX range
"mpr:<name>" on entry and pop it on exit (torch.cuda.nvtx); otherwise a stage
costs one flag test.  The stages: prepare, octree, splat, solve, iso,
extract, copy-out (core.reconstruct and friends) and one range per batch
wave (batch.reconstruct_many).
"""

from __future__ import annotations

import contextlib
import os

ENABLED = os.environ.get("MPR_B200_NVTX", "0") == "1"


@contextlib.contextmanager
def stage(name: str):
    if not ENABLED:
        yield
        return
    import torch

    torch.cuda.nvtx.range_push(f"mpr:{name}")
    try:
        yield
    finally:
        torch.cuda.nvtx.range_pop()
