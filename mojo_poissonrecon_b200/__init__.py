"""B200-native screened Poisson surface reconstruction (sm_100a CUDA kernels).

A drop-in for mojo-poissonrecon's Python API (python/mojo_poissonrecon/
__init__.py): the same public names, signatures, defaults and return types,
computed on the GPU through the C ABI of libpoisson_b200.so.
"""

from .buildlib import build
from .core import (
    FlatOctree,
    GridSolution,
    Mesh,
    build_octree,
    extract_isosurface,
    oriented_points_from_mesh,
    reconstruct,
    reconstruct_mesh,
    solve_screened_poisson,
)
from .attributes import interpolate_attributes
from .ply import read_ply, write_ply

__version__ = "0.1.0"
__all__ = [
    "FlatOctree",
    "GridSolution",
    "Mesh",
    "build",
    "build_octree",
    "extract_isosurface",
    "interpolate_attributes",
    "oriented_points_from_mesh",
    "reconstruct",
    "read_ply",
    "reconstruct_mesh",
    "solve_screened_poisson",
    "write_ply",
]
