"""ctypes binding of libpoisson_b200.so (the sm_100a C ABI in include/poisson_b200.h).

This is the GPU counterpart of the reference's loader
(python/mojo_poissonrecon/_lib.py): a signature table, a lazy `lib()`, and the
buffer guards.  Buffers are CUDA torch tensors passed by `data_ptr()`; every
call is queued on the current torch CUDA stream.  There is no CPU fallback:
without the built library or a CUDA device every entry point raises.
"""

from __future__ import annotations

import ctypes
import os

import torch

from . import buildlib as _build

I = ctypes.c_int64
F = ctypes.c_double
P = ctypes.c_void_p
S = ctypes.c_size_t
C = ctypes.c_int

_SIGNATURES = {
    "pb_last_error": ([], ctypes.c_char_p),
    "pb_version": ([], C),
    "pb_launch_count": ([], ctypes.c_longlong),
    "pb_init": ([C], C),
    "pb_octree_codes_f64": ([P, I, I, P, P], C),
    "pb_octree_workspace_size": ([I, I], S),
    "pb_octree_count": ([P, I, I, P, P, S, P], C),
    "pb_octree_emit": ([I, I, P, I, P, P, P, P, P, P, P, S, P], C),
    "pb_splat_workspace_size": ([I, I], S),
    "pb_splat_f64": ([P, P, I, I, I, P, P, P, P, P, F, P, P, S, P], C),
    "pb_splat_attributes_workspace_size": ([I], S),
    "pb_splat_attributes_f64": ([P, P, I, I, I, P, I, P, P, S, P], C),
    "pb_sample_attributes_f64": ([P, I, P, I, P, I, P, P], C),
    "pb_assemble_f64": ([P, P, P, P, P, I, F, F, P], C),
    "pb_relax_f64": ([P, P, P, I, F, I, P], C),
    "pb_residual_workspace_size": ([I], S),
    "pb_residual_f64": ([P, P, P, P, I, F, P, P, S, P], C),
    "pb_norm_f64": ([P, I, P, P, S, P], C),
    "pb_restrict_f64": ([P, P, I, P], C),
    "pb_prolong_add_f64": ([P, P, I, P], C),
    "pb_iso_value_workspace_size": ([I], S),
    "pb_iso_value_f64": ([P, P, P, I, I, I, P, P, S, P], C),
    "pb_dual_workspace_size": ([I], S),
    "pb_dual_vertices_f64": ([P, P, I, F, P, P, P, I, P, P, S, P], C),
    "pb_dual_vertices_f64_isoptr": ([P, P, I, P, P, P, P, I, P, P, S, P], C),
    "pb_dual_vertex_count_f64_noalloc": ([P, I, F, P, P], C),
    "pb_dual_faces_f64": ([P, I, F, P, P, I, P, P, S, P], C),
    "pb_dual_faces_f64_isoptr": ([P, I, P, P, P, I, P, P, S, P], C),
    "pb_scale_f64": ([P, I, F, P], C),
    "pb_divide_f64": ([P, I, F, P], C),
    "pb_fill_f64": ([P, I, F, P], C),
    "pb_prepare_workspace_size": ([I], S),
    "pb_prepare_points_f64": ([P, P, I, F, P, P, P, P, P, S, P], C),
    "pb_unit_cube_check_f64": ([P, I, P, P], C),
    "pb_map_vertices_f64": ([P, I, P, P], C),
    "pb_level_geometry": ([I, P, P], C),
    "pb_level_setup_f32": ([P, I, F, P, P, P, P], C),
    "pb_defect_workspace_size": ([I], S),
    "pb_defect_f64": ([P, P, P, P, P, I, F, P, P, P, P, S, P], C),
    "pb_fcg_workspace_size": ([I], S),
    "pb_fcg_direction_f64": ([P, P, P, P, P, I, F, P, P, P, S, P], C),
    "pb_fcg_update_f64": ([P, P, P, P, P, P, P, P, I, F, P, P, P, S, P], C),
    "pb_loop_capture_begin": ([P, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_ulonglong)], C),
    "pb_loop_condition": ([ctypes.c_ulonglong, P, P, P, I, P, P], C),
    "pb_loop_capture_end": ([P, P, ctypes.POINTER(ctypes.c_void_p)], C),
    "pb_graph_launch": ([P, P], C),
    "pb_graph_destroy": ([P, P], C),
    "pb_note_launches": ([ctypes.c_longlong], C),
    "pb_sweep_tma_f32": ([P, P, P, P, I, I, I, P, P], C),
    "pb_prolong_fac_f32": ([P, P, P, I, P], C),
    "pb_extract_workspace_size": ([I], S),
    "pb_mesh_normals_workspace_size": ([I, I], S),
    "pb_mesh_normals_count_f64": ([P, I, P, I, P, P, S, P], C),
    "pb_mesh_normals_emit_f64": ([P, I, P, I, P, P, P, S, P], C),
    "pb_extract_count_f64": ([P, I, P, P, P, S, P], C),
    "pb_extract_emit_f64": ([P, P, I, P, P, P, P, P, S, P], C),
    "pb_residual_restrict_f32": ([P, P, P, P, P, I, P], C),
    "pb_residual_restrict_tma_f32": ([P, P, P, P, P, I, P, P], C),
    "pb_galerkin_workspace_size": ([I, C], S),
    "pb_galerkin_f32": ([P, I, C, P, P, P, S, P], C),
    "pb_level27_from7_f32": ([P, I, P, P], C),
    "pb_level27_finish_f32": ([P, I, P, P, P], C),
    "pb_packed27_size": ([I, ctypes.POINTER(I), ctypes.POINTER(I)], C),
    "pb_pack27_f32": ([P, I, P, P, P, P, P], C),
    "pb_relax27p_f32": ([P, P, P, P, P, P, P, I, P], C),
    "pb_residual_restrict27p_f32": ([P, P, P, P, P, P, P, I, P, P, P], C),
    "pb_coarse_inverse_f64": ([P, I, P, P], C),
    "pb_coarse27_image_size": ([I, P], S),
    "pb_coarse27_image_f32": ([I, P, P, P, P, P, P, S, P], C),
    "pb_coarse27_cycle_f32": ([I, P, P, P, P, I, I, I, P], C),
    "pb_batch_desc_bytes": ([I], S),
    "pb_batch_fcg_partials": ([I], I),
    "pb_batch_fcg_blocks": ([I, I], I),
    "pb_batch_describe": ([C, I, P, P, P, P, I, P, S, P], C),
    "pb_batch_launch": ([C, P, I, I, P, I, P], C),
    "pb_batch_loop_condition": ([ctypes.c_ulonglong, P, P, P, I, I, P, P], C),
    "pb_hierarchy_setup_f32": ([I, P, P, I, P, F, P, S, P, P, S, P], C),
    "pb_tune_set": ([I, I, I], C),
    "pb_tune_get": ([I, I], I),
    "pb_tune_clear": ([], C),
    "pb_checked_build": ([], C),
    "pb_check_status": ([ctypes.POINTER(ctypes.c_uint64), C], C),
}

# MPR_B200_CHECKED=1 loads the checked build (bounds-checked indices and stores
# reporting to a device word; pb_check_status) in place of the normal one.
CHECKED = os.environ.get("MPR_B200_CHECKED", "0") == "1"
LIBRARY_PATH = _build.CHECKED_LIBRARY if CHECKED else _build.LIBRARY
_loaded: ctypes.CDLL | None = None


class NativeError(RuntimeError):
    """A libpoisson_b200 call returned a non-zero status."""


def library_path() -> str:
    return LIBRARY_PATH


def lib() -> ctypes.CDLL:
    """Load (building first if the in-tree library is missing) and bind the C ABI."""
    global _loaded
    if _loaded is None:
        path = LIBRARY_PATH
        if not os.path.exists(path):
            path = _build.build(checked=CHECKED)
        cdll = ctypes.CDLL(path)
        for name, (argtypes, restype) in _SIGNATURES.items():
            fn = getattr(cdll, name)
            fn.argtypes = argtypes
            fn.restype = restype
        _loaded = cdll
    return _loaded


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


CHECK_SITES = {1: "padded FP32 level index", 2: "padded index in the FCG passes", 3: "TMA sweep store",
               4: "FCG pass-2 store", 5: "FP32 prolongation store", 6: "FP64 red-black store"}


def decode_check_word(word: int) -> tuple[int, int]:
    """(site, index) of a check word (site 0: no failure); sites in CHECK_SITES."""
    return int(word) >> 56, int(word) & ((1 << 56) - 1)


def check_word(clear: bool = True) -> int:
    """The checked build's device error word (0: no index left its array);
    always 0 in the normal build.  Synchronises the device."""
    word = ctypes.c_uint64()
    check(lib().pb_check_status(ctypes.byref(word), int(clear)), "check status")
    return int(word.value)


def check(status: int, what: str = "") -> None:
    if status != 0:
        message = lib().pb_last_error().decode(errors="replace")
        raise NativeError(f"{what or 'libpoisson_b200'} failed (status {status}): {message}")


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError(
            "mojo_poissonrecon_b200 runs only on a CUDA (sm_100) device; no CUDA device is visible"
        )
    return torch.device("cuda", torch.cuda.current_device())


def stream_handle(stream: torch.cuda.Stream | None = None) -> int:
    s = torch.cuda.current_stream() if stream is None else stream
    return int(s.cuda_stream)


def dptr(t: torch.Tensor | None) -> int | None:
    """Device address of a contiguous CUDA tensor (None passes through as NULL)."""
    if t is None:
        return None
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("device buffers must be CUDA tensors")
    if not t.is_contiguous():
        raise ValueError("device buffers must be contiguous")
    if t.dtype not in (torch.float64, torch.int64, torch.float32, torch.uint8, torch.int32):
        raise TypeError(f"unsupported device buffer dtype {t.dtype}")
    return t.data_ptr() or None


class Workspace:
    """A growable device scratch buffer reused across calls on one stream."""

    def __init__(self, device: torch.device):
        self.device = device
        self.buffer = torch.empty(0, dtype=torch.uint8, device=device)

    def get(self, nbytes: int) -> tuple[int, int]:
        nbytes = max(int(nbytes), 256)
        if self.buffer.numel() < nbytes:
            self.buffer = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        return self.buffer.data_ptr(), self.buffer.numel()
