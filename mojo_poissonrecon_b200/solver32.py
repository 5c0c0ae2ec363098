"""FP64-accurate solves driven by FP32 V-cycles (``precision="fp32_refined"``).

Defect correction (method="defect"):

    x = 0.5                                    (the reference's initial guess, core.py:270)
    r = b - A x,  ||r||                        FP64 (pb_defect_f64)
    while ||r|| > tol * ||b||:
        e = V(3,3)-cycle on A e = r from e = 0 FP32 (the reference's cycle shape)
        x = x + e;  r = b - A x                FP64, fused in one kernel

FCG(1) (method="fcg", the default): the same FP32 V-cycle preconditions FP64
flexible conjugate gradients (pb_fcg_step_f64), which needs about 2.5x fewer
V-cycles to reach the same FP64 residual.

The FP32 cycle reuses the reference's operator, red-black smoother, boundary-
normalised full weighting, trilinear prolongation and 40 sweeps on the 3^3
grid (core.py:141-193); levels of side <= 17 run in a single launch.  Each
outer step contracts the error like one FP64 V-cycle while the FP64 residual
keeps the fixed point exact, so the iterate converges to the FP64 solution.
"""

from __future__ import annotations

import ctypes
import math

import torch

from . import _native as nat
from .solver import SolveStats, level_sizes, norm

COARSE_N = 17  # levels of this side or smaller: one single-block launch

# When set to a list, every finest-level sweep launch appends (start, end, mode)
# CUDA events recorded on the launching stream around it (used by bench.py to
# time the dominant kernel inside its timed region).
PROBE: list | None = None


class Level32:
    def __init__(self, n: int, screen64: torch.Tensor, pw: float, device: torch.device, lib, stream):
        self.n = n
        pitch, count = ctypes.c_int64(), ctypes.c_int64()
        nat.check(lib.pb_level_geometry(n, ctypes.byref(pitch), ctypes.byref(count)), "level geometry")
        self.count = count.value

        def zeros():
            return torch.zeros(self.count, dtype=torch.float32, device=device)

        self.D, self.invD, self.rhs, self.res, self.ea, self.eb = (zeros() for _ in range(6))
        nat.check(lib.pb_level_setup_f32(screen64.data_ptr(), n, pw, self.D.data_ptr(), self.invD.data_ptr(),
                                         stream), "level setup")


class Hierarchy32:
    """FP32 levels (padded layout) built from the FP64 screen hierarchy."""

    def __init__(self, screen: torch.Tensor, point_weight: float, workspace: nat.Workspace, z_chunk: int = 0):
        self.status = torch.zeros(1, dtype=torch.int32, device=screen.device)
        self.lib = nat.lib()
        self.stream = nat.stream_handle()
        self.ws = workspace
        self.pw = float(point_weight)
        self.z_chunk = int(z_chunk)
        L, s = self.lib, self.stream
        self.sizes = level_sizes(screen.shape[0])
        screens = [screen]
        for n in self.sizes[1:]:
            coarse = torch.empty((n, n, n), dtype=torch.float64, device=screen.device)
            nat.check(L.pb_restrict_f64(screens[-1].data_ptr(), coarse.data_ptr(), screens[-1].shape[0], s),
                      "restrict")
            nat.check(L.pb_scale_f64(coarse.data_ptr(), coarse.numel(), 4.0, s), "scale")
            screens.append(coarse)
        self.levels = [Level32(n, scr, self.pw, screen.device, L, s) for n, scr in zip(self.sizes, screens)]
        self.first_coarse = next(i for i, n in enumerate(self.sizes) if n <= COARSE_N)
        tail = self.levels[self.first_coarse:]
        k = len(tail)
        ptrs = lambda ts: (ctypes.c_void_p * k)(*[t.data_ptr() for t in ts])
        self._coarse_args = (
            k,
            (ctypes.c_int64 * k)(*[lv.n for lv in tail]),
            ptrs([lv.ea for lv in tail]),
            ptrs([lv.rhs for lv in tail]),
            ptrs([lv.res for lv in tail]),
            ptrs([lv.D for lv in tail]),
            ptrs([lv.invD for lv in tail]),
        )

    def _sweep(self, lv: Level32, src, dst, mode: int, coarse=None) -> None:
        """One red-black sweep dst <- S(src); mode 1 starts from zero, mode 2
        first adds the prolongated coarse correction to src in place."""
        L = self.lib
        if mode == 2:
            nat.check(L.pb_prolong_add_f32(coarse.data_ptr(), src.data_ptr(), lv.n, self.stream), "prolong32")
            mode = 0
        probe = PROBE if (PROBE is not None and lv is self.levels[0]) else None
        if probe is not None:
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
        nat.check(L.pb_sweep_tma_f32(None if src is None else src.data_ptr(), dst.data_ptr(), lv.rhs.data_ptr(),
                                     lv.invD.data_ptr(), lv.n, mode, self.z_chunk, self.status.data_ptr(),
                                     self.stream), "sweep")
        if probe is not None:
            end.record()
            probe.append((start, end, mode))

    def check_status(self) -> None:
        if int(self.status.item()):
            raise RuntimeError("FP32 sweep: a bounded wait on a TMA barrier gave up (status word set)")

    def v_cycle(self, level: int = 0, pre: int = 3, post: int = 3) -> torch.Tensor:
        """Correction for levels[level].rhs from a zero start; returns its tensor."""
        L, s = self.lib, self.stream
        if level >= self.first_coarse:
            k, sizes, e, rhs, res, D, invD = self._coarse_args
            nat.check(L.pb_coarse_cycle_f32(k, sizes, e, rhs, res, D, invD, pre, post, 40, s), "coarse cycle")
            return self.levels[level].ea
        lv = self.levels[level]
        a, b = lv.ea, lv.eb
        # pre-smoothing from zero: a <- S(0), then alternate
        self._sweep(lv, None, a, 1)
        src, dst = a, b
        for _ in range(pre - 1):
            self._sweep(lv, src, dst, 0)
            src, dst = dst, src
        nxt = self.levels[level + 1]
        nat.check(L.pb_residual_restrict_f32(src.data_ptr(), lv.rhs.data_ptr(), lv.D.data_ptr(), nxt.rhs.data_ptr(),
                                             lv.n, s), "residual_restrict32")
        coarse = self.v_cycle(level + 1, pre, post)
        # post-smoothing: the first sweep adds the prolongated correction on load
        self._sweep(lv, src, dst, 2, coarse)
        src, dst = dst, src
        for _ in range(post - 1):
            self._sweep(lv, src, dst, 0)
            src, dst = dst, src
        return src


def solve_refined(rhs: torch.Tensor, screen: torch.Tensor, point_weight: float, workspace: nat.Workspace, *,
                  tol: float = 1e-8, max_cycles: int = 200, has_points: bool = True,
                  z_chunk: int = 0, method: str = "fcg") -> tuple[torch.Tensor, SolveStats]:
    """FP64-accurate solve with FP32 V-cycles.

    method="fcg": flexible conjugate gradients FCG(1) in FP64 with the FP32
    V-cycle as preconditioner (default; about 2.5x fewer V-cycles).
    method="defect": plain defect correction, x += V(r), one V-cycle per step.
    stats.cycles counts V-cycles either way."""
    if method not in ("fcg", "defect"):
        raise ValueError("method must be 'fcg' or 'defect'")
    L = nat.lib()
    s = nat.stream_handle()
    n = rhs.shape[0]
    device = rhs.device
    stats = SolveStats()
    x = torch.empty_like(rhs)
    if not has_points:
        nat.check(L.pb_fill_f64(x.data_ptr(), x.numel(), 0.0, s), "fill")
        stats.residual_norm = 0.0
        stats.rhs_norm = 0.0
        return x, stats
    nat.check(L.pb_fill_f64(x.data_ptr(), x.numel(), 0.5, s), "fill")  # core.py:270
    h = Hierarchy32(screen, point_weight, workspace, z_chunk)
    bnorm = norm(rhs, workspace, torch.empty(1, dtype=torch.float64, device=device))
    norm2 = torch.empty(1, dtype=torch.float64, device=device)
    ws = nat.Workspace(device)
    ptr, size = ws.get(max(L.pb_defect_workspace_size(n), L.pb_fcg_workspace_size(n)))
    r32 = h.levels[0].rhs
    r64 = torch.empty_like(rhs) if method == "fcg" else None
    nat.check(L.pb_defect_f64(x.data_ptr(), None, None, rhs.data_ptr(), screen.data_ptr(), n, h.pw, r32.data_ptr(),
                              None if r64 is None else r64.data_ptr(), norm2.data_ptr(), ptr, size, s), "defect")
    stats.rhs_norm = float(bnorm.item())
    target = tol * stats.rhs_norm
    r = math.sqrt(float(norm2.item()))
    stats.history.append(r)
    if method == "defect":
        x_next = torch.empty_like(rhs)
        while r > target and stats.cycles < max_cycles:
            e = h.v_cycle(0)
            nat.check(L.pb_defect_f64(x.data_ptr(), e.data_ptr(), x_next.data_ptr(), rhs.data_ptr(),
                                      screen.data_ptr(), n, h.pw, r32.data_ptr(), None, norm2.data_ptr(), ptr, size,
                                      s), "defect")
            x, x_next = x_next, x
            stats.cycles += 1
            r = math.sqrt(float(norm2.item()))
            stats.history.append(r)
    else:
        p_prev, p, q = torch.empty_like(rhs), torch.empty_like(rhs), torch.empty_like(rhs)
        scal = torch.zeros(8, dtype=torch.float64, device=device)
        while r > target and stats.cycles < max_cycles:
            z = h.v_cycle(0)
            nat.check(L.pb_fcg_step_f64(z.data_ptr(), p_prev.data_ptr(), p.data_ptr(), q.data_ptr(), x.data_ptr(),
                                        r64.data_ptr(), r32.data_ptr(), screen.data_ptr(), n, h.pw,
                                        scal.data_ptr(), int(stats.cycles == 0), ptr, size, s), "fcg step")
            p_prev, p = p, p_prev
            stats.cycles += 1
            r = math.sqrt(max(float(scal[4].item()), 0.0))
            stats.history.append(r)
        # the recurrence r -= alpha q drifts from b - A x by rounding; report the true residual
        nat.check(L.pb_defect_f64(x.data_ptr(), None, None, rhs.data_ptr(), screen.data_ptr(), n, h.pw,
                                  r32.data_ptr(), None, norm2.data_ptr(), ptr, size, s), "defect")
        r = math.sqrt(float(norm2.item()))
    h.check_status()
    stats.residual_norm = r
    return x, stats
