"""Device-resident screened-Poisson multigrid.

Reference: python/mojo_poissonrecon/core.py:141-193 (_v_cycle) and :267-296
(hierarchy, cycle loop, final residual).  The reference keeps one NumPy grid
per level and drives the native kernels level by level; here the hierarchy
lives in HBM as torch tensors and every operator is a libpoisson_b200 kernel
on one CUDA stream.

Two solve modes:

* ``precision="fp64"`` — the reference algorithm: V(3,3) cycles with
  red-black Gauss-Seidel, boundary-normalised full weighting, trilinear
  prolongation and 40 sweeps on the 3^3 grid, all in FP64, from the initial
  guess 0.5.  With ``tol=None`` it runs exactly ``cycles`` cycles and is
  bit-identical to the reference.  With ``tol`` it repeats cycles until the
  relative residual ||b - A x||_2 / ||b||_2 <= tol.
* ``precision="fp32_refined"`` — defect correction: the FP64 residual of the
  FP64 iterate drives one FP32 V-cycle on A e = r from e = 0, and x += e in
  FP64, until the FP64 relative residual reaches ``tol``.  (Implemented in
  solver32.py.)
"""

from __future__ import annotations

from dataclasses import dataclass, field

import torch

from . import _native as nat


def level_sizes(n: int) -> list[int]:
    """Grid sides of the hierarchy: n, (n+1)/2, ... down to 3 (core.py:267-269)."""
    sizes = [n]
    while sizes[-1] > 3:
        sizes.append((sizes[-1] + 1) // 2)
    return sizes


@dataclass
class SolveStats:
    cycles: int = 0
    residual_norm: float = float("nan")
    rhs_norm: float = float("nan")
    history: list = field(default_factory=list)

    @property
    def relative_residual(self) -> float:
        if not self.rhs_norm > 0:
            return 0.0 if self.residual_norm == 0 else float("inf")
        return self.residual_norm / self.rhs_norm


class Hierarchy64:
    """FP64 grids of every level, allocated once and reused across cycles."""

    def __init__(self, screen: torch.Tensor, point_weight: float, workspace: nat.Workspace):
        self.device = screen.device
        self.pw = float(point_weight)
        self.sizes = level_sizes(screen.shape[0])
        self.ws = workspace
        self.lib = nat.lib()
        self.stream = nat.stream_handle()
        L, s = self.lib, self.stream
        self.screens = [screen]
        for n in self.sizes[1:]:
            coarse = torch.empty((n, n, n), dtype=torch.float64, device=self.device)
            fine = self.screens[-1]
            nat.check(L.pb_restrict_f64(fine.data_ptr(), coarse.data_ptr(), fine.shape[0], s), "restrict")
            nat.check(L.pb_scale_f64(coarse.data_ptr(), coarse.numel(), 4.0, s), "scale")
            self.screens.append(coarse)
        self.solutions = [torch.empty((n, n, n), dtype=torch.float64, device=self.device) for n in self.sizes]
        self.rhs = [None] + [torch.empty((n, n, n), dtype=torch.float64, device=self.device) for n in self.sizes[1:]]
        self.residuals = [torch.empty((n, n, n), dtype=torch.float64, device=self.device) for n in self.sizes]
        self.norm = torch.empty(1, dtype=torch.float64, device=self.device)

    def fill(self, value: float) -> None:
        for t in self.solutions:
            nat.check(self.lib.pb_fill_f64(t.data_ptr(), t.numel(), value, self.stream), "fill")

    def relax(self, level: int, iterations: int) -> None:
        n = self.sizes[level]
        nat.check(self.lib.pb_relax_f64(self.solutions[level].data_ptr(), self.rhs[level].data_ptr(),
                                        self.screens[level].data_ptr(), n, self.pw, iterations, self.stream),
                  "relax")

    def residual(self, level: int, out_norm: torch.Tensor | None = None) -> None:
        n = self.sizes[level]
        ptr, size = self.ws.get(self.lib.pb_residual_workspace_size(n))
        norm = self.norm if out_norm is None else out_norm
        nat.check(self.lib.pb_residual_f64(self.solutions[level].data_ptr(), self.rhs[level].data_ptr(),
                                           self.screens[level].data_ptr(), self.residuals[level].data_ptr(), n,
                                           self.pw, norm.data_ptr(), ptr, size, self.stream), "residual")

    def v_cycle(self, level: int, pre: int = 3, post: int = 3) -> None:
        """core.py:141-193."""
        L, s = self.lib, self.stream
        n = self.sizes[level]
        if n <= 3:
            self.relax(level, 40)
            return
        self.relax(level, pre)
        self.residual(level)
        nat.check(L.pb_restrict_f64(self.residuals[level].data_ptr(), self.rhs[level + 1].data_ptr(), n, s),
                  "restrict")
        coarse = self.solutions[level + 1]
        nat.check(L.pb_fill_f64(coarse.data_ptr(), coarse.numel(), 0.0, s), "fill")
        self.v_cycle(level + 1, pre, post)
        nat.check(L.pb_prolong_add_f64(coarse.data_ptr(), self.solutions[level].data_ptr(), n, s), "prolong")
        self.relax(level, post)


def norm(values: torch.Tensor, workspace: nat.Workspace, out: torch.Tensor) -> torch.Tensor:
    L = nat.lib()
    ptr, size = workspace.get(1 << 16)  # per-block partial sums: at most 148*16 doubles
    nat.check(L.pb_norm_f64(values.data_ptr(), values.numel(), out.data_ptr(), ptr, size, nat.stream_handle()),
              "norm")
    return out


def solve_fp64(rhs: torch.Tensor, screen: torch.Tensor, point_weight: float, workspace: nat.Workspace, *,
               cycles: int = 4, tol: float | None = None, max_cycles: int = 200,
               has_points: bool = True) -> tuple[torch.Tensor, SolveStats]:
    """The reference's FP64 solve (core.py:267-296) on device grids.

    Returns the level-0 solution and stats; stats.residual_norm is the absolute
    final ||rhs - A x||_2 as the reference reports it."""
    h = Hierarchy64(screen, point_weight, workspace)
    h.rhs[0] = rhs
    stats = SolveStats()
    h.fill(0.5)  # core.py:270
    if has_points:
        if tol is None:
            for _ in range(cycles):
                h.v_cycle(0)
            stats.cycles = cycles
        else:
            rhs_norm = norm(rhs, workspace, torch.empty(1, dtype=torch.float64, device=rhs.device))
            stats.rhs_norm = float(rhs_norm.item())
            target = tol * stats.rhs_norm
            while stats.cycles < max_cycles:
                h.v_cycle(0)
                stats.cycles += 1
                h.residual(0)
                r = float(h.norm.item())
                stats.history.append(r)
                if r <= target:
                    break
    else:
        nat.check(h.lib.pb_fill_f64(h.solutions[0].data_ptr(), h.solutions[0].numel(), 0.0, h.stream), "fill")
    h.residual(0)  # core.py:289-296: absolute final residual norm
    stats.residual_norm = float(h.norm.item())
    if stats.rhs_norm != stats.rhs_norm:  # nan: not computed yet
        rhs_norm = norm(rhs, workspace, torch.empty(1, dtype=torch.float64, device=rhs.device))
        stats.rhs_norm = float(rhs_norm.item())
    return h.solutions[0], stats
