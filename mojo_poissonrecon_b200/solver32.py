"""FP64-accurate solves driven by FP32 V-cycles (``precision="fp32_refined"``).

FCG(1) (the default, ``RefinedEngine``): the FP32 V-cycle preconditions FP64
flexible conjugate gradients:

    x = 0.5                                  (the reference's initial guess, core.py:270)
    r = b - A x                              FP64 (pb_defect_f64)
    while ||r|| > tol * ||b||:               evaluated on the device
        z = V-cycle on A e = r, e = 0        FP32
        p = z - beta p;  x += alpha p;  r = b - A x                 FP64 (pb_fcg_direction_f64,
                                                                         pb_fcg_update_f64;
                                                                         p stored in FP32)

One iteration touches the same buffers every time, so the engine captures it
once as the body of a CUDA graph WHILE node whose condition a device kernel
sets from ||r||^2 (pb_loop_condition); a solve is then one graph launch with
no host synchronisation per iteration.  The prologue (level set-up, x0 and its
residual, ||b||) is captured once as a second graph.  Engines (hierarchy,
vectors, graphs) are cached per device, grid side, point weight and slot and
reused across solves.

Defect correction (``precision="fp32_defect"``): x += V(r), one FP32 V-cycle
per FP64 residual, eager launches.

The FP32 cycle: level 0 is the reference's operator with its red-black
Gauss-Seidel smoother (core.py:141-193; the reference runs 3 sweeps each way,
the preconditioner level0_sweeps(n)); the coarser levels are Galerkin
operators with screening-scaled transfers (mg27.cu), smoothed by
COARSE_SWEEPS sweeps each way (on levels of side > 9 with their couplings
packed per colour in FP16), which cut the cycles needed for a given residual
2-4x against the reference's rediscretised hierarchy.  Levels of side <= 9
run in a single launch from shared memory, the 3^3 level solved exactly with
its inverse (built once per set-up).  Convergence is always measured with the
reference's FP64 operator.
"""

from __future__ import annotations

import collections
import ctypes
import math
import threading

import torch

from . import _native as nat
from . import _sync
from .solver import SolveStats, level_sizes, norm

COARSE_N = 9  # levels of this side or smaller: one single-block launch
TMA_MIN_N = 33  # smallest side the TMA sweep takes (level 0 below it is a 27-point level)
COARSE_SWEEPS = 1  # pre- and post-smoothing sweeps on every level below level 0
RESTRICT_VARIANT = 8  # tuning parameter: 2 = level 0's residual-restriction staged by TMA


def level0_sweeps(n: int) -> tuple[int, int]:
    """(pre, post) smoothing sweeps on level 0 of the FCG preconditioner.
    Measured on B200 (solve time to rel-res 1e-8, torus and sphere-union clouds,
    depths 7-9, one or two coarse sweeps, V(1,1) to V(5,5)): V(1,2) with one
    coarse sweep is fastest at every depth tried (depth 8: 6 iterations in
    6.7 ms against 7.1 ms for V(2,2) and 8.1 ms for V(3,3) with two coarse
    sweeps); a cheaper cycle moves the iteration count by one at most."""
    return (1, 2)
MAX_ITER = 512  # capacity of the device iteration history (and hard cap)
GALERKIN_SCRATCH = 512 << 20  # bytes; larger Galerkin products run in slabs of coarse planes

# When true, RefinedEngine runs its iterations as eager launches with a host
# read of the residual after each (the same kernels as the captured loop), for
# profilers that do not follow kernels inside a graph's conditional node.
EAGER_LOOP = False

# When true, each engine captures its per-solve prologue (set-up, start, norm)
# once as a CUDA graph and replays it.
SETUP_GRAPH = True

# Graph captures (the iteration loops here and in batch.py, the prologue graph)
# run one at a time in the process: serving lanes capture on their own
# streams, and the capture APIs are kept out of each other's way.
GRAPH_CAPTURE_LOCK = threading.RLock()

# When set to a list, every finest-level sweep launched eagerly appends
# (start, end, mode) CUDA events recorded on the launching stream around it.
PROBE: list | None = None


class Level32:
    """Padded FP32 arrays of one level (zero-filled so the ghosts stay zero).

    Every level has work arrays (rhs, ea, eb), 1/diagonal (invD) and its
    prolongation weights (weights).  Level 0 also keeps the reference's
    7-point operator as its diagonal D.  Levels that run the 27-point kernels
    (all but a level 0 of side >= TMA_MIN_N) hold their operator as 14 planes
    `coef` and a residual array `res`."""

    def __init__(self, n: int, device: torch.device, lib, first: bool):
        self.n = n
        pitch, count = ctypes.c_int64(), ctypes.c_int64()
        nat.check(lib.pb_level_geometry(n, ctypes.byref(pitch), ctypes.byref(count)), "level geometry")
        self.count = count.value

        def zeros(*lead):
            return torch.zeros(*lead, self.count, dtype=torch.float32, device=device)

        self.seven = first and n >= TMA_MIN_N
        self.invD, self.rhs, self.ea, self.eb, self.weights = (zeros() for _ in range(5))
        # level 0's residual is fused into its restriction; 27-point levels store theirs
        self.res = None if self.seven else zeros()
        self.D = zeros() if first else None
        self.coef = None if self.seven else zeros(14)

        self.packed = None

    def pack(self, device: torch.device, lib) -> None:
        """Per-colour packed FP16 couplings and 1/diagonal for the multi-block
        27-point kernels (mg27.cu); filled by Hierarchy32.setup."""
        hb, ib = ctypes.c_int64(), ctypes.c_int64()
        nat.check(lib.pb_packed27_size(self.n, ctypes.byref(hb), ctypes.byref(ib)), "packed27 size")
        h = lambda: torch.zeros(hb.value // 2, dtype=torch.float16, device=device)
        f = lambda: torch.zeros(ib.value // 4, dtype=torch.float32, device=device)
        self.packed = (h(), h(), f(), f())

    def packed_ptrs(self) -> tuple:
        return tuple(t.data_ptr() for t in self.packed)

    def tensors(self) -> list:
        return [t for t in (self.invD, self.rhs, self.res, self.ea, self.eb, self.weights, self.D, self.coef)
                if t is not None] + list(self.packed or ())


def galerkin_scratch_bytes(n: int, levels=None) -> int:
    """Bytes of the Galerkin products' scratch for a hierarchy of side n."""
    lib = nat.lib()
    sizes = level_sizes(n) if levels is None else [lv.n for lv in levels]
    first_seven = sizes[0] >= TMA_MIN_N
    fine27 = [m for i, m in enumerate(sizes[:-1]) if not (i == 0 and first_seven)]
    need = max([lib.pb_galerkin_workspace_size(m, 0) for m in fine27], default=0)
    one_plane = max([27 * 4 * 3 * ((m + 1) // 2) * (m + (m + 1) // 2) for m in fine27], default=0)
    return int(min(need, max(GALERKIN_SCRATCH, one_plane)))


class Hierarchy32:
    """FP32 preconditioner levels.  Level 0 is the reference's operator (its
    red-black sweeps staged by TMA); the levels below are Galerkin operators
    P_s^T A P_s / 8 built on the device by `setup` (mg27.cu), down to 3^3,
    which is solved exactly with its inverse."""

    def __init__(self, n: int, device: torch.device, z_chunk: int = 0, coarse_sweeps: int | None = None,
                 galerkin_ws: torch.Tensor | None = None, transient_coef: bool = False):
        """transient_coef: packed levels keep their 14 coefficient planes only
        during `setup` (allocated there, freed once packed), which saves their
        memory between solves at the cost of a fill per set-up."""
        self.status = torch.zeros(1, dtype=torch.int32, device=device)
        self.lib = nat.lib()
        self.device = device
        self.z_chunk = int(z_chunk)
        self.coarse_sweeps = COARSE_SWEEPS if coarse_sweeps is None else int(coarse_sweeps)
        self.sizes = level_sizes(n)
        self.levels = [Level32(m, device, self.lib, i == 0) for i, m in enumerate(self.sizes)]
        self.first_coarse = next(i for i, m in enumerate(self.sizes) if m <= COARSE_N)
        self.transient_coef = bool(transient_coef)
        for lv in self.levels[:self.first_coarse]:
            if not lv.seven:
                lv.pack(device, self.lib)
                if self.transient_coef:
                    lv.coef = None
        self.inverse = torch.zeros(27 * 27, dtype=torch.float64, device=device)  # of the 3^3 level, FP64
        # scratch of the separable Galerkin products (27-point fine levels), at most GALERKIN_SCRATCH bytes;
        # hierarchies set up one after another on one stream may share one (galerkin_ws)
        size = galerkin_scratch_bytes(n, self.levels)
        if galerkin_ws is not None and galerkin_ws.numel() * 4 >= size:
            self.galerkin_ws = galerkin_ws
        else:
            self.galerkin_ws = torch.empty((size + 3) // 4, dtype=torch.float32, device=device)
        # levels of side <= COARSE_N: one block from their image (couplings, 1/diagonal, weights, inverse)
        tail = self.levels[self.first_coarse:]
        k = len(tail)
        ptrs = lambda ts: (ctypes.c_void_p * k)(*[t.data_ptr() for t in ts])
        self._tail = (k, (ctypes.c_int64 * k)(*[lv.n for lv in tail]))
        image_bytes = self.lib.pb_coarse27_image_size(*self._tail)
        if image_bytes == 0:
            raise ValueError(f"no single-block image for levels {[lv.n for lv in tail]}")
        self.image = torch.zeros(image_bytes // 4, dtype=torch.float32, device=device)
        self._image_args = (*self._tail, ptrs([lv.coef for lv in tail]), ptrs([lv.invD for lv in tail]),
                            ptrs([lv.weights for lv in tail]), self.inverse.data_ptr(), self.image.data_ptr(),
                            image_bytes)
        self.pw = None

    @property
    def stream(self) -> int:
        return nat.stream_handle()

    def nbytes(self) -> int:
        return sum(t.numel() * t.element_size() for lv in self.levels for t in lv.tensors()) + \
            self.inverse.numel() * 8 + self.image.numel() * 4 + self.galerkin_ws.numel() * 4

    def setup(self, screen: torch.Tensor, point_weight: float) -> None:
        """Level 0 from the FP64 screen (D = (deg + pw*screen) h^-2, core.py:150-163),
        then each coarser level's Galerkin operator from the one above it, the
        packed forms, the 3^3 inverse and the coarse image: one library call
        (pb_hierarchy_setup_f32)."""
        self.pw = float(point_weight)
        for i, lv in enumerate(self.levels):  # zero-filled: the kernels write interior nodes only
            if lv.coef is None and not lv.seven:
                lv.coef = torch.zeros(14, lv.count, dtype=torch.float32, device=self.device)
        K, A = len(self.levels), 8
        arrays = (ctypes.c_void_p * (K * A))()
        for i, lv in enumerate(self.levels):
            row = [lv.D, lv.invD, lv.weights, lv.coef] + list(lv.packed or (None,) * 4)
            for k, t in enumerate(row):
                arrays[i * A + k] = None if t is None else t.data_ptr()
        sides = (ctypes.c_int64 * K)(*[lv.n for lv in self.levels])
        nat.check(self.lib.pb_hierarchy_setup_f32(K, sides, arrays, self.first_coarse, screen.data_ptr(), self.pw,
                                                  self.galerkin_ws.data_ptr(), self.galerkin_ws.numel() * 4,
                                                  self.inverse.data_ptr(), self.image.data_ptr(),
                                                  self.image.numel() * 4, self.stream), "hierarchy setup")
        if self.transient_coef:
            for lv in self.levels:
                if lv.packed is not None:
                    lv.coef = None  # freed once this stream's set-up has run (stream-ordered allocator)

    def _sweep(self, lv: Level32, src, dst, mode: int, coarse=None) -> None:
        """One red-black sweep dst <- S(src); mode 1 starts from zero, mode 2
        first adds the prolongated coarse correction to src in place."""
        L, s = self.lib, self.stream
        if mode == 2:
            nat.check(L.pb_prolong_fac_f32(coarse.data_ptr(), src.data_ptr(), lv.weights.data_ptr(), lv.n, s),
                      "prolong32")
            mode = 0
        if not lv.seven:
            nat.check(L.pb_relax27p_f32(None if mode == 1 else src.data_ptr(), dst.data_ptr(), lv.rhs.data_ptr(),
                                        *lv.packed_ptrs(), lv.n, s), "relax27p")
            return
        probe = PROBE if (PROBE is not None and lv is self.levels[0]) else None
        if probe is not None:
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
        nat.check(L.pb_sweep_tma_f32(None if src is None else src.data_ptr(), dst.data_ptr(), lv.rhs.data_ptr(),
                                     lv.invD.data_ptr(), lv.n, mode, self.z_chunk, self.status.data_ptr(), s),
                  "sweep")
        if probe is not None:
            end.record()
            probe.append((start, end, mode))

    def check_status(self) -> None:
        if int(self.status.item()):
            raise RuntimeError("FP32 cycle: a bounded wait on a TMA barrier gave up (status word set)")

    def v_cycle(self, level: int = 0, pre: int = 3, post: int = 3) -> torch.Tensor:
        """Correction for levels[level].rhs from a zero start; returns its tensor.
        (pre, post) sweeps on level 0, `coarse_sweeps` each way below it."""
        L, s = self.lib, self.stream
        if level > 0:
            pre = post = self.coarse_sweeps
        if level >= self.first_coarse:
            lv = self.levels[self.first_coarse]
            nat.check(L.pb_coarse27_cycle_f32(*self._tail, self.image.data_ptr(), lv.rhs.data_ptr(), lv.ea.data_ptr(),
                                              pre, post, self.coarse_sweeps, s), "coarse cycle")
            return lv.ea
        lv = self.levels[level]
        a, b = lv.ea, lv.eb
        self._sweep(lv, None, a, 1)  # pre-smoothing from zero
        src, dst = a, b
        for _ in range(pre - 1):
            self._sweep(lv, src, dst, 0)
            src, dst = dst, src
        nxt = self.levels[level + 1]
        if lv.seven and L.pb_tune_get(RESTRICT_VARIANT, lv.n) == 2:
            nat.check(L.pb_residual_restrict_tma_f32(src.data_ptr(), lv.rhs.data_ptr(), lv.D.data_ptr(),
                                                     lv.weights.data_ptr(), nxt.rhs.data_ptr(), lv.n,
                                                     self.status.data_ptr(), s), "residual_restrict_tma")
        elif lv.seven:
            nat.check(L.pb_residual_restrict_f32(src.data_ptr(), lv.rhs.data_ptr(), lv.D.data_ptr(),
                                                 lv.weights.data_ptr(), nxt.rhs.data_ptr(), lv.n, s),
                      "residual_restrict32")
        else:
            nat.check(L.pb_residual_restrict27p_f32(src.data_ptr(), lv.rhs.data_ptr(), *lv.packed_ptrs(),
                                                    lv.weights.data_ptr(), lv.n, lv.res.data_ptr(),
                                                    nxt.rhs.data_ptr(), s), "residual_restrict27p")
        coarse = self.v_cycle(level + 1, pre, post)
        self._sweep(lv, src, dst, 2, coarse)  # post-smoothing; the first adds the correction
        src, dst = dst, src
        for _ in range(post - 1):
            self._sweep(lv, src, dst, 0)
            src, dst = dst, src
        return src


_TUNED: set = set()


def apply_tuning(lib, n: int, device: torch.device) -> None:
    """Load the autotuner's cached launch parameters for side n on this GPU
    (tune.py) into the library's table, once per (device, side); skipped when
    MPR_B200_TUNE=0."""
    import os

    key = (device.index, n)
    if key in _TUNED or os.environ.get("MPR_B200_TUNE", "1") == "0":
        return
    from . import tune

    gpu = tune.gpu_name(device)
    for side in level_sizes(n):  # per-level parameters are cached under each level's side
        tune.apply(lib, gpu, side)
    _TUNED.add(key)


LEAN_MIN_N = 513  # engines of this side or larger run lean (RefinedEngine)
_WARM: set = set()  # (device, side) whose kernels have run once outside a capture


class RefinedEngine:
    """FCG(1) state for one grid side and point weight, reused across solves.

    Lean engines (side >= LEAN_MIN_N, where a grid is 1 GB and more) keep
    between solves only the hierarchy's operators: they solve on the caller's
    rhs and screen in place instead of copies, hand the final iterate out
    instead of a clone, release the FCG vectors after each solve, keep the
    packed levels' coefficient planes only during set-up, and re-capture the
    iteration graph per solve (its pointers change), with an eager prologue.

    Not thread-safe: one engine serves one stream at a time (the batch and
    serving paths create one engine per concurrent slot)."""

    def __init__(self, n: int, point_weight: float, device: torch.device, lean: bool | None = None):
        self.n = n
        self.pw = float(point_weight)
        self.device = device
        self.lib = nat.lib()
        self.lean = n >= LEAN_MIN_N if lean is None else bool(lean)
        apply_tuning(self.lib, n, device)  # before any launch shape is captured
        # Graph capture needs a stream other than the legacy default stream;
        # the engine's buffers are allocated on it and it runs every solve.
        self.stream = torch.cuda.Stream(device=device)
        with torch.cuda.stream(self.stream):
            self._allocate(n, device)

    def _allocate(self, n: int, device: torch.device) -> None:
        self.h = Hierarchy32(n, device, transient_coef=self.lean)
        if self.lean:
            self.screen = self.b = None  # bound per solve
            self.xs = self.ps = None  # allocated per solve
        else:
            self.screen, self.b = self._f64(), self._f64()
            self._vectors()
        self.scal = torch.zeros(8, dtype=torch.float64, device=device)
        self.ctrl = torch.zeros(2, dtype=torch.float64, device=device)
        self.flags = torch.zeros(4, dtype=torch.int32, device=device)
        self.history = torch.zeros(MAX_ITER, dtype=torch.float64, device=device)
        self.norm2 = torch.empty(1, dtype=torch.float64, device=device)
        self.bnorm = torch.empty(1, dtype=torch.float64, device=device)
        self.ws = nat.Workspace(device)
        self.ws_ptr, self.ws_size = self.ws.get(max(self.lib.pb_defect_workspace_size(n),
                                                    self.lib.pb_fcg_workspace_size(n)))
        self.norm_ws = nat.Workspace(device)
        self.norm_ws.get(1 << 16)
        self.graph = ctypes.c_void_p()
        self.exec = ctypes.c_void_p()
        self.setup_graph = None
        self.prologue_launches = 0
        self.body_launches = 0

    def _f64(self) -> torch.Tensor:
        return torch.empty((self.n,) * 3, dtype=torch.float64, device=self.device)

    def _vectors(self) -> None:
        n, device = self.n, self.device
        self.xs = (self._f64(), self._f64())  # iterate, alternating by iteration parity
        f32 = lambda: torch.empty((n, n, n), dtype=torch.float32, device=device)
        self.ps = (f32(), f32())  # search direction (stored in FP32), alternating by iteration parity

    def _drop_graph(self) -> None:
        if self.exec.value or self.graph.value:
            self.lib.pb_graph_destroy(self.exec, self.graph)
        self.exec, self.graph = ctypes.c_void_p(), ctypes.c_void_p()

    def __del__(self):
        try:
            if self.exec.value or self.graph.value:
                self.lib.pb_graph_destroy(self.exec, self.graph)
        except Exception:
            pass

    def nbytes(self) -> int:
        owned = [t for t in (self.screen, self.b) if t is not None and not self.lean]
        owned += list(self.xs or ()) + list(self.ps or ())
        return sum(t.numel() * t.element_size() for t in owned) + self.h.nbytes()

    def _iteration(self, handle: int) -> None:
        L, s = self.lib, nat.stream_handle()
        z = self.h.v_cycle(0, *level0_sweeps(self.n))
        r32 = self.h.levels[0].rhs
        p0, p1 = (t.data_ptr() for t in self.ps)
        x0, x1 = (t.data_ptr() for t in self.xs)
        nat.check(L.pb_fcg_direction_f64(z.data_ptr(), p0, p1, r32.data_ptr(), self.screen.data_ptr(), self.n,
                                         self.pw, self.scal.data_ptr(), self.flags.data_ptr(), self.ws_ptr,
                                         self.ws_size, s), "fcg direction")
        nat.check(L.pb_fcg_update_f64(z.data_ptr(), p0, p1, x0, x1, self.b.data_ptr(), self.screen.data_ptr(),
                                      r32.data_ptr(), self.n, self.pw, self.scal.data_ptr(), self.flags.data_ptr(),
                                      self.ws_ptr, self.ws_size, s), "fcg update")
        nat.check(L.pb_loop_condition(handle, self.scal.data_ptr(), self.ctrl.data_ptr(), self.flags.data_ptr(),
                                      MAX_ITER, self.history.data_ptr(), s), "loop condition")

    def _capture(self) -> None:
        """Capture one iteration as the body of a device-evaluated WHILE loop."""
        with GRAPH_CAPTURE_LOCK:
            self._capture_locked()

    def _capture_locked(self) -> None:
        L = self.lib
        s = nat.stream_handle()
        handle = ctypes.c_ulonglong()
        before = L.pb_launch_count()
        nat.check(L.pb_loop_capture_begin(s, ctypes.byref(self.graph), ctypes.byref(handle)), "loop capture")
        try:
            self._iteration(handle.value)
        except Exception:
            end = ctypes.c_void_p()
            L.pb_loop_capture_end(s, self.graph, ctypes.byref(end))
            self.graph = ctypes.c_void_p()
            raise
        nat.check(L.pb_loop_capture_end(s, self.graph, ctypes.byref(self.exec)), "loop capture end")
        self.body_launches = L.pb_launch_count() - before

    def _start(self) -> None:
        """x[0] = 0.5, r = b - A x (its FP32 copy for the first V-cycle), ||r||^2;
        iteration counter and first-step flag reset."""
        L, s = self.lib, nat.stream_handle()
        x0 = self.xs[0]
        nat.check(L.pb_fill_f64(x0.data_ptr(), x0.numel(), 0.5, s), "fill")  # core.py:270
        nat.check(L.pb_defect_f64(x0.data_ptr(), None, None, self.b.data_ptr(), self.screen.data_ptr(), self.n,
                                  self.pw, self.h.levels[0].rhs.data_ptr(), None, self.norm2.data_ptr(),
                                  self.ws_ptr, self.ws_size, s), "defect")
        self.flags.zero_()
        self.flags[0:1].fill_(1)  # a device fill, no host copy (capturable)

    def solve(self, rhs: torch.Tensor, screen: torch.Tensor, tol: float,
              max_cycles: int) -> tuple[torch.Tensor, SolveStats]:
        """Solve on the engine's stream, ordered after the caller's stream's
        work (rhs, screen) and before its later work (the returned field)."""
        caller = torch.cuda.current_stream(self.device)
        self.stream.wait_stream(caller)
        if self.lean:
            rhs.record_stream(self.stream)
            screen.record_stream(self.stream)
        with torch.cuda.stream(self.stream):
            x, stats = self._solve(rhs, screen, tol, max_cycles)
            if not self.lean:
                x = x.clone()
        caller.wait_stream(self.stream)
        if self.lean:
            x.record_stream(caller)  # allocated on the engine's stream, used on the caller's from here
        return x, stats

    def _prologue(self) -> None:
        """The per-solve work before the iterations, on the engine's own buffers:
        the levels' set-up (D, Galerkin products, packing, coarse image), x0 and
        its residual, ||b||."""
        self.h.setup(self.screen, self.pw)
        self._start()
        norm(self.b, self.norm_ws, self.bnorm)

    def _run_prologue(self) -> None:
        """The prologue as one graph launch: its ~45 launches touch the same
        pointers on every solve, so they are captured once per engine (after one
        eager run that sets kernel attributes and loads the modules) and
        replayed, which takes their host launch cost off small solves.  Lean
        engines run it eagerly (their pointers change per solve)."""
        if not SETUP_GRAPH or EAGER_LOOP or self.lean:
            self._prologue()
            return
        if self.setup_graph is None:
            self._prologue()
            g = torch.cuda.CUDAGraph()
            with GRAPH_CAPTURE_LOCK:
                before = self.lib.pb_launch_count()
                g.capture_begin(capture_error_mode="thread_local")  # other threads (serving lanes) stay free
                try:
                    self._prologue()
                finally:
                    g.capture_end()
            self.prologue_launches = self.lib.pb_launch_count() - before
            self.setup_graph = g
        self.setup_graph.replay()
        self.lib.pb_note_launches(self.prologue_launches)  # the replayed kernels, for the launch counter

    def _solve(self, rhs: torch.Tensor, screen: torch.Tensor, tol: float, max_cycles: int):
        L, s = self.lib, nat.stream_handle()
        stats = SolveStats()
        if self.lean:
            self.screen, self.b = screen, rhs
            self._vectors()
            self._drop_graph()
        else:
            self.screen.copy_(screen)
            self.b.copy_(rhs)
        try:
            x, stats = self._iterate(stats, tol, max_cycles)
        finally:
            if self.lean:  # nothing of this solve stays bound to the engine
                self.screen = self.b = None
                self.xs = self.ps = None
                self._drop_graph()
        return x, stats

    def _iterate(self, stats: SolveStats, tol: float, max_cycles: int):
        L, s = self.lib, nat.stream_handle()
        self._run_prologue()
        _sync.wait("solver prologue")
        both = torch.cat([self.norm2, self.bnorm]).cpu()
        stats.rhs_norm = float(both[1])
        r = math.sqrt(max(float(both[0]), 0.0))
        stats.history.append(r)
        stats.residual_norm = r
        target = tol * stats.rhs_norm
        it = 0
        if r > target and max_cycles > 0:
            self.ctrl.copy_(torch.tensor([target * target, float(max_cycles)], dtype=torch.float64))
            if EAGER_LOOP:
                while True:
                    self._iteration(0)
                    done = int(self.flags[1].item())
                    r2 = float(self.scal[4].item())
                    if not (r2 > target * target and done < min(MAX_ITER, max_cycles)):
                        break
            else:
                if not self.exec.value:
                    warm_key = (self.device.index, self.n)
                    if warm_key not in _WARM:
                        # one eager iteration first sets kernel attributes and loads the
                        # kernels' modules outside any capture (once per process and
                        # side); its effect is discarded by restarting below
                        self._iteration(0)
                        self._start()
                        _WARM.add(warm_key)
                    self._capture()
                nat.check(L.pb_graph_launch(self.exec, s), "graph launch")
            _sync.wait("solver iterations")
            tail = torch.cat([self.flags[1:2].to(torch.float64), self.scal[4:5]]).cpu()
            it = int(tail[0])
            if not EAGER_LOOP:
                L.pb_note_launches(it * self.body_launches)
            stats.cycles = it
            stats.history.extend(math.sqrt(max(v, 0.0)) for v in self.history[:it].cpu().tolist())
            # pass 2 computes the true residual b - A x of every iterate
            stats.residual_norm = math.sqrt(max(float(tail[1]), 0.0))
        self.h.check_status()
        return self.xs[it & 1], stats


_ENGINES: "collections.OrderedDict[tuple, RefinedEngine]" = collections.OrderedDict()
_ENGINE_LOCK = threading.Lock()
ENGINE_CACHE_SIZE = 32
ENGINE_CACHE_FRACTION = 0.3  # of the device's memory kept in cached engines at most
_LOCAL = threading.local()


def current_slot() -> int:
    """Engine slot of the calling thread (serving lanes set their own)."""
    return getattr(_LOCAL, "slot", 0)


def set_slot(slot: int) -> None:
    _LOCAL.slot = int(slot)


def _cached_bytes() -> int:
    return sum(e.nbytes() for e in _ENGINES.values())


def engine_for(n: int, point_weight: float, device: torch.device, slot: int | None = None) -> RefinedEngine:
    """A cached engine for (device, n, point_weight, slot); least recently used
    engines are dropped beyond ENGINE_CACHE_SIZE entries or ENGINE_CACHE_FRACTION
    of device memory (and all of them when an allocation runs out of memory).
    The caller owns the returned engine until its solve returns: one slot per
    concurrent thread."""
    slot = current_slot() if slot is None else slot
    key = (device.index, n, float(point_weight), slot)
    with _ENGINE_LOCK:
        eng = _ENGINES.pop(key, None)
        if eng is None:
            budget = ENGINE_CACHE_FRACTION * torch.cuda.get_device_properties(device).total_memory
            estimate = 96 * n**3
            while _ENGINES and (len(_ENGINES) >= ENGINE_CACHE_SIZE or _cached_bytes() + estimate > budget):
                _ENGINES.popitem(last=False)
            try:
                eng = RefinedEngine(n, point_weight, device)
            except torch.cuda.OutOfMemoryError:
                _ENGINES.clear()
                torch.cuda.empty_cache()
                eng = RefinedEngine(n, point_weight, device)
        _ENGINES[key] = eng
        return eng


def clear_engines() -> None:
    """Drop the cached engines and the batched solver's pooled cloud states."""
    _ENGINES.clear()
    from . import batch

    batch.clear_pool()


def solve_refined(rhs: torch.Tensor, screen: torch.Tensor, point_weight: float, workspace: nat.Workspace, *,
                  tol: float = 1e-8, max_cycles: int = 200, has_points: bool = True,
                  method: str = "fcg", slot: int | None = None) -> tuple[torch.Tensor, SolveStats]:
    """FP64-accurate solve with FP32 V-cycles; stats.cycles counts V-cycles.

    method="fcg": FCG(1) on a cached RefinedEngine (graph-driven loop).
    method="defect": plain defect correction, x += V(r), eager launches."""
    if method not in ("fcg", "defect"):
        raise ValueError("method must be 'fcg' or 'defect'")
    L = nat.lib()
    s = nat.stream_handle()
    n = rhs.shape[0]
    device = rhs.device
    if not has_points:
        x = torch.empty_like(rhs)
        nat.check(L.pb_fill_f64(x.data_ptr(), x.numel(), 0.0, s), "fill")
        stats = SolveStats()
        stats.residual_norm = 0.0
        stats.rhs_norm = 0.0
        return x, stats
    if method == "fcg":
        return engine_for(n, point_weight, device, slot).solve(rhs, screen, tol, max_cycles)
    stats = SolveStats()
    x = torch.empty_like(rhs)
    nat.check(L.pb_fill_f64(x.data_ptr(), x.numel(), 0.5, s), "fill")
    h = Hierarchy32(n, device)
    h.setup(screen, point_weight)
    bnorm = norm(rhs, workspace, torch.empty(1, dtype=torch.float64, device=device))
    norm2 = torch.empty(1, dtype=torch.float64, device=device)
    ws = nat.Workspace(device)
    ptr, size = ws.get(L.pb_defect_workspace_size(n))
    r32 = h.levels[0].rhs
    nat.check(L.pb_defect_f64(x.data_ptr(), None, None, rhs.data_ptr(), screen.data_ptr(), n, h.pw, r32.data_ptr(),
                              None, norm2.data_ptr(), ptr, size, s), "defect")
    stats.rhs_norm = float(bnorm.item())
    target = tol * stats.rhs_norm
    r = math.sqrt(float(norm2.item()))
    stats.history.append(r)
    x_next = torch.empty_like(rhs)
    while r > target and stats.cycles < max_cycles:
        e = h.v_cycle(0)
        nat.check(L.pb_defect_f64(x.data_ptr(), e.data_ptr(), x_next.data_ptr(), rhs.data_ptr(), screen.data_ptr(),
                                  n, h.pw, r32.data_ptr(), None, norm2.data_ptr(), ptr, size, s), "defect")
        x, x_next = x_next, x
        stats.cycles += 1
        r = math.sqrt(float(norm2.item()))
        stats.history.append(r)
    h.check_status()
    stats.residual_norm = r
    return x, stats
