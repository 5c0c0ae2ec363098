"""Many clouds in one solve: grouped launches across a batch of uneven clouds.

The reference solves one cloud at a time and, inside it, one level at a time
(python/mojo_poissonrecon/core.py:141-193, driven per cycle at :270-287).
`BatchSolver` runs the refined solver (FP64 FCG(1) preconditioned by the FP32
V-cycle, as solver32.RefinedEngine) for K clouds of any depth >= 5 together:
every step of the V-cycle and of FCG is ONE launch over the grids of all
clouds at that step (pb_batch_launch over a descriptor table, batch.cuh):

    level 0 (every cloud):       sweep from zero, residual + restriction
    level l = 1, 2, ... (every cloud that has a packed level l):
                                 sweep from zero, residual, restriction
    levels of side <= 9:         one block per cloud (the shared-memory cycle)
    back up, level l ... 1:      prolongation, sweep
    level 0:                     prolongation, two sweeps
    FCG pass 1, its per-cloud sums, pass 2, its per-cloud sums, loop condition

One batch iteration is captured once as the body of a CUDA graph WHILE node;
every cloud keeps its own iteration count, buffer parity and scalars on the
device, and a cloud that reaches its tolerance turns inactive: its blocks
return at once in every later launch, so its iterate stays as it converged
while the others iterate on.  The solve is one graph launch for the batch.

`reconstruct_many` is the batched `reconstruct`: one host-to-device copy for
all clouds, their preparation, splats, the batched solve, iso-values and
extraction queued with one host synchronisation for the kept-point counts and
one for the mesh sizes, and the meshes copied back together.  Clouds too small
for the batched solver (depth < 5) and the FP64 precision go through the
single-cloud path.  Results are bit-identical to `core.reconstruct` of each
cloud alone: the same kernels run on the same data in the same order per
cloud, and every kernel is deterministic.
"""

from __future__ import annotations

import collections
import concurrent.futures
import ctypes
import math
import threading

import numpy as np
import torch

from . import _native as nat
from . import _sync, _trace, core
from .solver import SolveStats, norm
from .solver32 import (GRAPH_CAPTURE_LOCK, MAX_ITER, TMA_MIN_N, Hierarchy32, apply_tuning, galerkin_scratch_bytes,
                       level0_sweeps)

# descriptor kinds (include/poisson_b200.h)
SWEEP, SWEEP_ZERO, PROLONG32, RESIDUAL_RESTRICT32 = 0, 1, 2, 3
RELAX27P, RELAX27P_ZERO, RESIDUAL27P, RESTRICT27, COARSE27 = 4, 5, 6, 7, 8
FCG_DIRECTION, FCG_DIRECTION_FINISH, FCG_UPDATE, FCG_SUM = 9, 10, 11, 12
PTRS = 12
MIN_DEPTH = 5  # level 0 of side >= 33 (the TMA sweep)


def _bits(value: float) -> int:
    return int(np.array([value], dtype=np.float64).view(np.int64)[0])


class _Launch:
    """One grouped launch: its descriptors on the device and its block count."""

    def __init__(self, lib, kind: int, grids: list, device: torch.device, z_chunk: int = 0, first_side: int = 0):
        self.kind = kind
        self.count = len(grids)
        self.first_side = first_side
        clouds = np.array([g[0] for g in grids], dtype=np.int64)
        sides = np.array([g[1] for g in grids], dtype=np.int64)
        ptrs = np.zeros((self.count, PTRS), dtype=np.uint64)
        aux = np.zeros((self.count, 4), dtype=np.int64)
        for i, g in enumerate(grids):
            for k, p in enumerate(g[2]):
                ptrs[i, k] = 0 if p is None else int(p)
            for k, a in enumerate(g[3] if len(g) > 3 else ()):
                aux[i, k] = int(a)
        nbytes = int(lib.pb_batch_desc_bytes(self.count))
        raw = np.zeros(nbytes + 64, dtype=np.uint8)
        off = (-raw.ctypes.data) % 64
        host = raw[off:off + nbytes]
        blocks = ctypes.c_int64()
        nat.check(lib.pb_batch_describe(kind, self.count, clouds.ctypes.data, sides.ctypes.data, ptrs.ctypes.data,
                                        aux.ctypes.data, z_chunk, host.ctypes.data, nbytes, ctypes.byref(blocks)),
                  f"batch describe (kind {kind})")
        self.blocks = int(blocks.value)
        self.desc = torch.from_numpy(host.copy()).to(device)  # torch allocations are 256-byte aligned

    def run(self, lib, flags: torch.Tensor, stream: int) -> None:
        nat.check(lib.pb_batch_launch(self.kind, self.desc.data_ptr(), self.count, self.blocks, flags.data_ptr(),
                                      self.first_side, stream), f"batch launch (kind {self.kind})")


class _Cloud:
    """One cloud's solver state: its FP32 hierarchy and FP64/FP32 FCG vectors.
    Every solve overwrites all of it (the hierarchy's ghosts stay zero), so a
    cloud state of the same side can serve any later batch."""

    def __init__(self, n: int, device: torch.device, galerkin_ws: torch.Tensor):
        self.n = n
        self.device = device
        self.h = Hierarchy32(n, device, galerkin_ws=galerkin_ws)
        f64 = lambda: torch.empty((n, n, n), dtype=torch.float64, device=device)
        f32 = lambda: torch.empty((n, n, n), dtype=torch.float32, device=device)
        self.xs = (f64(), f64())
        self.ps = (f32(), f32())
        self.nbytes = self.h.nbytes() - self.h.galerkin_ws.numel() * 4 + 12 * n ** 3 * 2


# Cloud states of finished batches, per (device, side), reused by later ones
# (allocating a batch's hierarchies costs about 20 tensors per level per cloud);
# at most POOL_FRACTION of the device's memory, least recently returned first out.
POOL_FRACTION = 0.25
_POOL: "collections.OrderedDict[int, _Cloud]" = collections.OrderedDict()
_POOL_LOCK = threading.Lock()
_STREAMS = threading.local()


def _stream(device: torch.device) -> torch.cuda.Stream:
    """This thread's stream for batched solves on `device`: one for the life of
    the thread, so the caching allocator reuses the memory of earlier batches."""
    table = getattr(_STREAMS, "by_device", None)
    if table is None:
        table = _STREAMS.by_device = {}
    if device.index not in table:
        table[device.index] = torch.cuda.Stream(device=device)
    return table[device.index]


# The per-cloud prologue (hierarchy set-up, x0 and its residual, ||b||) is ~50 small
# launches per cloud; PROLOGUE_LANES host threads issue it on as many streams, each
# with its own scratch, so the launches of different clouds overlap on the host and
# on the device.  Only where one Galerkin scratch is at most PROLOGUE_SCRATCH bytes.
PROLOGUE_LANES = 4
PROLOGUE_SCRATCH = 256 << 20
_PROLOGUE_POOL = concurrent.futures.ThreadPoolExecutor(max_workers=PROLOGUE_LANES,
                                                       thread_name_prefix="mpr-prologue")


def _lane_streams(device: torch.device, count: int) -> list:
    """This thread's prologue streams on `device` (kept for the life of the thread)."""
    table = getattr(_STREAMS, "lanes", None)
    if table is None:
        table = _STREAMS.lanes = {}
    lanes = table.setdefault(device.index, [])
    while len(lanes) < count:
        lanes.append(torch.cuda.Stream(device=device))
    return lanes[:count]


class _PrologueLane:
    """One prologue lane's stream and scratch (Galerkin, defect, norm)."""

    def __init__(self, lib, device: torch.device, stream: torch.cuda.Stream, galerkin_ws: torch.Tensor,
                 defect_bytes: int):
        self.stream = stream
        self.galerkin_ws = galerkin_ws
        self.defect_ws = nat.Workspace(device)
        self.defect_ptr, self.defect_size = self.defect_ws.get(defect_bytes)
        self.norm_ws = nat.Workspace(device)
        self.norm_ws.get(1 << 16)


def _take_cloud(n: int, device: torch.device, galerkin_ws: torch.Tensor) -> _Cloud:
    with _POOL_LOCK:
        for key, c in _POOL.items():
            if c.n == n and c.device == device:
                del _POOL[key]
                c.h.galerkin_ws = galerkin_ws  # the batch's own scratch: batches on other lanes run concurrently
                return c
    return _Cloud(n, device, galerkin_ws)


def _return_clouds(clouds) -> None:
    if not clouds:
        return
    device = clouds[0].device
    cap = POOL_FRACTION * torch.cuda.get_device_properties(device).total_memory
    with _POOL_LOCK:
        for c in clouds:
            c.h.galerkin_ws = None  # not kept alive by the pool
            _POOL[id(c)] = c
        total = sum(c.nbytes for c in _POOL.values())
        while _POOL and total > cap:
            _, c = _POOL.popitem(last=False)
            total -= c.nbytes


def clear_pool() -> None:
    """Drop every pooled cloud state (their memory returns to torch's cache)."""
    with _POOL_LOCK:
        _POOL.clear()


class BatchSolver:
    """FP64 FCG(1) with FP32 V-cycles for K clouds at once (module docstring).

    sides: grid side per cloud (2^d + 1, d >= 5).  Buffers stay allocated for
    repeated solves of clouds with the same sides (the right-hand sides and
    screens are bound per solve, so the captured graph is rebuilt per solve)."""

    def __init__(self, sides, device: torch.device | None = None):
        self.lib = nat.lib()
        self.device = nat.require_cuda() if device is None else device
        self.sides = [int(n) for n in sides]
        if not self.sides:
            raise ValueError("a batch needs at least one cloud")
        for n in self.sides:
            if n < TMA_MIN_N or (n - 1) & (n - 2):
                raise ValueError(f"batched solves need sides 2^d + 1 >= {TMA_MIN_N} (got {n})")
        for n in set(self.sides):
            apply_tuning(self.lib, n, self.device)
        self.stream = _stream(self.device)
        K = len(self.sides)
        with torch.cuda.stream(self.stream):
            scratch = max(galerkin_scratch_bytes(n) for n in set(self.sides))
            self.galerkin_ws = torch.empty((scratch + 3) // 4, dtype=torch.float32, device=self.device)
            self.clouds = [_take_cloud(n, self.device, self.galerkin_ws) for n in self.sides]
            self.flags = torch.zeros((K, 4), dtype=torch.int32, device=self.device)
            self.scal = torch.zeros((K, 8), dtype=torch.float64, device=self.device)
            self.ctrl = torch.zeros((K, 2), dtype=torch.float64, device=self.device)
            self.history = torch.zeros((K, MAX_ITER), dtype=torch.float64, device=self.device)
            self.norm2 = torch.zeros(K, dtype=torch.float64, device=self.device)
            self.bnorm = torch.zeros(K, dtype=torch.float64, device=self.device)
            self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
            parts = [int(self.lib.pb_batch_fcg_partials(n)) for n in self.sides]
            self.part_offsets = np.concatenate([[0], np.cumsum(parts)]).astype(np.int64)
            self.partials = torch.zeros(int(self.part_offsets[-1]), dtype=torch.float64, device=self.device)
            defect = max(int(self.lib.pb_defect_workspace_size(n)) for n in set(self.sides))
            lanes = min(PROLOGUE_LANES, K) if scratch <= PROLOGUE_SCRATCH else 1
            streams = [self.stream] if lanes == 1 else _lane_streams(self.device, lanes)
            self.lanes = [_PrologueLane(self.lib, self.device, streams[0], self.galerkin_ws, defect)]
            for j in range(1, lanes):
                ws = torch.empty_like(self.galerkin_ws)
                self.lanes.append(_PrologueLane(self.lib, self.device, streams[j], ws, defect))
            for k, c in enumerate(self.clouds):  # cloud k's set-up runs on lane k % lanes
                c.h.galerkin_ws = self.lanes[k % lanes].galerkin_ws
        self.graph = ctypes.c_void_p()
        self.exec = ctypes.c_void_p()
        self.body_launches = 0
        self.launches = []

    def release(self) -> None:
        """Hand the cloud states to the pool for later batches (after the solve's
        results have been read: the caller's stream has waited for this one)."""
        self.stream.synchronize()
        clouds, self.clouds = self.clouds, []
        _return_clouds(clouds)

    def __del__(self):
        try:
            if self.exec.value or self.graph.value:
                self.lib.pb_graph_destroy(self.exec, self.graph)
        except Exception:
            pass

    # -- the launch schedule -------------------------------------------------------
    def _plan(self, rhs, screen, pws) -> list:
        """The grouped launches of one iteration, in order, for the bound rhs/screen."""
        dev, lib = self.device, self.lib
        st = self.status.data_ptr()
        plan = []

        def add(kind, grids, **kw):
            if grids:
                plan.append(_Launch(lib, kind, grids, dev, **kw))

        cl = self.clouds
        K = len(cl)
        l0 = [c.h.levels[0] for c in cl]
        # level-0 sweeps: whole planes per block when the launch's tiles fill the
        # GPU several times over, else z chunks that give about two waves
        tiles = sum(max(1, (c.n - 1) // 64) * max(1, (c.n - 1) // 16) for c in cl)
        slots = 2 * 148
        chunks = 1 if tiles >= 4 * slots else -(-2 * slots // tiles)
        z_chunk = 0 if chunks == 1 else max(16, -(-max(self.sides) // chunks))
        # level 0 down: V(pre, post) with pre = level0_sweeps(n)[0] (1: the sweep from zero)
        for c in cl:
            if level0_sweeps(c.n) != (1, 2):
                raise ValueError("the batched cycle implements V(1, 2) on level 0")
        add(SWEEP_ZERO, [(k, cl[k].n, (None, l0[k].ea.data_ptr(), l0[k].rhs.data_ptr(), l0[k].invD.data_ptr(), st))
                         for k in range(K)], z_chunk=z_chunk)
        add(RESIDUAL_RESTRICT32, [(k, cl[k].n, (l0[k].ea.data_ptr(), l0[k].rhs.data_ptr(), l0[k].D.data_ptr(),
                                                l0[k].weights.data_ptr(), cl[k].h.levels[1].rhs.data_ptr()))
                                  for k in range(K)])
        depth_max = max(c.h.first_coarse for c in cl)
        # packed levels down (coarse_sweeps = 1 each way)
        for lvl in range(1, depth_max):
            idx = [k for k in range(K) if lvl < cl[k].h.first_coarse]
            lv = {k: cl[k].h.levels[lvl] for k in idx}
            nx = {k: cl[k].h.levels[lvl + 1] for k in idx}
            for k in idx:
                if cl[k].h.coarse_sweeps != 1:
                    raise ValueError("the batched cycle implements one sweep each way below level 0")
            add(RELAX27P_ZERO, [(k, lv[k].n, (None, lv[k].ea.data_ptr(), lv[k].rhs.data_ptr(), *lv[k].packed_ptrs()))
                                for k in idx])
            add(RESIDUAL27P, [(k, lv[k].n, (lv[k].ea.data_ptr(), lv[k].rhs.data_ptr(), *lv[k].packed_ptrs(),
                                            lv[k].weights.data_ptr(), lv[k].res.data_ptr())) for k in idx])
            add(RESTRICT27, [(k, lv[k].n, (lv[k].res.data_ptr(), nx[k].rhs.data_ptr())) for k in idx])
        # levels of side <= 9: one block per cloud
        tails = [c.h.levels[c.h.first_coarse] for c in cl]
        sides = {t.n for t in tails}
        for side in sorted(sides):
            idx = [k for k in range(K) if tails[k].n == side]
            add(COARSE27, [(k, side, (cl[k].h.image.data_ptr(), tails[k].rhs.data_ptr(), tails[k].ea.data_ptr()),
                            (1, 1, 1)) for k in idx], first_side=side)

        def result(k, lvl):  # the correction level lvl of cloud k returns upwards
            h = cl[k].h
            return h.levels[lvl].ea if lvl >= h.first_coarse else h.levels[lvl].eb

        for lvl in range(depth_max - 1, 0, -1):
            idx = [k for k in range(K) if lvl < cl[k].h.first_coarse]
            lv = {k: cl[k].h.levels[lvl] for k in idx}
            add(PROLONG32, [(k, lv[k].n, (result(k, lvl + 1).data_ptr(), lv[k].ea.data_ptr(),
                                          lv[k].weights.data_ptr())) for k in idx])
            add(RELAX27P, [(k, lv[k].n, (lv[k].ea.data_ptr(), lv[k].eb.data_ptr(), lv[k].rhs.data_ptr(),
                                         *lv[k].packed_ptrs())) for k in idx])
        # level 0 up: prolongation into ea, sweeps ea -> eb -> ea
        add(PROLONG32, [(k, cl[k].n, (result(k, 1).data_ptr(), l0[k].ea.data_ptr(), l0[k].weights.data_ptr()))
                        for k in range(K)])
        add(SWEEP, [(k, cl[k].n, (l0[k].ea.data_ptr(), l0[k].eb.data_ptr(), l0[k].rhs.data_ptr(),
                                  l0[k].invD.data_ptr(), st)) for k in range(K)], z_chunk=z_chunk)
        add(SWEEP, [(k, cl[k].n, (l0[k].eb.data_ptr(), l0[k].ea.data_ptr(), l0[k].rhs.data_ptr(),
                                  l0[k].invD.data_ptr(), st)) for k in range(K)], z_chunk=z_chunk)
        # FCG(1): z = l0.ea, r32 = l0.rhs
        part = [self.partials[int(self.part_offsets[k]):].data_ptr() for k in range(K)]
        scal = [self.scal[k].data_ptr() for k in range(K)]
        add(FCG_DIRECTION, [(k, cl[k].n, (l0[k].ea.data_ptr(), cl[k].ps[0].data_ptr(), cl[k].ps[1].data_ptr(),
                                          l0[k].rhs.data_ptr(), screen[k].data_ptr(), part[k]), (_bits(pws[k]),))
                            for k in range(K)])
        add(FCG_DIRECTION_FINISH, [(k, cl[k].n, (part[k], scal[k]), (int(lib.pb_batch_fcg_blocks(cl[k].n, 0)),))
                                   for k in range(K)])
        add(FCG_UPDATE, [(k, cl[k].n, (l0[k].ea.data_ptr(), cl[k].ps[0].data_ptr(), cl[k].ps[1].data_ptr(),
                                       cl[k].xs[0].data_ptr(), cl[k].xs[1].data_ptr(), rhs[k].data_ptr(),
                                       screen[k].data_ptr(), l0[k].rhs.data_ptr(), scal[k], part[k]),
                          (_bits(pws[k]),)) for k in range(K)])
        add(FCG_SUM, [(k, cl[k].n, (part[k], self.scal[k, 4:].data_ptr()),
                       (int(lib.pb_batch_fcg_blocks(cl[k].n, 1)),)) for k in range(K)])
        return plan

    def _iteration(self, handle: int) -> None:
        s = nat.stream_handle()
        for launch in self.launches:
            launch.run(self.lib, self.flags, s)
        nat.check(self.lib.pb_batch_loop_condition(handle, self.scal.data_ptr(), self.ctrl.data_ptr(),
                                                   self.flags.data_ptr(), len(self.clouds), MAX_ITER,
                                                   self.history.data_ptr(), s), "batch loop condition")

    def _capture(self) -> None:
        with GRAPH_CAPTURE_LOCK:
            self._capture_locked()

    def _capture_locked(self) -> None:
        L = self.lib
        s = nat.stream_handle()
        handle = ctypes.c_ulonglong()
        if self.exec.value or self.graph.value:
            L.pb_graph_destroy(self.exec, self.graph)
            self.exec, self.graph = ctypes.c_void_p(), ctypes.c_void_p()
        before = L.pb_launch_count()
        nat.check(L.pb_loop_capture_begin(s, ctypes.byref(self.graph), ctypes.byref(handle)), "batch loop capture")
        try:
            self._iteration(handle.value)
        except Exception:
            end = ctypes.c_void_p()
            L.pb_loop_capture_end(s, self.graph, ctypes.byref(end))
            self.graph = ctypes.c_void_p()
            raise
        nat.check(L.pb_loop_capture_end(s, self.graph, ctypes.byref(self.exec)), "batch loop capture end")
        self.body_launches = L.pb_launch_count() - before

    # -- solve -----------------------------------------------------------------------
    def solve(self, rhs: list, screen: list, point_weights, tol: float = 1e-8, max_cycles: int = 200,
              phases=None):
        """Solve A_k x_k = b_k for every cloud to ||b_k - A_k x_k|| <= tol ||b_k||.

        rhs, screen: per cloud dense FP64 (n, n, n) CUDA tensors (read in place;
        they must stay alive and unchanged until this returns).  Returns the
        list of fields (new tensors) and the list of SolveStats."""
        K = len(self.clouds)
        if len(rhs) != K or len(screen) != K:
            raise ValueError("one rhs and one screen per cloud")
        pws = [float(point_weights)] * K if np.isscalar(point_weights) else [float(p) for p in point_weights]
        for k in range(K):
            n = self.sides[k]
            for t in (rhs[k], screen[k]):
                if tuple(t.shape) != (n, n, n) or t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous():
                    raise ValueError(f"cloud {k}: rhs and screen must be contiguous CUDA float64 ({n},)*3 tensors")
        caller = torch.cuda.current_stream(self.device)
        self.stream.wait_stream(caller)
        for t in list(rhs) + list(screen):
            t.record_stream(self.stream)
        with torch.cuda.stream(self.stream):
            xs, stats = self._solve(rhs, screen, pws, tol, max_cycles, phases)
        caller.wait_stream(self.stream)
        return [x.clone() for x in xs], stats  # on the caller's stream

    def _prologue_lane(self, j: int, start: torch.cuda.Event, rhs, screen, pws) -> None:
        """Lane j's clouds (k = j, j + lanes, ...): levels' set-up, x0 = 0.5 and its
        residual, ||b||; on the lane's stream, after `start`."""
        L, lane = self.lib, self.lanes[j]
        if lane.stream is not self.stream:
            lane.stream.wait_event(start)
        with torch.cuda.device(self.device), torch.cuda.stream(lane.stream):  # a worker thread's device too
            s = nat.stream_handle()
            for k in range(j, len(self.clouds), len(self.lanes)):
                c = self.clouds[k]
                c.h.setup(screen[k], pws[k])
                x0 = c.xs[0]
                nat.check(L.pb_fill_f64(x0.data_ptr(), x0.numel(), 0.5, s), "fill")  # core.py:270
                nat.check(L.pb_defect_f64(x0.data_ptr(), None, None, rhs[k].data_ptr(), screen[k].data_ptr(),
                                          c.n, pws[k], c.h.levels[0].rhs.data_ptr(), None,
                                          self.norm2[k:k + 1].data_ptr(), lane.defect_ptr, lane.defect_size, s),
                          "defect")
                norm(rhs[k], lane.norm_ws, self.bnorm[k:k + 1])

    def _prologue(self, rhs, screen, pws) -> None:
        """Every cloud's prologue, spread over the prologue lanes (host threads
        and streams), then joined back into the solver's stream."""
        if len(self.lanes) == 1:
            self._prologue_lane(0, None, rhs, screen, pws)
            return
        start = torch.cuda.Event()
        start.record(self.stream)
        jobs = [_PROLOGUE_POOL.submit(self._prologue_lane, j, start, rhs, screen, pws)
                for j in range(len(self.lanes))]
        errors = [f.exception() for f in jobs]
        for lane in self.lanes:  # join every lane, also after an error
            self.stream.wait_stream(lane.stream)
        for e in errors:
            if e is not None:
                raise e

    def _solve(self, rhs, screen, pws, tol, max_cycles, phases=None):
        mark = phases.mark if phases is not None else (lambda name: None)
        L, s = self.lib, nat.stream_handle()
        K = len(self.clouds)
        self._prologue(rhs, screen, pws)
        # per-cloud control on the device: target ||r||^2, cap; active while above target
        target = tol * self.bnorm  # ||b|| (not squared), as the single-cloud engine forms it
        target2 = target * target
        self.ctrl[:, 0] = target2
        self.ctrl[:, 1] = float(max_cycles)
        self.flags.zero_()
        self.flags[:, 0] = 1
        self.flags[:, 2] = ((self.norm2 > target2) & (max_cycles > 0)).to(torch.int32)
        self.scal.zero_()
        mark("solver prologue")
        self.launches = self._plan(rhs, screen, pws)
        self._capture()
        mark("solver plan and capture")
        nat.check(L.pb_graph_launch(self.exec, s), "batch graph launch")
        _sync.wait("batched solver iterations")
        host = torch.cat([self.flags[:, 1].to(torch.float64), self.scal[:, 4], self.norm2, self.bnorm,
                          self.status.to(torch.float64)]).cpu().numpy()
        its = host[:K].astype(np.int64)
        if host[4 * K] != 0:
            raise RuntimeError("batched FP32 sweep: a bounded wait on a TMA barrier gave up (status word set)")
        # iterations run = the largest per-cloud count; each launched the body's kernels
        L.pb_note_launches(int(its.max(initial=0)) * self.body_launches)
        hist = self.history[:, :max(1, int(its.max(initial=0)))].cpu().numpy()
        fields, stats = [], []
        for k, c in enumerate(self.clouds):
            st = SolveStats()
            st.rhs_norm = float(host[3 * K + k])
            r0 = math.sqrt(max(host[2 * K + k], 0.0))
            st.history.append(r0)
            it = int(its[k])
            st.cycles = it
            st.history.extend(math.sqrt(max(v, 0.0)) for v in hist[k, :it])
            st.residual_norm = math.sqrt(max(host[K + k], 0.0)) if it else r0
            fields.append(c.xs[it & 1])
            stats.append(st)
        return fields, stats


def _footprint(depth: int, points: int) -> int:
    from .serve import footprint_bytes

    return footprint_bytes(depth, points)


class _Phases:
    """Host wall time per phase of reconstruct_many (profile=dict), each phase
    closed by a device synchronisation; a no-op without a dict."""

    def __init__(self, sink: dict | None):
        import time

        self.sink, self.clock = sink, time.perf_counter
        self.t = self.clock() if sink is not None else 0.0

    def mark(self, name: str) -> None:
        if self.sink is None:
            return
        torch.cuda.synchronize()
        now = self.clock()
        self.sink[name] = self.sink.get(name, 0.0) + (now - self.t)
        self.t = now


def reconstruct_many(clouds, *, depth: int = 6, point_weight: float = 4.0, confidence: bool = False,
                     scale: float = 1.1, samples_per_node: float = 1.5, tol: float = 1e-8, max_cycles: int = 200,
                     budget_bytes: int | None = None, device_out: bool = False, profile: dict | None = None) -> list:
    """Reconstruct many clouds with batched solves (module docstring).

    clouds: (points, normals) or (points, normals, depth) tuples (NumPy or
    torch).  Precision is "fp32_refined" to relative residual `tol`.  Clouds
    run in waves whose estimated device footprint fits `budget_bytes`
    (default: 60 % of the device's free memory).  Returns core.Mesh objects in
    input order, bit-identical to core.reconstruct of each cloud alone.
    profile: a dict that receives the host seconds of each phase (with a
    device synchronisation after each, so only for measurements)."""
    phases = _Phases(profile)
    dev = nat.require_cuda()
    items = []
    for k, cloud in enumerate(clouds):
        p, nrm = cloud[0], cloud[1]
        d = int(cloud[2]) if len(cloud) > 2 else int(depth)
        items.append((k, core._points(p), core._points(nrm), d))
    for _, p, nrm, d in items:
        if tuple(p.shape) != tuple(nrm.shape):
            raise ValueError("points and normals must have the same shape")
        if not 2 <= d <= core.MAX_DEPTH:
            raise ValueError(f"depth must be between 2 and {core.MAX_DEPTH}")
    if budget_bytes is None:
        free, _ = torch.cuda.mem_get_info(dev)
        budget_bytes = int(0.6 * free)
    out: list = [None] * len(items)
    small = [it for it in items if it[3] < MIN_DEPTH]
    for k, p, nrm, d in small:  # below the batched solver's smallest level 0
        out[k] = core.reconstruct(p, nrm, depth=d, point_weight=point_weight, confidence=confidence, scale=scale,
                                  samples_per_node=samples_per_node, precision="fp32_refined", tol=tol,
                                  max_cycles=max_cycles, device_out=device_out)
    phases.mark("validate and small clouds")
    big = sorted((it for it in items if it[3] >= MIN_DEPTH), key=lambda it: -it[3])
    wave, used = [], 0
    for it in big:
        need = _footprint(it[3], len(it[1]))
        if wave and used + need > budget_bytes:
            _run_wave(wave, out, dev, point_weight, confidence, scale, samples_per_node, tol, max_cycles, device_out,
                      phases)
            wave, used = [], 0
        wave.append(it)
        used += need
    if wave:
        _run_wave(wave, out, dev, point_weight, confidence, scale, samples_per_node, tol, max_cycles, device_out,
                  phases)
    return out


def _run_wave(wave, out, dev, point_weight, confidence, scale, samples_per_node, tol, max_cycles, device_out,
              phases: _Phases):
    with _trace.stage(f"batch wave of {len(wave)}"):
        _run_wave_body(wave, out, dev, point_weight, confidence, scale, samples_per_node, tol, max_cycles,
                       device_out, phases)


def _run_wave_body(wave, out, dev, point_weight, confidence, scale, samples_per_node, tol, max_cycles, device_out,
                   phases: _Phases):
    L = nat.lib()
    ctx = core._Context()
    s = ctx.stream
    # one pinned staging buffer and one host-to-device copy for the wave's points and normals
    sizes = [len(p) for _, p, _, _ in wave]
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    total = int(offsets[-1])
    staging = torch.empty((2, max(total, 1), 3), dtype=torch.float64, pin_memory=True)
    for j, (_, p, nrm, _) in enumerate(wave):
        a, b = int(offsets[j]), int(offsets[j + 1])
        for slot, arr in ((0, p), (1, nrm)):
            src = arr if isinstance(arr, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(arr))
            staging[slot, a:b].copy_(src.to(torch.float64))
    both = staging.to(dev, non_blocking=True)
    phases.mark("stage and upload")
    # preparation of every cloud, then one read of all kept counts
    kept = torch.zeros(len(wave), dtype=torch.int64, device=dev)
    maps = torch.empty((len(wave), 4), dtype=torch.float64, device=dev)
    prepared = []
    prep_ws = nat.Workspace(dev)
    for j, (_, p, _, _) in enumerate(wave):
        a, b = int(offsets[j]), int(offsets[j + 1])
        count = b - a
        out_p = torch.empty((count, 3), dtype=torch.float64, device=dev)
        out_n = torch.empty((count, 3), dtype=torch.float64, device=dev)
        if count:
            ptr, size = prep_ws.get(L.pb_prepare_workspace_size(count))
            ctx.check(L.pb_prepare_points_f64(both[0, a:b].data_ptr(), both[1, a:b].data_ptr(), count, scale,
                                              out_p.data_ptr(), out_n.data_ptr(), kept[j:j + 1].data_ptr(),
                                              maps[j].data_ptr(), ptr, size, s), "prepare points")
        prepared.append((out_p, out_n))
    _sync.wait("prepare points")
    kept_h = kept.cpu().numpy()
    del both
    phases.mark("prepare")
    solve_idx, grids, accepted_all = [], [], []
    for j, (_, _, _, d) in enumerate(wave):
        k = int(kept_h[j])
        if k == 0:
            grids.append(None)
            accepted_all.append(None)
            continue
        dp, dn = prepared[j][0][:k], prepared[j][1][:k]
        prepared[j] = (dp, dn)
        g, acc = core._splat_assemble(ctx, dp, dn, d, point_weight, confidence, samples_per_node)
        grids.append(g)
        accepted_all.append(acc)
        solve_idx.append(j)
    ctx.ws = nat.Workspace(dev)  # the splats' scratch is not needed past this point
    phases.mark("splat and assemble")
    fields = {}
    stats = {}
    if solve_idx:
        solver = BatchSolver([(1 << wave[j][3]) + 1 for j in solve_idx], dev)
        phases.mark("solver allocation")
        f, st = solver.solve([grids[j]["rhs"] for j in solve_idx], [grids[j]["screen"] for j in solve_idx],
                             point_weight, tol=tol, max_cycles=max_cycles, phases=phases)
        for j, fj, sj in zip(solve_idx, f, st):
            fields[j], stats[j] = fj, sj
        solver.release()
        del solver
    phases.mark("solve")
    # iso-values and extraction counts for every cloud, then one read of all counts
    pending = []
    counts = torch.zeros((len(wave), 2), dtype=torch.int64, device=dev)
    ws_list = {}
    for j in solve_idx:
        dp, dn = prepared[j]
        iso = core._iso_value(ctx, fields[j], dp, dn, confidence)
        n = fields[j].shape[0]
        ws = nat.Workspace(dev)
        ptr, size = ws.get(L.pb_extract_workspace_size(n))
        ctx.check(L.pb_extract_count_f64(fields[j].data_ptr(), n, iso.data_ptr(), counts[j].data_ptr(), ptr, size, s),
                  "extract count")
        ws_list[j] = (ws, ptr, size)
        pending.append((j, iso))
    acc_check = torch.stack([a for a in accepted_all if a is not None]) if solve_idx else None
    _sync.wait("extract count")
    host_counts = counts.cpu().numpy()
    phases.mark("iso and extraction counts")
    if acc_check is not None:
        acc_h = acc_check.cpu().numpy().ravel()
        for j, a in zip(solve_idx, acc_h):
            if int(a) != int(kept_h[j]):
                raise RuntimeError(f"splat accepted {int(a)} of {int(kept_h[j])} validated samples")
    results = {}
    for j, iso in pending:
        nv, nf = (int(v) for v in host_counts[j])
        n = fields[j].shape[0]
        vertices = torch.empty((nv, 3), dtype=torch.float64, device=dev)
        vdens = torch.empty(nv, dtype=torch.float64, device=dev)
        faces = torch.empty((nf, 3), dtype=torch.int64, device=dev)
        _, ptr, size = ws_list[j]
        if nv:
            ctx.check(L.pb_extract_emit_f64(fields[j].data_ptr(), grids[j]["density"].data_ptr(), n, iso.data_ptr(),
                                            vertices.data_ptr(), vdens.data_ptr(), faces.data_ptr() if nf else None,
                                            ptr, size, s), "extract emit")
            ctx.check(L.pb_map_vertices_f64(vertices.data_ptr(), nv, maps[j].data_ptr(), s), "map vertices")
        results[j] = (vertices, faces, vdens, iso)
    phases.mark("extraction emit")
    # meshes to the host together (pinned buffers, one synchronisation)
    flat = []
    for j in sorted(results):
        flat.extend(results[j])
    host = core._host_all(flat, device_out)
    for i, j in enumerate(sorted(results)):
        v, f, dd, iso = host[4 * i: 4 * i + 4]
        iso_v = float(iso[0]) if not device_out else float(iso[0].item())
        out[wave[j][0]] = core.Mesh(v, f, dd, iso_v, float(stats[j].residual_norm))
    for j in range(len(wave)):
        if j not in results:
            out[wave[j][0]] = _empty_mesh(dev, device_out)
    phases.mark("results to host")


def _empty_mesh(dev, device_out: bool):
    if device_out:
        return core.Mesh(torch.empty((0, 3), dtype=torch.float64, device=dev),
                         torch.empty((0, 3), dtype=torch.int64, device=dev),
                         torch.empty(0, dtype=torch.float64, device=dev))
    return core.Mesh(np.empty((0, 3), np.float64), np.empty((0, 3), np.int64), np.empty(0))
