"""Continuous batching of reconstructions on one GPU.

A `Server` keeps `lanes` workers.  Requests wait in a FIFO queue; a free lane
takes the queue's head and, from the requests queued behind it, those of the
same depth and parameters (up to `max_batch`) while their estimated device
footprints fit next to the requests already in flight, and runs them as one
batch: `batch.reconstruct_many`, whose solver does one grouped launch per
solver step for all of the batch's clouds.
A request that arrives while batches are on the GPU joins the next batch a
lane takes, so the GPU never waits for a batch boundary while work is queued,
and with two or more lanes one batch's host work (preparation, result copies)
overlaps another's device work.  Every request's mesh is bit-identical to
`core.reconstruct` of it alone (the batched path runs the same kernels on the
same data per cloud, and every kernel is deterministic).

Failure handling, all on the host:
* a request larger than the whole budget is refused at submission (MemoryError);
* `deadline` (seconds after arrival): a request still queued at its deadline
  is dropped with DeadlineExceeded; a running batch's device waits poll with
  the latest deadline of its requests (_sync) and a request finishing past its
  own deadline is reported as DeadlineExceeded;
* a client may cancel a queued request (Future.cancel());
* a batch whose device allocation fails (out of memory) releases the solver
  caches and runs again one request at a time; a request that still does not
  fit gets MemoryError, and serving continues;
* any other error of a batch is attributed by running its requests one at a
  time, so one bad request fails alone.

`reconstruct_batch` runs a list of clouds through a temporary server.
"""

from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import torch

from . import _sync, core, solver32

# Fields of the request kwargs that may differ inside one batch, and the
# reconstruction parameters that must match for requests to share one.
_PER_CLOUD = ("depth",)
_SHARED = ("point_weight", "confidence", "scale", "samples_per_node", "precision", "tol", "max_cycles", "cycles",
           "device_out")


def _pitch(m: int) -> int:
    return ((m + 5) + 7) & ~7


def _padded(m: int) -> int:
    return (m + 2) * (m + 2) * _pitch(m)


def _levels(n: int) -> list:
    sizes = [n]
    while sizes[-1] > 3:
        sizes.append((sizes[-1] + 1) // 2)
    return sizes


def hierarchy_bytes(n: int) -> int:
    """Device bytes of the FP32 preconditioner of side n (solver32.Hierarchy32):
    level 0 six padded arrays; every level below it 20 (14 coefficient planes
    and six work arrays); levels of side 17..129 also their packed couplings
    (two colours of 64 + 4 bytes per compact node)."""
    total = 0
    for i, m in enumerate(_levels(n)):
        if i == 0 and m >= solver32.TMA_MIN_N:
            total += 6 * 4 * _padded(m)
            continue
        total += 20 * 4 * _padded(m)
        if m > solver32.COARSE_N:  # packed per colour
            total += 2 * 68 * (m * m * ((m + 1) // 2))
    return total + 8 * 27 * 27 + 64 * 1024  # 3^3 inverse (FP64), coarse image


def footprint_bytes(depth: int, points: int) -> int:
    """Peak device bytes of one FP32-refined reconstruction at `depth` with
    `points` samples in a batch: the inputs and their prepared copies, the six
    FP64 grids and the splat's workspace while splatting; then density, screen
    and rhs, the FP32 hierarchy, the FCG vectors (x twice in FP64, p twice in
    FP32), the Galerkin scratch and the returned field during the solve, with
    the extraction workspace and an allowance for the mesh after it.  Sizes
    come from the library's own size queries where it has one."""
    from . import _native as nat

    n = (1 << depth) + 1
    N = n ** 3
    lib = nat.lib()
    inputs = 4 * 24 * points
    splat_ws = int(lib.pb_splat_workspace_size(max(points, 1), n))
    splat = 6 * 8 * N + splat_ws
    solve = 3 * 8 * N + hierarchy_bytes(n) + 2 * 8 * N + 2 * 4 * N + solver32.galerkin_scratch_bytes(n) + 8 * N
    extract = int(lib.pb_extract_workspace_size(n)) + 256 * n * n
    # the splat's workspace is counted in both phases: the caching allocator may
    # keep its block resident into the solve
    return int(inputs + splat_ws + max(6 * 8 * N, solve + extract))


@dataclass
class Timing:
    arrival: float = 0.0
    start: float = 0.0
    end: float = 0.0

    @property
    def latency_ms(self) -> float:
        return (self.end - self.arrival) * 1e3

    @property
    def service_ms(self) -> float:
        return (self.end - self.start) * 1e3


@dataclass
class _Request:
    points: object
    normals: object
    kwargs: dict
    footprint: int
    future: Future
    deadline: float | None = None  # time.monotonic() by which it must finish
    timing: Timing = field(default_factory=Timing)


class Server:
    """Admit and run reconstructions concurrently (see the module docstring).

    submit() returns a Future whose result is (Mesh, Timing)."""

    def __init__(self, lanes: int = 2, memory_fraction: float = 0.6, device: int | None = None,
                 budget_bytes: int | None = None, runner=None, batch_runner=None, max_batch: int = 64,
                 drain_limit_s: float = 600.0, group_depths: bool = True, lookahead: int = 256, on_result=None,
                 **defaults):
        """runner: optional callable(points, normals, **kwargs) -> result that
        replaces one GPU reconstruction; batch_runner: optional callable(list of
        (points, normals, kwargs)) -> list of results (or exceptions) that
        replaces a batched one.  With either, the queueing, admission and
        failure logic runs without a device, as the tests do.  max_batch = 1
        runs one reconstruction per lane at a time (core.reconstruct).
        drain_limit_s bounds how long a lane waits for the device work of a
        request that overran its deadline before it gives the lane up.
        group_depths: a batch takes requests of its head's depth only;
        lookahead: how many queued requests behind the head a lane scans.
        on_result: optional callable(mesh) -> value that the future gets in the
        mesh's place (a caller that writes meshes out or keeps only their sizes
        need not hold every mesh until it reads its future)."""
        if lanes < 1:
            raise ValueError("lanes must be positive")
        if max_batch < 1:
            raise ValueError("max_batch must be positive")
        self._runner = runner
        self._batch_runner = batch_runner
        self.max_batch = int(max_batch)
        self.drain_limit_s = float(drain_limit_s)
        self.group_depths = bool(group_depths)
        self.lookahead = int(lookahead)
        self.on_result = on_result
        self._fake = runner is not None or batch_runner is not None
        if not self._fake:
            self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
            total = torch.cuda.get_device_properties(self.device).total_memory
            self.budget = int(memory_fraction * total) if budget_bytes is None else int(budget_bytes)
        else:
            self.device = None
            self.budget = int(budget_bytes if budget_bytes is not None else 1 << 40)
        self.defaults = dict(precision="fp32_refined", tol=1e-8)
        self.defaults.update(defaults)
        self._queue: collections.deque[_Request] = collections.deque()
        self._cv = threading.Condition()
        self._inflight_bytes = 0
        self._inflight = 0
        self._closed = False
        self.completed = 0
        self.batches = 0
        self.lost_lanes = 0
        self._threads = [threading.Thread(target=self._lane, args=(i,), daemon=True) for i in range(lanes)]
        for t in self._threads:
            t.start()

    # -- client side ----------------------------------------------------------
    def submit(self, points, normals, deadline: float | None = None, **kwargs) -> Future:
        args = dict(self.defaults)
        args.update(kwargs)
        depth = int(args.get("depth", 6))
        count = len(points)
        fp = footprint_bytes(depth, count)
        req = _Request(points, normals, args, fp, Future())
        req.timing.arrival = time.perf_counter()
        if deadline is not None:
            req.deadline = time.monotonic() + float(deadline)
        if req.footprint > self.budget:
            req.future.set_exception(MemoryError(
                f"request needs about {req.footprint / 2**30:.1f} GiB, more than the server's budget of "
                f"{self.budget / 2**30:.1f} GiB"))
            return req.future
        with self._cv:
            if self._closed:
                raise RuntimeError("server is closed")
            self._queue.append(req)
            self._cv.notify_all()
        return req.future

    def close(self, wait: bool = True) -> None:
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        if wait:
            for t in self._threads:
                t.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def inflight_bytes(self) -> int:
        return self._inflight_bytes

    # -- lanes ----------------------------------------------------------------
    def _expire_queued(self) -> None:
        """Drop queued requests that were cancelled or whose deadline passed (lock held)."""
        now = time.monotonic()
        keep = collections.deque()
        for r in self._queue:
            if r.future.cancelled():
                continue
            if r.deadline is not None and now >= r.deadline:
                r.timing.end = time.perf_counter()
                r.future.set_exception(_sync.DeadlineExceeded("deadline passed while the request was queued"))
                continue
            keep.append(r)
        self._queue = keep

    def _compatible(self, a: _Request, b: _Request) -> bool:
        return all(a.kwargs.get(k) == b.kwargs.get(k) for k in _SHARED)

    def _take(self) -> list | None:
        """The next batch: the queue's head (alone if nothing is in flight and it
        needs the whole budget) and, from the next `lookahead` queued requests,
        those that suit the same batch (same parameters and, with
        group_depths, the same depth, so small requests do not wait on deep
        ones) while they fit next to what is in flight.  Requests passed over
        keep their places."""
        with self._cv:
            while True:
                self._expire_queued()
                if self._queue:
                    head = self._queue[0]
                    if self._inflight == 0 or self._inflight_bytes + head.footprint <= self.budget:
                        self._queue.popleft()
                        taken = [head] if head.future.set_running_or_notify_cancel() else []
                        used = self._inflight_bytes + (head.footprint if taken else 0)
                        if taken:
                            rest = collections.deque()
                            scanned = 0
                            while self._queue and len(taken) < self.max_batch and scanned < self.lookahead:
                                nxt = self._queue.popleft()
                                scanned += 1
                                if (self._compatible(head, nxt) and used + nxt.footprint <= self.budget
                                        and (not self.group_depths or
                                             nxt.kwargs.get("depth") == head.kwargs.get("depth"))):
                                    if nxt.future.set_running_or_notify_cancel():
                                        used += nxt.footprint
                                        taken.append(nxt)
                                    continue
                                rest.append(nxt)
                            rest.extend(self._queue)
                            self._queue = rest
                        if not taken:
                            continue
                        self._inflight += len(taken)
                        self._inflight_bytes = used
                        return taken
                elif self._closed:
                    return None
                self._cv.wait(timeout=0.05)

    def _release(self, reqs: list) -> None:
        with self._cv:
            self._inflight -= len(reqs)
            self._inflight_bytes -= sum(r.footprint for r in reqs)
            self.completed += len(reqs)
            self.batches += 1
            self._cv.notify_all()

    def _deliver(self, req: _Request, result) -> None:
        req.timing.end = time.perf_counter()
        if isinstance(result, BaseException):
            req.future.set_exception(result)
        elif req.deadline is not None and time.monotonic() > req.deadline:
            req.future.set_exception(_sync.DeadlineExceeded("the request finished after its deadline"))
        else:
            if self.on_result is not None:
                try:
                    result = self.on_result(result)
                except BaseException as error:
                    req.future.set_exception(error)
                    return
            req.future.set_result((result, req.timing))

    def _run_one(self, req: _Request):
        if self._runner is not None:
            return self._runner(req.points, req.normals, **req.kwargs)
        if self._batch_runner is not None:
            out = self._batch_runner([(req.points, req.normals, req.kwargs)])[0]
            if isinstance(out, BaseException):
                raise out
            return out
        kw = dict(req.kwargs)
        return core.reconstruct(req.points, req.normals, **kw)

    def _run_batch(self, reqs: list) -> list:
        """Results (or exceptions) of a batch, in order."""
        if (self._batch_runner is None and self._runner is not None) or \
                (self.max_batch == 1 and self._batch_runner is None):
            out = []
            for r in reqs:
                try:
                    out.append(self._run_one(r))
                except BaseException as error:  # reported to its own client
                    out.append(error)
            return out
        if self._batch_runner is not None:
            return list(self._batch_runner([(r.points, r.normals, r.kwargs) for r in reqs]))
        from . import batch

        kw = reqs[0].kwargs
        if kw.get("precision", "fp64") != "fp32_refined" or kw.get("cycles") is not None or \
                any(k not in _SHARED and k not in _PER_CLOUD for k in kw):
            return [self._safe_one(r) for r in reqs]
        shared = {k: kw[k] for k in _SHARED if k in kw and k not in ("precision", "cycles")}
        clouds = [(r.points, r.normals, int(r.kwargs.get("depth", 6))) for r in reqs]
        return batch.reconstruct_many(clouds, budget_bytes=self.budget, **shared)

    def _safe_one(self, req: _Request):
        try:
            return self._run_one(req)
        except BaseException as error:
            return error

    def _run_with_recovery(self, reqs: list) -> list:
        try:
            return self._run_batch(reqs)
        except _sync.DeadlineExceeded as error:
            return [error] * len(reqs)
        except (torch.cuda.OutOfMemoryError, MemoryError):
            # device memory refused: release cached solver state, then one at a time
            solver32.clear_engines()
            if torch.cuda.is_available():
                torch.cuda.empty_cache()
            out = []
            for r in reqs:
                try:
                    out.append(self._run_one(r))
                except (torch.cuda.OutOfMemoryError, MemoryError) as error:
                    out.append(MemoryError(f"device memory refused for this request: {error}"))
                except BaseException as error:
                    out.append(error)
            return out
        except BaseException:
            if len(reqs) == 1:
                raise
            return [self._safe_one(r) for r in reqs]  # attribute the failure to its request

    def _lane(self, index: int) -> None:
        stream = None
        if not self._fake:
            torch.cuda.set_device(self.device)
            solver32.set_slot(index + 1)  # slot 0 is the submitting thread's own
            stream = torch.cuda.Stream(device=self.device)
        while True:
            reqs = self._take()
            if reqs is None:
                return
            start = time.perf_counter()
            for r in reqs:
                r.timing.start = start
            deadlines = [r.deadline for r in reqs]
            when = None if any(d is None for d in deadlines) else max(deadlines)
            lane_ok = True
            try:
                with _sync.deadline(when):
                    if stream is None:
                        results = self._run_with_recovery(reqs)
                    else:
                        with torch.cuda.stream(stream):
                            results = self._run_with_recovery(reqs)
                            _sync.wait("lane results")
                            stream.synchronize()
            except BaseException as error:
                results = [error] * len(reqs)
            if stream is not None and any(isinstance(r, _sync.DeadlineExceeded) for r in results):
                # the device work of an overrun keeps its memory until it finishes
                try:
                    _sync.poll(_recorded(stream), time.monotonic() + self.drain_limit_s, "lane drain")
                except _sync.DeadlineExceeded:
                    lane_ok = False
            for r, res in zip(reqs, results):
                self._deliver(r, res)
            self._release(reqs)
            if not lane_ok:
                with self._cv:
                    self.lost_lanes += 1
                return


def _recorded(stream):
    event = torch.cuda.Event()
    event.record(stream)
    return event.query


def reconstruct_batch(clouds, *, lanes: int = 2, max_batch: int = 64, **kwargs) -> list:
    """Reconstruct many clouds through a temporary server; `clouds` holds
    (points, normals) or (points, normals, depth) tuples.  Returns the meshes
    in input order."""
    with Server(lanes=lanes, max_batch=max_batch, **kwargs) as server:
        futures = []
        for cloud in clouds:
            if len(cloud) == 3:
                p, nrm, depth = cloud
                futures.append(server.submit(p, nrm, depth=int(depth)))
            else:
                p, nrm = cloud
                futures.append(server.submit(p, nrm))
        return [f.result()[0] for f in futures]
