"""Continuous batching of reconstructions on one GPU.

A `Server` keeps `lanes` workers; each owns a CUDA stream and its own solver
engines (grid hierarchies, FCG vectors and the captured iteration graph stay
on the device between requests), so several reconstructions run on the device
at once.  Requests wait in a FIFO queue and are admitted as soon as a lane is
free and their estimated HBM footprint fits next to the requests already in
flight; a request that arrives while others are running starts as soon as
those conditions hold, without waiting for a batch boundary.  Every request
runs exactly the single-request code path (`core.reconstruct`), so its result
is the same alone and in the mix: all kernels are deterministic.

`reconstruct_batch` runs a list of clouds through a temporary server.
"""

from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import torch

from . import core, solver32


def footprint_bytes(depth: int, points: int) -> int:
    """Device bytes one reconstruction at `depth` with `points` samples needs
    transiently (grids, solver vectors, FP32 levels, splat records, extraction)."""
    n = (1 << depth) + 1
    grids = 8 * n**3 * 9            # FP64: density, screen, rhs, solver copies, cell map
    levels = 4 * (n + 2) ** 2 * (((n + 5) + 7) & ~7) * 6 * 8 // 7  # FP32 hierarchy
    samples = points * (48 * 2 + 8 * 24)
    return int(grids + levels + samples)


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
    timing: Timing = field(default_factory=Timing)


class Server:
    """Admit and run reconstructions concurrently (see the module docstring).

    submit() returns a Future whose result is (Mesh, Timing)."""

    def __init__(self, lanes: int = 4, memory_fraction: float = 0.6, device: int | None = None,
                 budget_bytes: int | None = None, runner=None, **defaults):
        """runner: optional callable(points, normals, **kwargs) -> result that
        replaces the GPU reconstruction (the queueing and admission logic is
        then exercised without a device, as the tests do)."""
        if lanes < 1:
            raise ValueError("lanes must be positive")
        self._runner = runner
        if runner is None:
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
        self._threads = [threading.Thread(target=self._lane, args=(i,), daemon=True) for i in range(lanes)]
        for t in self._threads:
            t.start()

    # -- client side ----------------------------------------------------------
    def submit(self, points, normals, **kwargs) -> Future:
        args = dict(self.defaults)
        args.update(kwargs)
        depth = int(args.get("depth", 6))
        count = len(points)
        req = _Request(points, normals, args, footprint_bytes(depth, count), Future())
        req.timing.arrival = time.perf_counter()
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

    # -- lanes ----------------------------------------------------------------
    def _take(self) -> _Request | None:
        with self._cv:
            while True:
                if self._queue:
                    head = self._queue[0]
                    if self._inflight == 0 or self._inflight_bytes + head.footprint <= self.budget:
                        self._queue.popleft()
                        self._inflight += 1
                        self._inflight_bytes += head.footprint
                        return head
                elif self._closed:
                    return None
                self._cv.wait(timeout=0.5)

    def _release(self, req: _Request) -> None:
        with self._cv:
            self._inflight -= 1
            self._inflight_bytes -= req.footprint
            self.completed += 1
            self._cv.notify_all()

    def _lane(self, index: int) -> None:
        stream = None
        if self._runner is None:
            torch.cuda.set_device(self.device)
            solver32.set_slot(index + 1)  # slot 0 is the submitting thread's own
            stream = torch.cuda.Stream(device=self.device)
        while True:
            req = self._take()
            if req is None:
                return
            req.timing.start = time.perf_counter()
            try:
                if stream is None:
                    result = self._runner(req.points, req.normals, **req.kwargs)
                else:
                    with torch.cuda.stream(stream):
                        result = core.reconstruct(req.points, req.normals, **req.kwargs)
                        stream.synchronize()
                req.timing.end = time.perf_counter()
                req.future.set_result((result, req.timing))
            except BaseException as error:  # report it to the submitter, keep serving
                req.timing.end = time.perf_counter()
                req.future.set_exception(error)
            finally:
                self._release(req)


def reconstruct_batch(clouds, *, lanes: int = 4, **kwargs) -> list:
    """Reconstruct many clouds concurrently; `clouds` holds (points, normals) or
    (points, normals, depth) tuples.  Returns the meshes in input order."""
    with Server(lanes=lanes, **kwargs) as server:
        futures = []
        for cloud in clouds:
            if len(cloud) == 3:
                p, nrm, depth = cloud
                futures.append(server.submit(p, nrm, depth=int(depth)))
            else:
                p, nrm = cloud
                futures.append(server.submit(p, nrm))
        return [f.result()[0] for f in futures]
