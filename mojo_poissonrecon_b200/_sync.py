"""Host waits on the device with an optional per-thread deadline.

The public API synchronises the host a few times per reconstruction (point
counts, the solver's iteration count, mesh sizes, the result copies).  A
serving lane sets a deadline for its thread (`deadline`); every such wait then
polls a CUDA event instead of blocking and raises DeadlineExceeded once the
deadline passes, so a request that overruns is reported to its client while
the lane stays responsive.  Work already queued on the device is not
cancelled: it finishes in stream order, and the lane accounts its memory until
it has.  Without a deadline `wait` returns at once and the caller's blocking
copy does the synchronisation, as before.
"""

from __future__ import annotations

import contextlib
import threading
import time

_LOCAL = threading.local()


class DeadlineExceeded(TimeoutError):
    """A host wait on the device ran past the calling thread's deadline."""


@contextlib.contextmanager
def deadline(when: float | None):
    """Within the block, device waits of this thread give up at time.monotonic() >= when."""
    previous = getattr(_LOCAL, "deadline", None)
    _LOCAL.deadline = when
    try:
        yield
    finally:
        _LOCAL.deadline = previous


def current_deadline() -> float | None:
    return getattr(_LOCAL, "deadline", None)


def poll(query, when: float, what: str = "device work", clock=time.monotonic, sleep=time.sleep) -> None:
    """Call query() until it returns true; raise DeadlineExceeded once clock() >= when.
    The poll interval starts at 20 us and doubles up to 1 ms."""
    delay = 2e-5
    while not query():
        if clock() >= when:
            raise DeadlineExceeded(f"{what}: deadline passed before the device finished")
        sleep(delay)
        delay = min(2 * delay, 1e-3)


def wait(what: str = "device work", stream=None) -> None:
    """Wait for the work queued so far on `stream` (default: the current
    stream) when this thread has a deadline; otherwise return at once."""
    when = current_deadline()
    if when is None:
        return
    import torch

    event = torch.cuda.Event()
    event.record(stream)
    poll(event.query, when, what)
