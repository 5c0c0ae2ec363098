"""Continuous batching: admission by HBM footprint, overlap of requests that
arrive while others run, batches formed from whatever is queued, host-side
failure handling (deadlines, cancellation, allocator refusal, one bad request
in a batch), and identical results alone and in the mix."""

import threading
import time

import numpy as np
import pytest

from mojo_poissonrecon_b200 import serve


class FakeGPU:
    """Stands in for the device: records concurrency and the footprints in flight."""

    def __init__(self, server_ref, delay=0.05):
        self.lock = threading.Lock()
        self.active = 0
        self.max_active = 0
        self.delay = delay
        self.server_ref = server_ref
        self.max_bytes = 0
        self.starts = []

    def __call__(self, points, normals, **kw):
        with self.lock:
            self.active += 1
            self.max_active = max(self.max_active, self.active)
            self.starts.append(kw["tag"])
            self.max_bytes = max(self.max_bytes, self.server_ref[0]._inflight_bytes)
        time.sleep(kw.get("sleep", self.delay))
        with self.lock:
            self.active -= 1
        return kw["tag"]


def make_server(lanes, budget, delay=0.05):
    ref = []
    fake = FakeGPU(ref, delay)
    server = serve.Server(lanes=lanes, budget_bytes=budget, runner=fake, max_batch=1)
    ref.append(server)
    return server, fake


def test_footprint_grows_with_depth_and_points():
    assert serve.footprint_bytes(6, 1000) < serve.footprint_bytes(7, 1000) < serve.footprint_bytes(8, 1000)
    assert serve.footprint_bytes(8, 10_000) < serve.footprint_bytes(8, 1_000_000)


def test_admission_keeps_inflight_footprint_within_budget():
    fp = serve.footprint_bytes(7, 1000)
    server, fake = make_server(lanes=4, budget=int(2.5 * fp))  # room for two at a time
    futures = [server.submit(np.zeros((1000, 3)), np.ones((1000, 3)), depth=7, tag=i) for i in range(8)]
    results = [f.result(timeout=30)[0] for f in futures]
    server.close()
    assert results == list(range(8))
    assert fake.max_active == 2
    assert fake.max_bytes <= int(2.5 * fp)
    assert fake.starts == list(range(8))  # FIFO admission


def test_request_too_large_is_rejected_without_blocking_others():
    server, fake = make_server(lanes=2, budget=serve.footprint_bytes(6, 100) * 2)
    big = server.submit(np.zeros((10, 3)), np.ones((10, 3)), depth=10, tag="big")
    small = server.submit(np.zeros((10, 3)), np.ones((10, 3)), depth=6, tag="small")
    with pytest.raises(MemoryError):
        big.result(timeout=10)
    assert small.result(timeout=10)[0] == "small"
    server.close()


def test_request_arriving_mid_flight_starts_before_the_first_finishes():
    server, fake = make_server(lanes=2, budget=1 << 40)
    a = server.submit(np.zeros((10, 3)), np.ones((10, 3)), depth=6, tag="a", sleep=0.5)
    time.sleep(0.1)
    b = server.submit(np.zeros((10, 3)), np.ones((10, 3)), depth=6, tag="b", sleep=0.05)
    (ra, ta), (rb, tb) = a.result(timeout=10), b.result(timeout=10)
    server.close()
    assert tb.start < ta.end  # admitted while a was still running
    assert tb.end < ta.end


def test_failures_are_reported_and_serving_continues():
    def runner(points, normals, **kw):
        if kw["tag"] == "bad":
            raise ValueError("bad request")
        return kw["tag"]

    server = serve.Server(lanes=1, budget_bytes=1 << 40, runner=runner, max_batch=1)
    bad = server.submit(np.zeros((1, 3)), np.ones((1, 3)), depth=5, tag="bad")
    good = server.submit(np.zeros((1, 3)), np.ones((1, 3)), depth=5, tag="good")
    with pytest.raises(ValueError):
        bad.result(timeout=10)
    assert good.result(timeout=10)[0] == "good"
    server.close()


class FakeBatchGPU:
    """Stands in for the batched device path: records every batch's tags."""

    def __init__(self, delay=0.05, fail_tag=None, oom_batches=0):
        self.lock = threading.Lock()
        self.batches = []
        self.delay = delay
        self.fail_tag = fail_tag
        self.oom_batches = oom_batches

    def __call__(self, items):
        tags = [kw["tag"] for _, _, kw in items]
        with self.lock:
            self.batches.append(tags)
            oom = self.oom_batches > 0 and len(items) > 1
            if oom:
                self.oom_batches -= 1
        if oom:
            raise MemoryError("simulated device allocation refusal")
        if self.fail_tag in tags:
            raise ValueError("one request of the batch is bad")
        time.sleep(max(kw.get("sleep", self.delay) for _, _, kw in items))
        return tags


def cloud():
    return np.zeros((10, 3)), np.ones((10, 3))


def test_queued_requests_form_the_next_batch():
    fake = FakeBatchGPU(delay=0.3)
    server = serve.Server(lanes=1, budget_bytes=1 << 40, batch_runner=fake, max_batch=8, group_depths=False)
    first = server.submit(*cloud(), depth=6, tag=0)
    time.sleep(0.1)  # the first batch (one request) is on the "device"
    rest = [server.submit(*cloud(), depth=6 + (k % 2), tag=k) for k in range(1, 6)]
    assert first.result(timeout=10)[0] == 0
    assert [f.result(timeout=10)[0] for f in rest] == [1, 2, 3, 4, 5]
    server.close()
    assert fake.batches == [[0], [1, 2, 3, 4, 5]]  # arrivals during a batch run together next


def test_batches_group_one_depth_and_keep_the_others_in_order():
    fake = FakeBatchGPU(delay=0.2)
    server = serve.Server(lanes=1, budget_bytes=1 << 40, batch_runner=fake, max_batch=8)
    gate = server.submit(*cloud(), depth=5, tag="gate")
    time.sleep(0.05)
    order = [(6, "a"), (9, "b"), (6, "c"), (7, "d"), (9, "e"), (6, "f")]
    futures = [server.submit(*cloud(), depth=d, tag=t) for d, t in order]
    gate.result(timeout=10)
    assert [f.result(timeout=10)[0] for f in futures] == [t for _, t in order]
    server.close()
    assert fake.batches == [["gate"], ["a", "c", "f"], ["b", "e"], ["d"]]


def test_batches_respect_the_budget_and_max_batch():
    fp = serve.footprint_bytes(7, 10)
    fake = FakeBatchGPU(delay=0.05)
    server = serve.Server(lanes=1, budget_bytes=3 * fp, batch_runner=fake, max_batch=8)
    futures = [server.submit(*cloud(), depth=7, tag=k) for k in range(7)]
    assert [f.result(timeout=10)[0] for f in futures] == list(range(7))
    server.close()
    assert max(len(b) for b in fake.batches) <= 3
    assert sum(fake.batches, []) == list(range(7))  # FIFO


def test_deadline_passes_while_queued():
    fake = FakeBatchGPU(delay=0.4)
    server = serve.Server(lanes=1, budget_bytes=1 << 40, batch_runner=fake, max_batch=1)
    busy = server.submit(*cloud(), depth=6, tag="busy")
    time.sleep(0.05)
    late = server.submit(*cloud(), deadline=0.1, depth=6, tag="late")
    ok = server.submit(*cloud(), depth=6, tag="ok")
    with pytest.raises(serve._sync.DeadlineExceeded):
        late.result(timeout=10)
    assert busy.result(timeout=10)[0] == "busy" and ok.result(timeout=10)[0] == "ok"
    server.close()
    assert ["late"] not in fake.batches  # never started


def test_deadline_during_a_device_wait():
    """A device wait that never completes (a fake event) gives up at the
    request's deadline; the lane then serves the next request."""
    from mojo_poissonrecon_b200 import _sync

    def runner(points, normals, **kw):
        if kw["tag"] == "stuck":
            _sync.poll(lambda: False, _sync.current_deadline(), "fake device work")
        return kw["tag"]

    server = serve.Server(lanes=1, budget_bytes=1 << 40, runner=runner, max_batch=1)
    t0 = time.monotonic()
    stuck = server.submit(*cloud(), deadline=0.2, depth=6, tag="stuck")
    nxt = server.submit(*cloud(), depth=6, tag="next")
    with pytest.raises(_sync.DeadlineExceeded):
        stuck.result(timeout=10)
    assert time.monotonic() - t0 < 5
    assert nxt.result(timeout=10)[0] == "next"
    server.close()


def test_poll_gives_up_at_the_deadline_with_a_fake_clock():
    from mojo_poissonrecon_b200 import _sync

    now = [0.0]
    sleeps = []

    def sleep(dt):
        sleeps.append(dt)
        now[0] += dt

    with pytest.raises(_sync.DeadlineExceeded):
        _sync.poll(lambda: False, 0.01, "x", clock=lambda: now[0], sleep=sleep)
    assert now[0] >= 0.01 and max(sleeps) <= 1e-3
    calls = iter([False, False, True])
    _sync.poll(lambda: next(calls), 1.0, "y", clock=lambda: 0.0, sleep=lambda dt: None)
    assert _sync.current_deadline() is None
    with _sync.deadline(5.0):
        assert _sync.current_deadline() == 5.0
    assert _sync.current_deadline() is None


def test_cancelled_request_never_runs():
    fake = FakeBatchGPU(delay=0.3)
    server = serve.Server(lanes=1, budget_bytes=1 << 40, batch_runner=fake, max_batch=1)
    busy = server.submit(*cloud(), depth=6, tag="busy")
    time.sleep(0.05)
    gone = server.submit(*cloud(), depth=6, tag="gone")
    assert gone.cancel()
    after = server.submit(*cloud(), depth=6, tag="after")
    assert busy.result(timeout=10)[0] == "busy" and after.result(timeout=10)[0] == "after"
    server.close()
    assert ["gone"] not in fake.batches


def test_allocator_refusal_retries_one_at_a_time():
    fake = FakeBatchGPU(delay=0.01, oom_batches=1)
    server = serve.Server(lanes=1, budget_bytes=1 << 40, batch_runner=fake, max_batch=8)
    gate = server.submit(*cloud(), depth=6, tag="gate", sleep=0.2)
    time.sleep(0.05)
    futures = [server.submit(*cloud(), depth=6, tag=k) for k in range(3)]
    assert gate.result(timeout=10)[0] == "gate"
    assert [f.result(timeout=10)[0] for f in futures] == [0, 1, 2]
    server.close()
    assert [0, 1, 2] in fake.batches and [0] in fake.batches and [2] in fake.batches


def test_allocator_refusal_of_a_single_request_is_reported():
    def runner(points, normals, **kw):
        if kw["tag"] == "huge":
            raise MemoryError("simulated device allocation refusal")
        return kw["tag"]

    server = serve.Server(lanes=1, budget_bytes=1 << 40, runner=runner, max_batch=4)
    huge = server.submit(*cloud(), depth=6, tag="huge")
    fine = server.submit(*cloud(), depth=6, tag="fine")
    with pytest.raises(MemoryError):
        huge.result(timeout=10)
    assert fine.result(timeout=10)[0] == "fine"
    server.close()


def test_one_bad_request_fails_alone_inside_a_batch():
    fake = FakeBatchGPU(delay=0.01, fail_tag="bad")
    server = serve.Server(lanes=1, budget_bytes=1 << 40, batch_runner=fake, max_batch=8)
    gate = server.submit(*cloud(), depth=6, tag="gate", sleep=0.2)
    time.sleep(0.05)
    futures = {t: server.submit(*cloud(), depth=6, tag=t) for t in ("a", "bad", "b")}
    gate.result(timeout=10)
    assert futures["a"].result(timeout=10)[0] == "a" and futures["b"].result(timeout=10)[0] == "b"
    with pytest.raises(ValueError):
        futures["bad"].result(timeout=10)
    server.close()


def test_footprint_model_counts_the_solver_levels():
    # level 0 of side 257: six padded FP32 arrays; the model is dominated by the
    # grids and the hierarchy at depth >= 8
    n = 257
    h = serve.hierarchy_bytes(n)
    assert h > 6 * 4 * n ** 3
    assert h < 12 * 4 * n ** 3
    assert serve.footprint_bytes(8, 0) > 4 * 8 * n ** 3 + h


@pytest.mark.gpu
def test_footprint_model_bounds_the_measured_peak():
    """The admission model against torch's peak allocation of one batched
    reconstruction per depth (within -10 % .. +40 %)."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mojo_poissonrecon_b200 import batch, solver32, workloads

    rng = np.random.default_rng(3)
    for depth, count in ((6, 20_000), (7, 50_000), (8, 200_000)):
        p, n = workloads.torus(count, noise=0.0, confidence=None, rng=rng)
        solver32.clear_engines()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        base = torch.cuda.memory_allocated()
        torch.cuda.reset_peak_memory_stats()
        batch.reconstruct_many([(p, n, depth)], tol=1e-8)
        torch.cuda.synchronize()
        peak = torch.cuda.max_memory_allocated() - base
        model = serve.footprint_bytes(depth, count)
        assert 0.9 * peak <= model <= 1.4 * peak, (depth, peak, model)


@pytest.mark.gpu
def test_same_result_alone_and_in_the_mix():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import mojo_poissonrecon_b200 as mpr
    from mojo_poissonrecon_b200 import workloads

    rng = np.random.default_rng(0)
    clouds = []
    for k in range(8):
        size = int(rng.integers(3_000, 60_000))
        depth = int(rng.integers(5, 8))
        if k % 2:
            p, n = workloads.ellipsoid(size, rng)
        else:
            p, n = workloads.torus(size, noise=0.0, confidence=None, rng=rng)
        clouds.append((p, n, depth))
    alone = [mpr.reconstruct(p, n, depth=d, precision="fp32_refined", tol=1e-8) for p, n, d in clouds]
    mixed = serve.reconstruct_batch(clouds, lanes=3)  # batches of whatever is queued
    single = serve.reconstruct_batch(clouds, lanes=3, max_batch=1)  # one reconstruction per lane
    for a, b in zip(alone, single):
        assert np.array_equal(a.vertices, b.vertices) and np.array_equal(a.faces, b.faces)
    for a, b in zip(alone, mixed):
        assert np.array_equal(a.vertices, b.vertices)
        assert np.array_equal(a.faces, b.faces)
        assert a.iso_value == b.iso_value and a.residual_norm == b.residual_norm


def test_on_result_replaces_the_result():
    server = serve.Server(lanes=1, budget_bytes=1 << 40, runner=lambda p, n, **kw: kw["tag"] * 2, max_batch=1,
                          on_result=lambda r: r + 1)
    f = server.submit(*cloud(), depth=6, tag=5)
    assert f.result(timeout=10)[0] == 11
    server.close()


def test_nvtx_stages_push_and_pop(monkeypatch):
    """With tracing on, a stage pushes one NVTX range and pops it, also when
    the stage raises; with tracing off it touches nothing."""
    import torch

    from mojo_poissonrecon_b200 import _trace

    calls = []
    monkeypatch.setattr(torch.cuda.nvtx, "range_push", lambda name: calls.append(("push", name)))
    monkeypatch.setattr(torch.cuda.nvtx, "range_pop", lambda: calls.append(("pop",)))
    monkeypatch.setattr(_trace, "ENABLED", False)
    with _trace.stage("solve"):
        pass
    assert calls == []
    monkeypatch.setattr(_trace, "ENABLED", True)
    with _trace.stage("solve"):
        pass
    try:
        with _trace.stage("extract"):
            raise ValueError("x")
    except ValueError:
        pass
    assert calls == [("push", "mpr:solve"), ("pop",), ("push", "mpr:extract"), ("pop",)]
