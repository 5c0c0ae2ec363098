"""Continuous batching: admission by HBM footprint, overlap of requests that
arrive while others run, and identical results alone and in the mix."""

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
    server = serve.Server(lanes=lanes, budget_bytes=budget, runner=fake)
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

    server = serve.Server(lanes=1, budget_bytes=1 << 40, runner=runner)
    bad = server.submit(np.zeros((1, 3)), np.ones((1, 3)), depth=5, tag="bad")
    good = server.submit(np.zeros((1, 3)), np.ones((1, 3)), depth=5, tag="good")
    with pytest.raises(ValueError):
        bad.result(timeout=10)
    assert good.result(timeout=10)[0] == "good"
    server.close()


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
    mixed = serve.reconstruct_batch(clouds, lanes=3)
    for a, b in zip(alone, mixed):
        assert np.array_equal(a.vertices, b.vertices)
        assert np.array_equal(a.faces, b.faces)
        assert a.iso_value == b.iso_value and a.residual_norm == b.residual_norm
