"""The autotuner's search and cache (tune.py) with a fake timer, and the
library's tuning table (pb_tune_set/get), all without a GPU."""

import pytest

from mojo_poissonrecon_b200 import tune


def test_candidates_cover_the_built_in_choice_and_stay_in_range():
    for param in tune.NAMES:
        for n in (33, 65, 257, 513):
            vals = tune.candidates(param, n)
            assert vals[0] == 0 and len(vals) == len(set(vals)) >= 2
            assert all(0 <= v <= max(n, 64) for v in vals)
    assert all(v >= 4 or v == 0 for v in tune.candidates(tune.SWEEP_Z_CHUNK, 257))
    assert min(v for v in tune.candidates(tune.FCG_UPDATE_PLANES, 257) if v) >= 8


def test_search_picks_the_fastest_with_a_fake_timer():
    calls = []
    cost = {0: 5.0, 8: 3.0, 12: 2.0, 16: 2.5, 24: 4.0, 32: 6.0, 48: 7.0, 64: 9.0}

    def time_one(value):
        calls.append(value)
        return cost[value]

    best, timings = tune.search(tune.FCG_UPDATE_PLANES, 257, time_one, repeats=3, warmup=1)
    assert best == 12 and timings[12] == 2.0
    assert len(calls) == 4 * len(cost)  # warm-up + repeats per candidate


def test_search_prefers_the_built_in_choice_on_ties():
    best, _ = tune.search(tune.RESTRICT_PLANES, 129, lambda v: 1.0, repeats=2, warmup=0)
    assert best == 0


def test_cache_round_trip_and_apply(tmp_path):
    from mojo_poissonrecon_b200 import _native

    lib = _native.lib()
    path = str(tmp_path / "tune.json")
    assert tune.load_cache(path) == {}
    tune.store_cache({tune.cache_key("GPU X", 257): {"sweep_z_chunk": {"best": 29},
                                                      "fcg_update_planes": {"best": 16},
                                                      "restrict_planes": {"best": 0}}}, path)
    lib.pb_tune_clear()
    try:
        chosen = tune.apply(lib, "GPU X", 257, path)
        assert chosen == {"sweep_z_chunk": 29, "fcg_update_planes": 16}
        assert lib.pb_tune_get(tune.SWEEP_Z_CHUNK, 257) == 29
        assert lib.pb_tune_get(tune.FCG_UPDATE_PLANES, 257) == 16
        assert lib.pb_tune_get(tune.RESTRICT_PLANES, 257) == 0
        assert tune.apply(lib, "GPU Y", 257, path) == {}  # keyed by GPU
        assert lib.pb_tune_set(tune.SWEEP_Z_CHUNK, 257, 0) == 0  # 0 clears
        assert lib.pb_tune_get(tune.SWEEP_Z_CHUNK, 257) == 0
    finally:
        lib.pb_tune_clear()


@pytest.mark.parametrize("args", [(11, 257, 4), (-1, 257, 4), (0, 1, 4), (0, 257, -2), (0, 257, 5000)])
def test_tune_table_rejects_bad_entries(args):
    from mojo_poissonrecon_b200 import _native

    lib = _native.lib()
    assert lib.pb_tune_set(*args) == 1


def test_grouped_fcg_launches_keep_the_built_in_planes():
    """Grouped (batched) FCG launches use 24 planes per block whatever the
    table says, so a batch's inner products have the single path's default
    partial-sum trees; the partial-sum capacity covers the shallowest choice."""
    from mojo_poissonrecon_b200 import _native

    lib = _native.lib()
    lib.pb_tune_clear()
    try:
        assert lib.pb_batch_fcg_blocks(257, 1) == 9 * 33 * 11  # 24 planes
        lib.pb_tune_set(tune.FCG_UPDATE_PLANES, 257, 8)
        assert lib.pb_batch_fcg_blocks(257, 1) == 9 * 33 * 11
        assert lib.pb_batch_fcg_partials(257) >= 9 * 33 * 33  # the 8-plane single-path grid fits too
    finally:
        lib.pb_tune_clear()
