"""Autotuner for the launch shapes of the refined solver's level-0 kernels.

The reference fixes its launch shape at build time (GRID_Z_CHUNK = 4 and
PARALLEL_GRID_THRESHOLD, src/capi.mojo:9-10).  Here the library keeps a table
of launch parameters per grid side (pb_tune_set, include/poisson_b200.h) that
its launchers consult; this module fills it by measurement:

* for each parameter and side it times every candidate value with CUDA events
  (the median of `repeats` launches after warm-up launches) on synthetic
  buffers of that side, and keeps the fastest;
* results are cached in a JSON file keyed by the GPU's name and the side
  (MPR_B200_TUNE_CACHE, default ~/.cache/mojo_poissonrecon_b200/tune.json),
  so a process applies the stored choice without measuring again.

Parameters searched (PB_TUNE_*): the TMA sweep's planes per block (z chunk),
the level-0 residual-restriction's coarse planes per block, the
prolongation's fine planes per block, and which compiled variant each FCG
pass runs (register budgets; cp.async prefetching for pass 2) and the sweep
(shared-ring depth with its resident blocks per SM).  These change
launch shapes only, never results: every node's arithmetic and every
reduction's order stay the same.
"""

from __future__ import annotations

import json
import os
import statistics
import threading

(SWEEP_Z_CHUNK, RESTRICT_PLANES, PROLONG_PLANES, FCG_DIRECTION_PLANES, FCG_UPDATE_PLANES, FCG_DIRECTION_VARIANT,
 FCG_UPDATE_VARIANT, SWEEP_VARIANT, RESTRICT_VARIANT, RELAX27_VARIANT, RESIDUAL27_VARIANT) = range(11)
NAMES = {SWEEP_Z_CHUNK: "sweep_z_chunk", RESTRICT_PLANES: "restrict_planes", PROLONG_PLANES: "prolong_planes",
         FCG_DIRECTION_PLANES: "fcg_direction_planes", FCG_UPDATE_PLANES: "fcg_update_planes",
         FCG_DIRECTION_VARIANT: "fcg_direction_variant", FCG_UPDATE_VARIANT: "fcg_update_variant",
         SWEEP_VARIANT: "sweep_variant", RESTRICT_VARIANT: "restrict_variant",
         RELAX27_VARIANT: "relax27_variant", RESIDUAL27_VARIANT: "residual27_variant"}
# Searched by autotune(): the parameters that never change results.  The FCG
# passes' planes per block also set the shape of their partial-sum trees, so a
# different value changes the inner products (and the iterates) by rounding;
# they stay at the built-in 24 unless set explicitly.
# The sweep's variant comes first: the z chunk is then searched for the variant chosen.
SEARCHED = (SWEEP_VARIANT, SWEEP_Z_CHUNK, RESTRICT_VARIANT, RESTRICT_PLANES, PROLONG_PLANES, FCG_DIRECTION_VARIANT,
            FCG_UPDATE_VARIANT, RELAX27_VARIANT, RESIDUAL27_VARIANT)
# Searched per packed level side of the hierarchy (not per the top side).
PER_LEVEL = (RELAX27_VARIANT, RESIDUAL27_VARIANT)
_LOCK = threading.Lock()


def cache_path() -> str:
    return os.environ.get("MPR_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "mojo_poissonrecon_b200", "tune.json"))


def candidates(param: int, n: int) -> list[int]:
    """Values tried for `param` at side n (0 = the launcher's built-in choice)."""
    if param == SWEEP_Z_CHUNK:
        vals = {0}
        for chunks in range(1, 17):
            zc = -(-n // chunks)
            if zc >= 4:
                vals.add(zc)
        return sorted(vals)
    if param == RESTRICT_PLANES:
        cn = (n + 1) // 2
        return [0] + [v for v in (1, 2, 3, 4, 6, 8, 12, 16) if v <= cn]
    if param == PROLONG_PLANES:
        return [0] + [v for v in (1, 2, 4, 8, 16, 32) if v <= n]
    if param in (FCG_DIRECTION_PLANES, FCG_UPDATE_PLANES):
        return [0] + [v for v in (8, 12, 16, 24, 32, 48, 64) if v <= max(n, 8)]
    if param == FCG_DIRECTION_VARIANT:
        return [0, 1, 2]
    if param == FCG_UPDATE_VARIANT:
        return [0, 1, 2, 3, 4]
    if param == SWEEP_VARIANT:
        return list(range(9))
    if param == RESTRICT_VARIANT:
        return [0, 1, 2, 3]
    if param in (RELAX27_VARIANT, RESIDUAL27_VARIANT):
        return [0, 1]
    raise ValueError(f"unknown tuning parameter {param}")


def search(param: int, n: int, time_one, repeats: int = 10, warmup: int = 2) -> tuple[int, dict]:
    """Time every candidate with time_one(value) -> seconds (called warmup +
    repeats times per candidate) and return (best value, {value: median s}).
    Ties go to the built-in choice (0), then to the smaller value."""
    timings = {}
    for value in candidates(param, n):
        for _ in range(warmup):
            time_one(value)
        timings[value] = statistics.median(time_one(value) for _ in range(repeats))
    best = min(timings, key=lambda v: (timings[v], v != 0, v))
    return best, timings


def load_cache(path: str | None = None) -> dict:
    path = cache_path() if path is None else path
    try:
        with open(path, encoding="utf8") as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def store_cache(entries: dict, path: str | None = None) -> None:
    path = cache_path() if path is None else path
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + f".{os.getpid()}.tmp"
    with open(tmp, "w", encoding="utf8") as f:
        json.dump(entries, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def cache_key(gpu: str, n: int) -> str:
    return f"{gpu}|n={n}"


def apply(lib, gpu: str, n: int, path: str | None = None) -> dict:
    """Load the cached choices for (gpu, n) into the library's table; returns them."""
    entry = load_cache(path).get(cache_key(gpu, n), {})
    chosen = {}
    for param, name in NAMES.items():
        value = int(entry.get(name, {}).get("best", 0))
        if value:
            lib.pb_tune_set(param, n, value)
            chosen[name] = value
    return chosen


def gpu_name(device=None) -> str:
    import torch

    return torch.cuda.get_device_name(device)


def autotune(n: int, device=None, repeats: int = 10, params=None, path: str | None = None,
             write: bool = True) -> dict:
    """Measure every parameter's candidates at side n on `device`, set the
    winners in the library's table and (write=True) store them in the cache.
    Returns {name: {"best": value, "default_s": s, "best_s": s, "timings": {...}}}."""
    import torch

    from . import _native as nat
    from .solver32 import Hierarchy32

    lib = nat.lib()
    dev = nat.require_cuda() if device is None else device
    params = list(SEARCHED) if params is None else list(params)
    gen = torch.Generator(device=dev).manual_seed(1234)
    h = Hierarchy32(n, dev)
    l0, l1 = h.levels[0], h.levels[1]
    if not l0.seven:
        raise ValueError(f"autotuning needs a level 0 on the TMA sweep (side >= 33, got {n})")
    for t in (l0.invD, l0.rhs, l0.ea, l0.eb, l0.D, l0.weights, l1.ea):
        t.uniform_(0.0, 1.0, generator=gen)
    f64 = lambda: torch.rand((n, n, n), dtype=torch.float64, device=dev, generator=gen)
    f32 = lambda: torch.rand((n, n, n), dtype=torch.float32, device=dev, generator=gen)
    x0, x1, b, screen = f64(), f64(), f64(), f64()
    p0, p1 = f32(), f32()
    scal = torch.tensor([1.0, 0.5, 0.25, 0.0, 0.0, 0, 0, 0], dtype=torch.float64, device=dev)
    flags = torch.tensor([0, 0, 1, 0], dtype=torch.int32, device=dev)
    ws = nat.Workspace(dev)
    ws_ptr, ws_size = ws.get(lib.pb_fcg_workspace_size(n))
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    s = stream.cuda_stream

    def launch(param):
        if param in (SWEEP_Z_CHUNK, SWEEP_VARIANT):
            return lambda: nat.check(lib.pb_sweep_tma_f32(l0.ea.data_ptr(), l0.eb.data_ptr(), l0.rhs.data_ptr(),
                                                          l0.invD.data_ptr(), n, 0, 0, status.data_ptr(), s), "sweep")
        if param in (RESTRICT_PLANES, RESTRICT_VARIANT):
            args = (l0.ea.data_ptr(), l0.rhs.data_ptr(), l0.D.data_ptr(), l0.weights.data_ptr(), l1.rhs.data_ptr(), n)

            def restrict():  # as the FP32 cycle chooses (Hierarchy32.v_cycle)
                if lib.pb_tune_get(RESTRICT_VARIANT, n) == 2:
                    nat.check(lib.pb_residual_restrict_tma_f32(*args, status.data_ptr(), s), "restrict")
                else:
                    nat.check(lib.pb_residual_restrict_f32(*args, s), "restrict")
            return restrict
        if param == PROLONG_PLANES:
            return lambda: nat.check(lib.pb_prolong_fac_f32(l1.ea.data_ptr(), l0.eb.data_ptr(),
                                                            l0.weights.data_ptr(), n, s), "prolong")
        if param in (FCG_DIRECTION_PLANES, FCG_DIRECTION_VARIANT):
            return lambda: nat.check(lib.pb_fcg_direction_f64(l0.ea.data_ptr(), p0.data_ptr(), p1.data_ptr(),
                                                              l0.rhs.data_ptr(), screen.data_ptr(), n, 4.0,
                                                              scal.data_ptr(), flags.data_ptr(), ws_ptr, ws_size, s),
                                     "fcg direction")
        return lambda: nat.check(lib.pb_fcg_update_f64(l0.ea.data_ptr(), p0.data_ptr(), p1.data_ptr(),
                                                       x0.data_ptr(), x1.data_ptr(), b.data_ptr(), screen.data_ptr(),
                                                       l0.rhs.data_ptr(), n, 4.0, scal.data_ptr(), flags.data_ptr(),
                                                       ws_ptr, ws_size, s), "fcg update")

    def level_launch(param, lv, nxt):  # one packed sweep or residual-restriction on level lv
        if param == RELAX27_VARIANT:
            return lambda: nat.check(lib.pb_relax27p_f32(lv.ea.data_ptr(), lv.eb.data_ptr(), lv.rhs.data_ptr(),
                                                         *lv.packed_ptrs(), lv.n, s), "relax27p")
        return lambda: nat.check(lib.pb_residual_restrict27p_f32(lv.ea.data_ptr(), lv.rhs.data_ptr(),
                                                                 *lv.packed_ptrs(), lv.weights.data_ptr(), lv.n,
                                                                 lv.res.data_ptr(), nxt.rhs.data_ptr(), s),
                                 "residual_restrict27p")

    jobs = []  # (param, side, launch, result name)
    for param in params:
        if param in PER_LEVEL:
            for lv, nxt in zip(h.levels[:-1], h.levels[1:]):
                if lv.packed is not None:
                    for t in (lv.ea, lv.rhs):
                        t.uniform_(0.0, 1.0, generator=gen)
                    jobs.append((param, lv.n, level_launch(param, lv, nxt), f"{NAMES[param]}@{lv.n}"))
        else:
            jobs.append((param, n, launch(param), NAMES[param]))
    result = {}
    with _LOCK:
        for param, side, fn, name in jobs:

            def time_one(value, fn=fn, param=param, side=side):
                nat.check(lib.pb_tune_set(param, side, value), "tune set")
                a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                fn()
                fn()
                e.record(stream)
                e.synchronize()
                return a.elapsed_time(e) / 2e3

            best, timings = search(param, side, time_one, repeats=repeats)
            nat.check(lib.pb_tune_set(param, side, best), "tune set")
            result[name] = {"best": best, "default_s": timings[0], "best_s": timings[best], "side": side,
                            "timings": {str(k): v for k, v in sorted(timings.items())}}
        if status.item():
            raise RuntimeError("autotune: a bounded TMA wait gave up during the measurement")
        if write:
            entries = load_cache(path)
            gpu = gpu_name(dev)
            for name, v in result.items():
                key = cache_key(gpu, v["side"])
                entries.setdefault(key, {})[name.split("@")[0]] = {"best": v["best"], "best_s": v["best_s"],
                                                                   "default_s": v["default_s"]}
            store_cache(entries, path)
    return result


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description="measure and cache launch parameters per grid side")
    ap.add_argument("--sides", type=int, nargs="+", default=[129, 257, 513])
    ap.add_argument("--repeats", type=int, default=10)
    args = ap.parse_args()
    for side in args.sides:
        print(side, json.dumps({k: (v["best"], round(v["default_s"] * 1e6, 1), round(v["best_s"] * 1e6, 1))
                                for k, v in autotune(side, repeats=args.repeats).items()}))
