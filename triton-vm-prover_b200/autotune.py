"""Autotuner for the table-commitment kernels.

Times candidate values of the library's tuning knobs (tvmc_set_tuning) on the
caller's own table shapes, keeps the fastest, and persists the choice in a JSON
cache keyed by device name and shape, so later processes start tuned:

    lde_mid_ctas        resident CTAs/SM of the fused LDE middle kernel (2, 3)
    hash_unfused_tree   1 = build all Merkle levels in the tree kernel (0, 1)
    batch_streams       worker streams of a tvmc_batch (1 .. 16)
    frugal_stripe_cols  columns per frugal stripe (multiples of 10)

Every candidate computes the same bits (the knobs only change scheduling and
register allocation), so tuning never affects results.
"""
from __future__ import annotations

import json
import os
import time

import tvmc

CACHE = os.environ.get("TVMC_TUNING_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "tvmc",
                                                          "tuning.json"))


def _device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name()
    except Exception:
        return "cuda"


def load(path: str = CACHE) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save(db: dict, path: str = CACHE) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(db, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def apply(knobs: dict) -> None:
    for k, v in knobs.items():
        tvmc.set_tuning(k, int(v))


def _time(fn, reps: int = 3) -> float:
    import torch
    fn()  # warm-up (also builds twiddle tables)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - t0)
    return best


def tune_commit(trace_ptr: int, trace_len: int, width: int, expansion: int = 4, offset: int = 7,
                stream=None, path: str = CACHE, force: bool = False) -> dict:
    """Tune the plain commit of one device-resident column-major table."""
    key = f"{_device_name()}|commit|{trace_len}x{width}x{expansion}"
    db = load(path)
    if key in db and not force:
        apply(db[key]["knobs"])
        return db[key]

    def run():
        c = tvmc.Commitment(trace_ptr, width=width, trace_len=trace_len, device_ptr=True,
                            expansion=expansion, offset=offset, stream=stream)
        c.sync()
        c.free()

    results = {}
    for ctas in (2, 3):
        for unfused in (0, 1):
            tvmc.set_tuning("lde_mid_ctas", ctas)
            tvmc.set_tuning("hash_unfused_tree", unfused)
            results[(ctas, unfused)] = _time(run)
    best = min(results, key=results.get)
    entry = {"knobs": {"lde_mid_ctas": best[0], "hash_unfused_tree": best[1]},
             "seconds": {f"{k[0]},{k[1]}": v for k, v in results.items()}}
    apply(entry["knobs"])
    db[key] = entry
    save(db, path)
    return entry


def tune_batch(shapes, fill, path: str = CACHE, force: bool = False, candidates=(1, 2, 4, 8, 16)) -> dict:
    """Tune batch_streams for a tvmc.Batch of `shapes`; fill(batch) loads inputs."""
    key = f"{_device_name()}|batch|" + ",".join(f"{s[0]}x{s[1]}" for s in shapes)
    db = load(path)
    if key in db and not force:
        apply(db[key]["knobs"])
        return db[key]
    results = {}
    for k in candidates:
        tvmc.set_tuning("batch_streams", k)
        with tvmc.Batch(shapes) as b:
            fill(b)
            results[k] = _time(b.run)
    best = min(results, key=results.get)
    entry = {"knobs": {"batch_streams": best}, "seconds": {str(k): v for k, v in results.items()}}
    apply(entry["knobs"])
    db[key] = entry
    save(db, path)
    return entry


def tune_frugal(trace_ptr: int, trace_len: int, width: int, expansion: int = 4, offset: int = 7,
                path: str = CACHE, force: bool = False, candidates=(10, 20, 40, 80)) -> dict:
    key = f"{_device_name()}|frugal|{trace_len}x{width}x{expansion}"
    db = load(path)
    if key in db and not force:
        apply(db[key]["knobs"])
        return db[key]
    results = {}
    for sc in candidates:
        tvmc.set_tuning("frugal_stripe_cols", sc)

        def run():
            with tvmc.Commitment(trace_ptr, width=width, trace_len=trace_len, device_ptr=True,
                                 expansion=expansion, offset=offset, frugal=True) as c:
                c.sync()

        results[sc] = _time(run, reps=2)
    best = min(results, key=results.get)
    entry = {"knobs": {"frugal_stripe_cols": best}, "seconds": {str(k): v for k, v in results.items()}}
    apply(entry["knobs"])
    db[key] = entry
    save(db, path)
    return entry
