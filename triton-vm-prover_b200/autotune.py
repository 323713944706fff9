"""Autotuner for the table-commitment kernels.

Times candidate values of the library's tuning knobs (tvmc_set_tuning) on the
caller's own table shapes, keeps the fastest, and persists the choice in a JSON
cache keyed by device name and shape, so later processes start tuned:

    lde_mid_variant     fused LDE middle kernel: per-coset global twiddles (1) or
                        inter-pass twiddles shared across cosets in shared memory (2)
    lde_mid_ctas        its resident CTAs/SM (2, 3)
    lde_split_l1        the LDE's four-step split N = n1 * n2 (balanced, or n1 = N^(1/2) / 4,
                        or n1 = 2^12 where valid)
    ntt_tile_log        words an NTT pass CTA moves per tile (2^12 .. 2^14)
    hash_unfused_tree   1 = build all Merkle levels in the tree kernel (0, 1)
    batch_streams       worker streams of a tvmc_batch (1 .. 16)
    batch_multi_hash    one multi-table row-hash launch for a batch (1) or per-table hashes (2)
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


def lde_candidates(log_n: int):
    """The LDE knob combinations worth timing for a trace of 2^log_n rows."""
    splits = [0] + [l1 for l1 in (log_n // 2 - 2, 12) if 6 <= l1 <= 12 and 6 <= log_n - l1 <= 12
                    and l1 != (log_n + 1) // 2]
    return [{"lde_mid_variant": v, "lde_mid_ctas": c, "lde_split_l1": s, "ntt_tile_log": t}
            for v in (1, 2) for c in (2, 3) for s in splits for t in (12, 13, 14)]


def tune_commit(trace_ptr: int, trace_len: int, width: int, expansion: int = 4, offset: int = 7,
                stream=None, path: str = CACHE, force: bool = False) -> dict:
    """Tune the plain commit of one device-resident column-major table: first
    the LDE knobs on the LDE alone (up to 64 of its columns), then the tree
    fusion on whole commits."""
    import torch
    key = f"{_device_name()}|commit|{trace_len}x{width}x{expansion}"
    db = load(path)
    if key in db and not force:
        apply(db[key]["knobs"])
        return db[key]
    log_n = trace_len.bit_length() - 1
    cols = max(1, min(width, 64))
    out = torch.empty(cols * trace_len * expansion, dtype=torch.int64, device="cuda")
    lde_s = {}
    for knobs in lde_candidates(log_n):
        apply(knobs)
        lde_s[tuple(knobs.values())] = _time(
            lambda: tvmc.lde_gpu(trace_ptr, cols, trace_len, out.data_ptr(), trace_len * expansion, offset,
                                 stream=stream))
    del out
    best_lde = dict(zip(("lde_mid_variant", "lde_mid_ctas", "lde_split_l1", "ntt_tile_log"),
                        min(lde_s, key=lde_s.get)))
    apply(best_lde)

    def run():
        c = tvmc.Commitment(trace_ptr, width=width, trace_len=trace_len, device_ptr=True,
                            expansion=expansion, offset=offset, stream=stream)
        c.sync()
        c.free()

    hash_s = {}
    for unfused in (0, 1):
        tvmc.set_tuning("hash_unfused_tree", unfused)
        hash_s[unfused] = _time(run)
    best_unfused = min(hash_s, key=hash_s.get)
    entry = {"knobs": dict(best_lde, hash_unfused_tree=best_unfused),
             "seconds": {"lde": {",".join(map(str, k)): v for k, v in lde_s.items()},
                         "commit_by_unfused_tree": {str(k): v for k, v in hash_s.items()}}}
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
    for multi in (1, 2):
        for k in candidates:
            tvmc.set_tuning("batch_streams", k)
            tvmc.set_tuning("batch_multi_hash", multi)
            with tvmc.Batch(shapes) as b:
                fill(b)
                results[(multi, k)] = _time(b.run)
    best = min(results, key=results.get)
    entry = {"knobs": {"batch_multi_hash": best[0], "batch_streams": best[1]},
             "seconds": {f"{m},{k}": v for (m, k), v in results.items()}}
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
