"""Benchmark of the table-commitment path on B200.

Workload (one step): commit the main table (2^20 rows x 379 base columns) and
the aux table (2^20 rows x 88 XFieldElement columns = 264 base limbs), each
extended x4 onto the coset 7*<w_{2^22}> (LDE), Tip5-hashed row by row, and
Merkle-committed -- two separate trees, as the prover commits main and aux.
Entries are uniform random field elements (synthetic; the reference publishes
no dataset for this path).

Printed JSON (rank 0): `value` = committed LDE cells/s with the traces already
in HBM (device-timed with CUDA events); `e2e` = the same through the public
C ABI from pinned host buffers (upload inside the timed region, roots read
back); `roofline` = the dominant kernel (Tip5 row hash + tree) against the SM
instruction-issue limit (SMs x 4 schedulers x 32 lanes x the SM clock sampled
during the timed region); `roofline_lde` = the LDE kernels against HBM;
`roofline_commit` = the whole step against the slower of its HBM bytes at the
measured copy bandwidth and its integer ops (Tip5 + NTT cost model) at the
issue limit; `cpu_baseline` = the reference's own CPU code (oracle/_ref) on a
bounded sample on this host's cores, extrapolated to the workload.

`--impl reference` times the reference's own CPU code (oracle/_ref, OpenMP on
every host core) on one full step of the same workload, plus the as-shipped
serial figure (one thread) on the 2^10 x 379 commit.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Further workloads (one JSON line each, one GPU):
    --workload batch     32 tables, heights 2^12..2^18 log-uniform by seed, widths
                         379 / 264 limbs 50/50, one graph-captured batch launch
                         (worker streams autotuned) vs committing each alone
    --workload frugal    2^22 x 379, x4 -> 2^24-row LDE streamed in 10-column
                         stripes (stripe width autotuned) vs the materialised commit
    --workload serving   Poisson arrivals of requests with heights 2^10..2^20
                         log-uniform and widths 379 / 264, 80 openings each, at swept
                         rates: p50/p99 latency and throughput of the serving loop
                         vs the plain per-request drop-in
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "triton-vm-prover_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

P = 0xFFFFFFFF00000001
LOG_N = 20
W_MAIN, W_AUX = 379, 264
EXPANSION = 4
OFFSET = 7
METRIC = "committed LDE cells/s"
# Tip5 integer-op cost model (32-bit ops): Goldilocks mul 16, add 4; one
# permutation = 5 x (12 x^7 @ 4 muls + 4 split-and-lookup @ 48 + MDS @ 640 + 16 RC adds @ 4).
OPS_PER_PERM = 5 * (12 * 4 * 16 + 4 * 48 + 640 + 16 * 4)
# NTT cost model: 24 int32 ops per butterfly or scale.
OPS_PER_NTT_MUL = 24
# Instruction issue of one SM per clock: 4 schedulers x 32 lanes.
ISSUE_LANES_PER_SM = 4 * 32


def perms_per_table(L: int, width: int) -> int:
    return L * (width // 10 + 1) + (L - 1)


def ntt_ops_per_table(n: int, width: int, expansion: int = EXPANSION) -> int:
    """Cost-model int32 ops of one table's LDE: per column an n-point inverse
    NTT, n coset scales and an (expansion*n)-point forward NTT."""
    L = expansion * n
    ln, lL = n.bit_length() - 1, L.bit_length() - 1
    return width * ((n // 2) * ln + n + (L // 2) * lL) * OPS_PER_NTT_MUL


def bytes_per_table(n: int, width: int, expansion: int = EXPANSION) -> int:
    """Algorithmic bytes of one commit: trace read, LDE written, leaf digests,
    internal nodes."""
    L = expansion * n
    return 8 * n * width + 8 * L * width + 40 * L + 40 * (L - 1)


def issue_limit_tops(sms: int, sm_mhz: float) -> float:
    """Thread-instructions per second the SMs can issue (T/s)."""
    return sms * ISSUE_LANES_PER_SM * sm_mhz * 1e6 / 1e12


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def max_over_ranks(x: float, device=None) -> float:
    """The maximum of x over all ranks (the job's time is its slowest rank's);
    x itself when not distributed.  device: where the collective's tensor lives
    (a CUDA device under NCCL, None = CPU under gloo)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, ranks: int, seconds_max: float) -> float:
    """Replicas (weak scaling): every rank processes units_per_rank; the job
    takes the slowest rank's time."""
    return ranks * units_per_rank / seconds_max


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.rows = []
        if self.proc is None:
            return
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.rows.append(f)

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def random_trace(torch, width, n, seed, dev):
    g = torch.Generator(device=dev).manual_seed(seed)
    hi = torch.randint(0, 2**32, (width, n), dtype=torch.int64, device=dev, generator=g)
    lo = torch.randint(0, 2**32, (width, n), dtype=torch.int64, device=dev, generator=g)
    x = (hi << 32) | lo
    # map the 2^32 - 1 values >= p onto [0, p): x - p == x + (2^32 - 1) mod 2^64
    ge = (hi == 0xFFFFFFFF) & (lo > 0)
    return torch.where(ge, x + 0xFFFFFFFF, x)


def cpu_reference_sample(log_n: int, threads: int | None = None):
    """Time the reference's CPU path (oracle/_ref) on a bounded sample and
    extrapolate to the full workload. Returns (cells_per_s, detail)."""
    from oracle import RefLib
    r = RefLib()
    if threads:
        r.set_threads(threads)
    cores = r.max_threads()
    n = 1 << log_n
    L = EXPANSION * n
    rng = np.random.default_rng(1)
    # LDE: `cores` full columns in parallel (OpenMP over columns)
    ncol = max(1, min(cores, 64))
    t = rng.integers(0, P, (ncol, n), dtype=np.uint64)
    t0 = time.perf_counter()
    lde = r.lde(t, EXPANSION, OFFSET)
    t_lde = time.perf_counter() - t0
    lde_total = t_lde * (W_MAIN + W_AUX) / ncol
    # row hashing: rows of width 379 and 264 (OpenMP over rows)
    rows = max(1024, min(L, 64 * cores))
    h_main = rng.integers(0, P, (W_MAIN, rows), dtype=np.uint64)
    t0 = time.perf_counter()
    r.hash_rows_cm(h_main)
    t_hm = time.perf_counter() - t0
    h_aux = rng.integers(0, P, (W_AUX, rows), dtype=np.uint64)
    t0 = time.perf_counter()
    r.hash_rows_cm(h_aux)
    t_ha = time.perf_counter() - t0
    hash_total = (t_hm + t_ha) * L / rows
    # Merkle tree (OpenMP per level inside MerkleTree)
    nl = min(L, 1 << 15)
    lv = rng.integers(0, P, (nl, 5), dtype=np.uint64)
    t0 = time.perf_counter()
    r.merkle(lv)
    t_m = time.perf_counter() - t0
    merkle_total = 2 * t_m * L / nl
    total = lde_total + hash_total + merkle_total
    cells = L * (W_MAIN + W_AUX)
    sample = (f"reference CPU code (oracle/_ref, OpenMP): LDE of {ncol} columns 2^{log_n}->2^{log_n + 2}, "
              f"Tip5 hash of {rows} rows x 379 and x 264, Merkle of {nl} leaves; extrapolated linearly to "
              f"2^{log_n + 2} rows x (379 + 264) columns (an estimate; --impl reference times a full step)")
    detail = {"lde_s": lde_total, "hash_s": hash_total, "merkle_s": merkle_total, "sample_s": t_lde + t_hm + t_ha +
              t_m, "est_commit_s": total}
    del lde
    return cells / total, cores, sample, detail


def host_mem_available() -> int:
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def run_reference(args):
    """The reference's own CPU path (oracle/_ref: LDE::extend_column per
    column, Tip5::hash_varlen per row, MerkleTree) on every host core.  The
    timed step is one full commit of the workload (main and aux tables, two
    trees); with W >= 1 warm-up steps of the 2^10 x 379 commit first.  A full
    CPU step takes minutes, so `--steps` is capped by --ref-max-seconds: the
    line reports the steps actually timed.  The sample extrapolation
    (cpu_reference_sample) runs first as a cross-check and as the fallback when
    the host lacks the memory or time for a full step."""
    ws, rank, _ = dist_info()
    if rank != 0:
        return
    from oracle import RefLib
    r = RefLib()
    cores = r.max_threads()
    n = 1 << args.log_n
    L = EXPANSION * n
    cells = L * (W_MAIN + W_AUX)
    rng = np.random.default_rng(0x7E5EED01)
    small = rng.integers(0, P, (W_MAIN, 1 << 10), dtype=np.uint64)
    for _ in range(args.warmup):
        r.commit(small, EXPANSION, OFFSET)
    # as-shipped serial figure: the 2^10 x 379 commit on one thread
    r.set_threads(1)
    t0 = time.perf_counter()
    r.commit(small, EXPANSION, OFFSET)
    serial_s = time.perf_counter() - t0
    r.set_threads(cores)
    est_v, _, est_sample, est_detail = cpu_reference_sample(args.log_n)
    est_s = est_detail["est_commit_s"]
    need = 8 * n * (W_MAIN + W_AUX) + 8 * L * max(W_MAIN, W_AUX) + 2 * (8 << 30)
    full = host_mem_available() >= need and est_s <= args.ref_max_seconds
    times = []
    if full:
        main_t = rng.integers(0, P, (W_MAIN, n), dtype=np.uint64)
        aux_t = rng.integers(0, P, (W_AUX, n), dtype=np.uint64)
        buf = np.empty(L * max(W_MAIN, W_AUX), dtype=np.uint64)
        budget = args.ref_max_seconds
        spent = 0.0
        while len(times) < max(1, args.steps) and spent + (times[-1] if times else est_s) <= budget:
            t0 = time.perf_counter()
            r.commit(main_t, EXPANSION, OFFSET, lde_buf=buf)
            r.commit(aux_t, EXPANSION, OFFSET, lde_buf=buf)
            times.append(time.perf_counter() - t0)
            spent += times[-1]
        del buf, main_t, aux_t
    if times:
        step_s = statistics.median(times)
        value = cells / step_s
        sample = (f"full steps timed: main 2^{args.log_n}x{W_MAIN} + aux 2^{args.log_n}x{W_AUX} limbs committed "
                  f"by the reference's CPU code (oracle/_ref, OpenMP over columns and rows, {cores} threads)")
    else:
        step_s = est_s
        value = est_v
        sample = est_sample + (" [fallback: host memory or the time cap does not allow a full step]")
    line = {"metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": args.gpus, "steps": len(times) or 0,
            "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * step_s,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64 (Goldilocks)",
            "data": "synthetic uniform field elements", "impl": "reference",
            "timed": "full step" if times else "extrapolated sample",
            "config": {"workload": f"main 2^{args.log_n}x{W_MAIN} + aux 2^{args.log_n}x{W_AUX} limbs, x4 LDE (offset 7), "
                                   "Tip5 row hash, Merkle (two trees)", "trace_len": n, "lde_len": L,
                       "widths": [W_MAIN, W_AUX], "expansion": EXPANSION, "cells_per_step": cells,
                       "parallelism": "cpu"},
            "cpu_baseline": {"value": value, "unit": "cells/s", "cores": cores, "kind": "reference",
                             "sample": sample, "cpu_model": cpu_model(),
                             "step_seconds": times,
                             "sample_estimate": {"value": est_v, "est_step_s": est_s, "sample": est_sample},
                             "serial_2p10x379": {"seconds": serial_s, "cells_per_s": (4 << 10) * W_MAIN / serial_s,
                                                 "threads": 1,
                                                 "what": "as-shipped serial path: LDE::extend_column per column, "
                                                         "Tip5::hash_varlen per row, MerkleTree, one thread"}},
            "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference_gpu(args):
    """The reference's own CUDA kernels for this path (oracle/_ref/libtvm_ref_gpu.so,
    compiled unchanged for sm_100a) on the same workload and GPU: batched
    randomized LDE with no randomizers (the plain LDE), hash_bfield_rows_gpu /
    hash_xfield_rows_gpu and merkle_tree_gpu, traces resident in HBM, each
    stage timed with CUDA events on the launching stream.  A 2^10 x 379 commit
    through the same kernels is checked against the oracle's root first."""
    import ctypes
    import torch
    from oracle import HERE as ORACLE_DIR, Oracle
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    path = os.path.join(ORACLE_DIR, "_ref", "libtvm_ref_gpu.so")
    if not os.path.exists(path):
        print(json.dumps({"impl": "reference", "workload": "reference GPU kernels",
                          "unavailable": f"{path} not built (make -C oracle refgpu needs the reference tree)"}))
        return
    R = ctypes.CDLL(path)
    vp, sz = ctypes.c_void_p, ctypes.c_size_t
    R.tvmrg_lde.argtypes = [vp, sz, sz, vp, sz, ctypes.c_uint64, vp, vp]
    R.tvmrg_hash_bfield_rows.argtypes = [vp, sz, sz, vp, vp]
    R.tvmrg_hash_xfield_rows.argtypes = [vp, sz, sz, vp, vp]
    R.tvmrg_merkle_tree.argtypes = [vp, vp, sz, vp]
    stream = torch.cuda.Stream(dev)
    sp = stream.cuda_stream

    def ck(rc, what):
        if rc != 0:
            raise RuntimeError(f"reference {what}: CUDA error {rc}")

    def commit(trace, w, n, lde, scratch, dig, tree, xfe):
        L = EXPANSION * n
        ck(R.tvmrg_lde(trace.data_ptr(), w, n, lde.data_ptr(), L, OFFSET, scratch.data_ptr(), sp), "LDE")
        if xfe:
            ck(R.tvmrg_hash_xfield_rows(lde.data_ptr(), L, w // 3, dig.data_ptr(), sp), "row hash")
        else:
            ck(R.tvmrg_hash_bfield_rows(lde.data_ptr(), L, w, dig.data_ptr(), sp), "row hash")
        ck(R.tvmrg_merkle_tree(dig.data_ptr(), tree.data_ptr(), L, sp), "Merkle")

    # parity: the 2^10 x 379 commit against the oracle
    o = Oracle()
    small = np.random.default_rng(0x7E5EED01).integers(0, P, (W_MAIN, 1 << 10), dtype=np.uint64)
    n1, L1 = 1 << 10, EXPANSION << 10
    t1 = torch.from_numpy(small.view(np.int64)).to(dev)
    lde1 = torch.empty(W_MAIN * L1, dtype=torch.int64, device=dev)
    s1 = torch.empty(W_MAIN * n1, dtype=torch.int64, device=dev)
    d1 = torch.empty(L1 * 5, dtype=torch.int64, device=dev)
    tr1 = torch.empty((2 * L1 - 1) * 5, dtype=torch.int64, device=dev)
    with torch.cuda.stream(stream):
        commit(t1, W_MAIN, n1, lde1, s1, d1, tr1, False)
    stream.synchronize()
    exp_lde = o.lde(small)
    got_lde = lde1.cpu().numpy().view(np.uint64).reshape(W_MAIN, L1) % P
    exp_root = o.merkle(o.hash_rows_cm(exp_lde))[1]
    got_root = tr1.cpu().numpy().view(np.uint64).reshape(-1, 5)[-1] % P
    parity = {"lde_equal": bool((got_lde == exp_lde).all()), "root_equal": bool((got_root == exp_root).all())}
    del t1, lde1, s1, d1, tr1

    n = 1 << args.log_n
    L = EXPANSION * n
    main = random_trace(torch, W_MAIN, n, 1000, dev)
    aux = random_trace(torch, W_AUX, n, 2000, dev)
    lde = torch.empty(max(W_MAIN, W_AUX) * L, dtype=torch.int64, device=dev)
    scratch = torch.empty(max(W_MAIN, W_AUX) * n, dtype=torch.int64, device=dev)
    dig = torch.empty(L * 5, dtype=torch.int64, device=dev)
    tree = torch.empty((2 * L - 1) * 5, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()

    def step(times=None):
        for name, t, w, xfe in (("main", main, W_MAIN, False), ("aux", aux, W_AUX, True)):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            ev[0].record(stream)
            ck(R.tvmrg_lde(t.data_ptr(), w, n, lde.data_ptr(), L, OFFSET, scratch.data_ptr(), sp), "LDE")
            ev[1].record(stream)
            if xfe:
                ck(R.tvmrg_hash_xfield_rows(lde.data_ptr(), L, w // 3, dig.data_ptr(), sp), "row hash")
            else:
                ck(R.tvmrg_hash_bfield_rows(lde.data_ptr(), L, w, dig.data_ptr(), sp), "row hash")
            ev[2].record(stream)
            ck(R.tvmrg_merkle_tree(dig.data_ptr(), tree.data_ptr(), L, sp), "Merkle")
            ev[3].record(stream)
            if times is not None:
                times.append((name, ev))

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        recs = []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(0) as clk:
            e0.record(stream)
            for _ in range(args.steps):
                step(recs)
            e1.record(stream)
            torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    stages = {}
    for name, ev in recs:
        d = stages.setdefault(name, {"lde": [], "row_hash": [], "merkle": []})
        d["lde"].append(ev[0].elapsed_time(ev[1]))
        d["row_hash"].append(ev[1].elapsed_time(ev[2]))
        d["merkle"].append(ev[2].elapsed_time(ev[3]))
    # per-step spread: the reference's LDE allocates and frees scratch inside
    # every call (cudaMalloc/cudaFree in randomized_lde_batch_impl), so its
    # stage times vary with the host and the allocator's state
    spread = {k: {s: [round(min(v), 2), round(max(v), 2)] for s, v in d.items()} for k, d in stages.items()}
    stages = {k: {s: statistics.median(v) for s, v in d.items()} for k, d in stages.items()}
    cells = L * (W_MAIN + W_AUX)
    line = {"metric": METRIC, "impl": "reference", "workload": "reference GPU kernels (sm_100a build)",
            "value": cells / (ms / 1e3), "unit": "cells/s", "ms_per_step": ms, "steps": args.steps,
            "warmup": args.warmup, "n_gpus": 1, "higher_is_better": True, "dtype": "u64 (Goldilocks)",
            "data": "synthetic uniform field elements",
            "config": {"workload": f"main 2^{args.log_n}x{W_MAIN} + aux 2^{args.log_n}x{W_AUX} limbs, x4 LDE "
                                   "(offset 7), Tip5 row hash, Merkle (two trees)", "trace_len": n, "lde_len": L,
                       "traces": "resident in HBM", "kernels": "randomized_lde_batch_gpu_preallocated (no "
                       "randomizers), hash_bfield_rows_gpu / hash_xfield_rows_gpu, merkle_tree_gpu"},
            "stage_ms_per_table": stages, "stage_ms_min_max": spread,
            "parity_2p10x379_vs_oracle": parity, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import tvmc
    ws, rank, local = dist_info()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    n = 1 << args.log_n
    L = EXPANSION * n
    main = random_trace(torch, W_MAIN, n, 1000 + rank, dev)
    aux = random_trace(torch, W_AUX, n, 2000 + rank, dev)
    cells_step = L * (W_MAIN + W_AUX)
    # pick the kernel knobs for this shape (cached per device and shape; untimed)
    import autotune
    tuned = autotune.tune_commit(main.data_ptr(), n, W_MAIN, EXPANSION, OFFSET, stream=sp) if W_MAIN else {}
    torch.cuda.synchronize()

    # main and aux are independent commitments: with --streams 2 the aux table
    # runs on a second stream (its row hash overlapping the other's LDE; the
    # per-phase times then overlap too, so the roofline lines assume 1 stream)
    stream2 = torch.cuda.Stream(dev) if args.streams > 1 else stream
    sp2 = stream2.cuda_stream
    # the end-to-end run always uses two streams: one table's upload overlaps
    # the other's kernels
    sp_e2e = torch.cuda.Stream(dev).cuda_stream

    def step(profile=False):
        a = tvmc.Commitment(main.data_ptr(), width=W_MAIN, trace_len=n, device_ptr=True, stream=sp,
                            profile=profile, expansion=EXPANSION, offset=OFFSET)
        b = tvmc.Commitment(aux.data_ptr(), width=W_AUX, trace_len=n, device_ptr=True, stream=sp2,
                            profile=profile, expansion=EXPANSION, offset=OFFSET)
        return a, b

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    # warm-up with the timed loop's own pattern (two steps live), so the
    # stream-ordered pool already holds what the timed steps reuse
    live = []
    for _ in range(args.warmup):
        cur = step()
        for c in live:
            c.free()
        live = list(cur)
    for c in live:
        c.free()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches0 = tvmc.lib().tvmc_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    live, phases = [], []
    with ClockSampler(local) as clk:
        ev0.record(stream)
        stream2.wait_event(ev0)
        for _ in range(args.steps):
            cur = step(profile=True)
            for c in live:  # free the previous step (host waits for it; the device stays busy)
                phases.append(c.phase_ms())
                c.free()
            live = list(cur)
        stream.wait_stream(stream2)
        ev1.record(stream)
        torch.cuda.synchronize()
        for c in live:
            phases.append(c.phase_ms())
            c.free()
    launches = tvmc.lib().tvmc_launch_count() - launches0
    t_ms = ev0.elapsed_time(ev1)
    barrier()
    t_max = max_over_ranks(t_ms, dev)
    value = whole_job_rate(cells_step * args.steps, ws, t_max / 1e3)

    # dominant kernel: Tip5 row hash + tree (phase 3); LDE phase against HBM
    hash_ms = [p[2] for p in phases]
    lde_ms = [p[1] for p in phases]
    widths = [W_MAIN, W_AUX] * args.steps
    ops = [perms_per_table(L, w) * OPS_PER_PERM for w in widths]
    achieved_int = sum(ops) / (sum(hash_ms) / 1e3) / 1e12
    lde_bytes = [8 * n * w + 8 * L * w for w in widths]
    achieved_hbm = sum(lde_bytes) / (sum(lde_ms) / 1e3) / 1e9
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    hbm_peak, hbm_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        hbm_peak, hbm_src = float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    clocks = clk.summary()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    sm_mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    int_peak = issue_limit_tops(sms, sm_mhz)
    # whole step: the slower of its HBM bytes and its integer work
    step_bytes = sum(bytes_per_table(n, w) for w in (W_MAIN, W_AUX))
    step_int_ops = sum(perms_per_table(L, w) * OPS_PER_PERM + ntt_ops_per_table(n, w) for w in (W_MAIN, W_AUX))
    hbm_ms = step_bytes / (hbm_peak * 1e9) * 1e3
    int_ms = step_int_ops / (int_peak * 1e12) * 1e3
    ms_step = t_max / args.steps
    roof_commit = {"bound": "int32" if int_ms >= hbm_ms else "hbm", "roofline_ms_per_step": max(hbm_ms, int_ms),
                   "ms_per_step": ms_step, "frac": max(hbm_ms, int_ms) / ms_step,
                   "hbm_ms": hbm_ms, "int_ms": int_ms, "bytes_per_step": step_bytes,
                   "int_ops_per_step": step_int_ops, "hbm_peak_gbs": hbm_peak, "hbm_peak_source": hbm_src,
                   "int_peak_tops": int_peak,
                   "cost_model": f"Tip5 {OPS_PER_PERM} int32 ops per permutation; NTT {OPS_PER_NTT_MUL} per "
                                 "butterfly or scale; bytes 8NW + 32NW + 40*4N + 40*(4N-1) per table"}
    # DRAM bytes per k_hash_rows launch: one ncu capture of the 2^18-row x 379-column
    # main-table launch (795.6 MB read + 16.0 MB written), scaled by rows
    traffic, traffic_src = None, None
    if W_MAIN == 379:
        traffic = (795.59e6 + 16.05e6) * L / (1 << 18)
        traffic_src = "ncu dram__bytes_read+write of a 2^18x379 launch, scaled by LDE rows (main table)"

    # e2e: pinned host traces through the public C ABI, roots read back
    e2e = None
    if not args.skip_e2e:
        h_main = torch.empty((W_MAIN, n), dtype=torch.int64, pin_memory=True)
        h_aux = torch.empty((W_AUX, n), dtype=torch.int64, pin_memory=True)
        h_main.copy_(main)
        h_aux.copy_(aux)
        hm, ha = h_main.numpy().view(np.uint64), h_aux.numpy().view(np.uint64)
        del main, aux
        torch.cuda.empty_cache()
        roots = []

        # Steps are pipelined as a prover committing tables back to back would:
        # step k+1's commits (uploads included) are issued before step k's roots
        # are read back, so its uploads overlap step k's row hash.  Every step's
        # uploads and root reads are inside the timed region.
        def issue():
            a = tvmc.Commitment(hm, stream=sp, expansion=EXPANSION, offset=OFFSET, discard_lde=True)
            b = tvmc.Commitment(ha, stream=sp_e2e, expansion=EXPANSION, offset=OFFSET, discard_lde=True)
            return a, b

        def finish(pair):
            roots.append(tuple(c.root() for c in pair))
            for c in pair:
                c.free()

        def run_e2e(steps):
            prev = None
            for _ in range(steps):
                cur = issue()
                if prev is not None:
                    finish(prev)
                prev = cur
            finish(prev)

        run_e2e(max(2, args.warmup))
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        run_e2e(args.steps)
        torch.cuda.synchronize()
        te = max_over_ranks(time.perf_counter() - t0, dev)
        e2e = {"value": whole_job_rate(cells_step * args.steps, ws, te), "unit": "cells/s",
               "h2d_bytes_per_step": 8 * n * (W_MAIN + W_AUX), "d2h_bytes_per_step": 2 * 40, "streams": 2,
               "pipelined": "step k+1 issued before step k's roots are read",
               "ms_per_step": 1e3 * te / args.steps}

        # the same from row-major host traces (the reference CPU layout,
        # vector<vector<BFE>>): upload, device transpose, LDE, hash, tree
        if not args.skip_row_major:
            rm = {}
            for w, hc in ((W_MAIN, h_main), (W_AUX, h_aux)):
                r = torch.empty((n, w), dtype=torch.int64, pin_memory=True)
                r.copy_(hc.t())
                rm[w] = r.numpy().view(np.uint64)

            def run_rm(steps):
                for _ in range(steps):
                    a = tvmc.Commitment(rm[W_MAIN], row_major=True, stream=sp, expansion=EXPANSION,
                                        offset=OFFSET, discard_lde=True)
                    b = tvmc.Commitment(rm[W_AUX], row_major=True, stream=sp_e2e, expansion=EXPANSION,
                                        offset=OFFSET, discard_lde=True)
                    a.root()
                    b.root()
                    a.free()
                    b.free()

            run_rm(max(1, args.warmup // 2))
            torch.cuda.synchronize()
            barrier()
            t0 = time.perf_counter()
            run_rm(args.steps)
            torch.cuda.synchronize()
            trm = max_over_ranks(time.perf_counter() - t0, dev)
            e2e["row_major"] = {"value": whole_job_rate(cells_step * args.steps, ws, trm), "unit": "cells/s",
                                "ms_per_step": 1e3 * trm / args.steps,
                                "transpose": "TMA tiles" if tvmc.get_tuning("transpose_tma") == 1
                                else "shared-memory tiles",
                                "what": "row-major pinned host traces (the reference CPU layout): upload, "
                                        "device transpose, LDE, row hash, tree; roots read back; not pipelined"}
            del rm

    # serving figures (BASELINE's metric names serving p50/p99 beside throughput)
    serving = None
    if rank == 0 and ws == 1 and not args.skip_serving and args.log_n == LOG_N:
        serving = serving_compact(torch, dev, h_main if e2e else None, h_aux if e2e else None)

    cpu = None
    if rank == 0 and ws == 1 and not args.skip_cpu:
        v, cores, sample, detail = cpu_reference_sample(args.log_n)
        cpu = {"value": v, "unit": "cells/s", "cores": cores, "kind": "reference", "sample": sample,
               "est_commit_s": detail["est_commit_s"], "extrapolated": True, "cpu_model": cpu_model()}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64 (Goldilocks)",
            "data": "synthetic uniform field elements",
            "config": {"workload": f"main 2^{args.log_n}x{W_MAIN} + aux 2^{args.log_n}x{W_AUX} limbs, x4 LDE (offset 7), "
                                   "Tip5 row hash, Merkle (two trees)",
                       "trace_len": n, "lde_len": L, "widths": [W_MAIN, W_AUX], "expansion": EXPANSION,
                       "cells_per_step": cells_step, "l2": "inputs (5.4 GB) larger than L2",
                       "tuning": tuned.get("knobs", {}), "tuning_s": tuned.get("seconds", {}),
                       "streams": args.streams,
                       "parallelism": "replicas" if ws > 1 else "1 gpu"},
            "roofline": {"bound": "int32", "kernel": "k_hash_rows + k_merkle_level + k_merkle_up (Tip5)",
                         "achieved": achieved_int, "peak": int_peak, "unit": "Top/s",
                         "frac": achieved_int / int_peak,
                         "peak_source": f"SM issue limit: {sms} SMs x {ISSUE_LANES_PER_SM} lanes x {sm_mhz:.0f} MHz "
                                        "(median SM clock sampled in the timed region)",
                         "traffic": traffic, "traffic_source": traffic_src,
                         "cost_model": f"{OPS_PER_PERM} int32 ops per Tip5 permutation",
                         "ms_per_step": sum(hash_ms) / args.steps,
                         "ms_per_table_min_max": [min(hash_ms), max(hash_ms)]},
            "roofline_commit": roof_commit,
            "phase_ms_per_table": {name: {"lde": statistics.median(p[1] for p in phases[i::2]),
                                          "hash_tree": statistics.median(p[2] for p in phases[i::2])}
                                   for i, name in enumerate(("main", "aux"))},
            "roofline_lde": {"bound": "hbm", "achieved": achieved_hbm, "peak": hbm_peak, "unit": "GB/s",
                             "frac": achieved_hbm / hbm_peak, "peak_source": hbm_src,
                             "bytes": "8*N*W read + 8*4N*W written per table",
                             "ms_per_step": sum(lde_ms) / args.steps,
                             "ms_per_table_min_max": [min(lde_ms), max(lde_ms)]},
            "e2e": e2e,
            "serving": serving,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _seeded_shapes(seed: int, count: int, lo: int, hi: int):
    rng = np.random.default_rng(seed)
    logs = rng.integers(lo, hi + 1, count)
    widths = rng.choice([W_MAIN, W_AUX], count)
    return [(1 << int(l), int(w)) for l, w in zip(logs, widths)]


def _event_ms(torch, stream, fn, reps):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run_batch(args):
    """32 uneven tables committed by one graph launch vs each committed alone."""
    import torch
    import tvmc
    import autotune
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    shapes = _seeded_shapes(0x7E5EED03, 32, 12, 18)
    traces = [random_trace(torch, w, n, 3000 + i, dev) for i, (n, w) in enumerate(shapes)]
    cells = sum(EXPANSION * n * w for n, w in shapes)

    import ctypes
    cudart = ctypes.CDLL("libcudart.so.12")

    def fill(b):  # device-to-device copies into the batch's own input buffers
        for i, t in enumerate(traces):
            cudart.cudaMemcpy(ctypes.c_void_p(b.input_ptr(i)), ctypes.c_void_p(t.data_ptr()),
                              ctypes.c_size_t(t.numel() * 8), 3)
        torch.cuda.synchronize()

    tuned = autotune.tune_batch(shapes, fill)
    with tvmc.Batch(shapes) as b:
        fill(b)
        torch.cuda.synchronize()
        for _ in range(args.warmup):
            b.run(stream.cuda_stream)
        launches0 = tvmc.lib().tvmc_launch_count()
        with ClockSampler(0) as clk:
            ms = _event_ms(torch, stream, lambda: b.run(stream.cuda_stream), args.steps)
        launches = (tvmc.lib().tvmc_launch_count() - launches0) // args.steps
        roots = b.roots()

    def alone():
        for t, (n, w) in zip(traces, shapes):
            c = tvmc.Commitment(t.data_ptr(), width=w, trace_len=n, device_ptr=True, stream=stream.cuda_stream,
                                discard_lde=True)
            c.free()

    for _ in range(args.warmup):
        alone()
    ms_alone = _event_ms(torch, stream, alone, args.steps)
    # the rate a GPU-filling commit reaches (the largest table of the batch
    # alone): the batch can go no faster than its cells at that rate
    big = max(range(len(shapes)), key=lambda i: shapes[i][0] * shapes[i][1])

    def largest():
        n, w = shapes[big]
        tvmc.Commitment(traces[big].data_ptr(), width=w, trace_len=n, device_ptr=True, stream=stream.cuda_stream,
                        discard_lde=True).free()

    largest()
    ms_big = _event_ms(torch, stream, largest, args.steps)
    big_rate = EXPANSION * shapes[big][0] * shapes[big][1] / (ms_big / 1e3)
    ideal_ms = 1e3 * cells / big_rate
    match = True
    for i, (t, (n, w)) in enumerate(zip(traces, shapes)):
        with tvmc.Commitment(t.data_ptr(), width=w, trace_len=n, device_ptr=True) as c:
            match = match and bool((c.root() == roots[i]).all())
    line = {"metric": "committed LDE cells/s", "workload": "batch", "value": cells / (ms / 1e3), "unit": "cells/s",
            "ms_per_batch": ms, "alone_ms": ms_alone, "speedup_vs_alone": ms_alone / ms,
            "ceiling": {"largest_table_cells_per_s": big_rate, "ideal_ms_at_that_rate": ideal_ms,
                        "ceiling_vs_alone": ms_alone / ideal_ms,
                        "what": "the batch's cells at the rate of its largest table committed alone"},
            "roots_equal_alone": match, "steps": args.steps, "warmup": args.warmup, "n_gpus": 1,
            "config": {"tables": len(shapes), "heights": [n for n, _ in shapes], "widths": [w for _, w in shapes],
                       "expansion": EXPANSION, "cells": cells, "tuning": tuned.get("knobs", {}),
                       "tuning_s": tuned.get("seconds", {})},
            "gpu_launches_per_batch": launches, "clocks": clk.summary(), "data": "synthetic uniform field elements"}
    print(json.dumps(line), flush=True)


def run_frugal(args):
    """2^22 x 379 streamed in stripes (the full LDE never exists) vs materialised."""
    import torch
    import tvmc
    import autotune
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    log_n = args.log_n if args.log_n != LOG_N else 22
    n, w = 1 << log_n, W_MAIN
    trace = random_trace(torch, w, n, 4000, dev)
    cells = EXPANSION * n * w
    tuned = autotune.tune_frugal(trace.data_ptr(), n, w)

    def commit(frugal):
        c = tvmc.Commitment(trace.data_ptr(), width=w, trace_len=n, device_ptr=True, stream=stream.cuda_stream,
                            frugal=frugal, discard_lde=True)
        c.free()

    for _ in range(args.warmup):
        commit(True)
    free0 = torch.cuda.mem_get_info(dev)[0]
    with ClockSampler(0) as clk:
        ms = _event_ms(torch, stream, lambda: commit(True), args.steps)
    for _ in range(1):
        commit(False)
    ms_mat = _event_ms(torch, stream, lambda: commit(False), max(1, args.steps // 2))
    with tvmc.Commitment(trace.data_ptr(), width=w, trace_len=n, device_ptr=True, frugal=True) as a, \
            tvmc.Commitment(trace.data_ptr(), width=w, trace_len=n, device_ptr=True, discard_lde=True) as b:
        same = bool((a.root() == b.root()).all())
    line = {"metric": "committed LDE cells/s", "workload": "frugal", "value": cells / (ms / 1e3), "unit": "cells/s",
            "ms_per_commit": ms, "materialised_ms": ms_mat, "root_equals_materialised": same,
            "lde_bytes_if_materialised": cells * 8, "steps": args.steps, "warmup": args.warmup, "n_gpus": 1,
            "config": {"trace_len": n, "width": w, "expansion": EXPANSION, "tuning": tuned.get("knobs", {}),
                       "tuning_s": tuned.get("seconds", {}), "free_bytes_before_timing": free0},
            "clocks": clk.summary(), "data": "synthetic uniform field elements"}
    print(json.dumps(line), flush=True)


class ServingStream:
    """The serving workload: Poisson arrivals of commitment requests with
    heights 2^10 .. 2^max_log log-uniform and widths 379 / 264 limbs by seed,
    80 openings each.  Request traces are prefixes of two pinned host tables
    (one per width), so every request is a contiguous column-major host trace.

    plain(): the per-request drop-in -- one tvmc_commit at a time in arrival
    order, root read back, then the openings.  served(): the serving loop.
    ceiling(): per shape class the GPU time of a commit with the trace already
    on the device and the time of the trace's host-to-device copy alone; no
    scheduler can exceed M / max(sum of GPU times, sum of copy times)."""

    def __init__(self, torch, dev, M, max_log, seed, h_main=None, h_aux=None):
        self.torch, self.dev, self.M = torch, dev, M
        self.shapes = _seeded_shapes(seed, M, 10, max_log)
        n_max = max(n for n, _ in self.shapes)
        host, self.host_t = {}, {}
        for w, h in ((W_MAIN, h_main), (W_AUX, h_aux)):
            if h is None or h.shape[0] != w or h.shape[1] < n_max:
                d = random_trace(torch, w, n_max, 5000 + w, dev)
                h = torch.empty((w, n_max), dtype=torch.int64, pin_memory=True)
                h.copy_(d)
                del d
            self.host_t[w] = h.reshape(-1)  # pinned; request traces are its prefixes
            host[w] = h.numpy().view(np.uint64).reshape(-1)
        torch.cuda.synchronize()
        self.reqs = [host[w][: w * n].reshape(w, n) for n, w in self.shapes]
        rng = np.random.default_rng(seed + 1)
        self.opens = [rng.integers(0, EXPANSION * n, 80) for n, _ in self.shapes]
        self.cells = [EXPANSION * n * w for n, w in self.shapes]
        self.large = np.array([c * 8 > (128 << 20) for c in self.cells])
        self.stream = torch.cuda.Stream(dev)

    @staticmethod
    def _wait_until(target):
        while time.monotonic_ns() < target:
            time.sleep(max(0.0, (target - time.monotonic_ns()) / 1e9 - 0.0005))

    def plain(self, arr_ns):
        import tvmc
        lat, svc = [], []
        t0 = time.monotonic_ns() + 20_000_000
        for i, t in enumerate(self.reqs):
            target = t0 + arr_ns[i]
            self._wait_until(target)
            start = time.monotonic_ns()
            c = tvmc.Commitment(t, stream=self.stream.cuda_stream, discard_lde=True)
            c.root()
            done = time.monotonic_ns()
            lat.append(done - target)
            svc.append(done - start)
            c.auth_paths(self.opens[i])
            c.free()
        return lat, (time.monotonic_ns() - t0 - arr_ns[0]) / 1e9, svc

    def served(self, arr_ns, streams=4, max_large=0, group_small=False):
        import threading
        import tvmc
        M = self.M
        lat, svc = [0] * M, [0] * M
        ids = [None] * M
        ready = [threading.Event() for _ in range(M)]
        t0 = time.monotonic_ns() + 20_000_000
        with tvmc.Server(streams=streams, max_large=max_large, group_small=group_small) as srv:
            def waiter():
                for i in range(M):
                    ready[i].wait()
                    srv.wait(ids[i])
                    srv.open(ids[i], self.opens[i])
                    _sub, start, done = srv.times(ids[i])
                    lat[i] = done - (t0 + arr_ns[i])
                    svc[i] = done - start
                    srv.release(ids[i])
            th = threading.Thread(target=waiter)
            th.start()
            for i, t in enumerate(self.reqs):
                self._wait_until(t0 + arr_ns[i])
                ids[i] = srv.submit(t)
                ready[i].set()
            th.join()
            stats = srv.stats()
        return lat, (time.monotonic_ns() - t0 - arr_ns[0]) / 1e9, stats, svc

    def summary(self, lat, span, svc):
        ms = np.array(lat) / 1e6
        sv = np.array(svc) / 1e6
        out = {"p50_ms": float(np.percentile(ms, 50)), "p99_ms": float(np.percentile(ms, 99)),
               "mean_ms": float(ms.mean()), "throughput_rps": self.M / span, "cells_per_s": sum(self.cells) / span}
        for name, sel in (("small", ~self.large), ("large", self.large)):
            if sel.any():
                out[f"{name}_p50_ms"] = float(np.percentile(ms[sel], 50))
                out[f"{name}_p99_ms"] = float(np.percentile(ms[sel], 99))
                out[f"{name}_service_mean_ms"] = float(sv[sel].mean())
        return out

    def arrivals(self, rho, service_s):
        lam = rho / service_s
        gaps = np.random.default_rng(int(rho * 1000)).exponential(1.0 / lam, self.M)
        return lam, [int(x) for x in (np.cumsum(gaps) - gaps[0]) * 1e9]

    def ceiling(self, span_plain):
        """GPU-only and copy-only time of the stream (CUDA events, per shape
        class, median of 3), against the plain path's back-to-back span."""
        import tvmc
        torch = self.torch
        gpu_ms, copy_ms = {}, {}
        st = self.stream
        for (n, w) in sorted(set(self.shapes)):
            d = torch.empty(w * n, dtype=torch.int64, device=self.dev)
            ht = self.host_t[w][: w * n]
            g, cp = [], []
            for k in range(4):
                e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
                with torch.cuda.stream(st):
                    e[0].record(st)
                    d.copy_(ht, non_blocking=True)
                    e[1].record(st)
                    e[2].record(st)
                    c = tvmc.Commitment(d.data_ptr(), width=w, trace_len=n, device_ptr=True,
                                        stream=st.cuda_stream, discard_lde=True)
                    e[3].record(st)
                st.synchronize()
                c.free()
                if k:
                    cp.append(e[0].elapsed_time(e[1]))
                    g.append(e[2].elapsed_time(e[3]))
            gpu_ms[(n, w)] = statistics.median(g)
            copy_ms[(n, w)] = statistics.median(cp)
            del d
        sum_gpu = sum(gpu_ms[s] for s in self.shapes) / 1e3
        sum_copy = sum(copy_ms[s] for s in self.shapes) / 1e3
        bound = max(sum_gpu, sum_copy)
        return {"gpu_busy_s": sum_gpu, "copy_s": sum_copy, "plain_span_s": span_plain,
                "plain_gpu_busy_frac": sum_gpu / span_plain, "plain_copy_frac": sum_copy / span_plain,
                "ceiling_rps": self.M / bound, "ceiling_vs_plain": span_plain / bound,
                "bound_by": "gpu" if sum_gpu >= sum_copy else "host-to-device copies"}


def serving_compact(torch, dev, h_main, h_aux, M=400, rho=3.0):
    """The serving figures for the default bench line: one offered load, plain
    vs served, plus the ceiling."""
    ss = ServingStream(torch, dev, M, LOG_N, 0x7E5EED05, h_main, h_aux)
    ss.plain([0] * M)  # warm-up: twiddle tables, pool, pinned paths
    ss.served([0] * M)
    lat0, span0, _ = ss.plain([0] * M)
    ceil = ss.ceiling(span0)
    lam, arr = ss.arrivals(rho, span0 / M)
    pl = ss.summary(*ss.plain(arr))
    sv_lat, sv_span, _, sv_svc = ss.served(arr)
    sv = ss.summary(sv_lat, sv_span, sv_svc)
    return {"requests": M, "load_vs_plain_capacity": rho, "rate_rps": lam,
            "plain": {k: pl[k] for k in ("p50_ms", "p99_ms", "throughput_rps")},
            "server": {k: sv[k] for k in ("p50_ms", "p99_ms", "throughput_rps")},
            "throughput_vs_plain": sv["throughput_rps"] / pl["throughput_rps"],
            "ceiling_vs_plain": ceil["ceiling_vs_plain"], "plain_gpu_busy_frac": ceil["plain_gpu_busy_frac"],
            "plain_copy_frac": ceil["plain_copy_frac"],
            "mix": f"heights 2^10..2^{LOG_N} log-uniform, widths 379/264, 80 openings each, pinned host traces"}


def run_serving(args):
    """Poisson arrivals, mixed sizes, 80 openings per request: serving loop vs
    the plain per-request drop-in (one commit at a time, in arrival order),
    swept over offered loads, with the ceiling any scheduler could reach."""
    import torch
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    M = args.requests
    ss = ServingStream(torch, dev, M, args.serve_max_log_n, 0x7E5EED05)
    zero = [0] * M
    ss.plain(zero)  # warm-up: twiddle tables, pool, pinned paths
    ss.served(zero, args.serve_streams, args.serve_max_large)
    lat0, span0, _ = ss.plain(zero)  # back-to-back: the plain path's service time
    service_s = span0 / M
    ceil = ss.ceiling(span0)
    rates = []
    for rho in args.serve_loads:
        lam, arr_ns = ss.arrivals(rho, service_s)
        pl, pspan, psvc = ss.plain(arr_ns)
        sv, sspan, stats, ssvc = ss.served(arr_ns, args.serve_streams, args.serve_max_large)
        entry = {"load_vs_plain_capacity": rho, "rate_rps": lam, "plain": ss.summary(pl, pspan, psvc),
                 "server": ss.summary(sv, sspan, ssvc), "server_peak_bytes": stats["bytes_peak"],
                 "server_budget_bytes": stats["budget"]}
        if args.serve_grouped:
            gp, gspan, _, gsvc = ss.served(arr_ns, args.serve_streams, args.serve_max_large, group_small=True)
            entry["server_grouped"] = ss.summary(gp, gspan, gsvc)
        rates.append(entry)
    line = {"metric": "serving latency p50/p99 and throughput", "workload": "serving", "requests": M,
            "plain_service_ms_mean": 1e3 * service_s, "ceiling": ceil,
            "config": {"heights": f"2^10..2^{args.serve_max_log_n} log-uniform", "widths": [W_MAIN, W_AUX],
                       "expansion": EXPANSION, "openings_per_request": 80, "server_streams": args.serve_streams,
                       "server_max_large_inflight": args.serve_max_large,
                       "small_large_split": "LDE <= 128 MB is small",
                       "host_buffers": "pinned; each request a contiguous prefix of one of two tables",
                       "latency": "arrival -> root committed (server: completion callback time)"},
            "rates": rates, "n_gpus": 1, "data": "synthetic uniform field elements"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--log-n", type=int, default=LOG_N)
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--width-main", type=int, default=W_MAIN, help="main-table columns (profiling sizes)")
    ap.add_argument("--width-aux", type=int, default=W_AUX, help="aux-table base limbs (profiling sizes)")
    ap.add_argument("--workload", choices=["commit", "batch", "frugal", "serving"], default="commit")
    ap.add_argument("--streams", type=int, default=1,
                    help="commit, device-timed part: main and aux on 1 or 2 streams (e2e always uses 2)")
    ap.add_argument("--reference-gpu", action="store_true",
                    help="with --impl reference: time the reference's own CUDA kernels (sm_100a build) instead")
    ap.add_argument("--ref-max-seconds", type=float, default=400.0,
                    help="reference arm: time budget for its full CPU steps")
    ap.add_argument("--requests", type=int, default=500, help="serving: requests per rate")
    ap.add_argument("--serve-grouped", action="store_true",
                    help="serving: also run the server with small-request grouping on (TVMC_SERVER_GROUP_SMALL)")
    ap.add_argument("--skip-serving", action="store_true", help="commit: no serving figures in the line")
    ap.add_argument("--skip-row-major", action="store_true", help="commit: no row-major e2e case")
    ap.add_argument("--serve-streams", type=int, default=4)
    ap.add_argument("--serve-max-log-n", type=int, default=20)
    ap.add_argument("--serve-max-large", type=int, default=0,
                    help="serving: large tables issued at once (0: the server's default)")
    ap.add_argument("--serve-loads", type=float, nargs="+", default=[0.5, 0.9, 1.5, 3.0],
                    help="serving: offered load as a multiple of the plain path's capacity")
    args = ap.parse_args()
    globals()["W_MAIN"], globals()["W_AUX"] = args.width_main, args.width_aux
    if args.impl == "reference" and args.reference_gpu:
        run_reference_gpu(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "frugal":
        run_frugal(args)
    elif args.workload == "serving":
        run_serving(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
