"""The multi-GPU host logic of bench.py on CPU, as two gloo ranks.

The path shards as independent replicas (no data-path collective): each rank
commits its own tables, the job's time is the slowest rank's (max over ranks)
and the whole-job rate is ranks x units per rank / that time.  The reference
arm runs on rank 0 only; other ranks exit 0 without work."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT

WORKER = r"""
import datetime, json, os, sys
sys.path.insert(0, os.environ["BENCH_ROOT"])
import torch.distributed as dist
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
import bench
rank = dist.get_rank()
t = bench.max_over_ranks(10.0 + 5.0 * rank)       # rank 1 is the slow one
rate = bench.whole_job_rate(100.0, dist.get_world_size(), t)
print(json.dumps({"rank": rank, "t": t, "rate": rate}))
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, ws, port):
    e = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
             MASTER_PORT=str(port), BENCH_ROOT=ROOT)
    e.pop("CUDA_VISIBLE_DEVICES", None)
    return e


def test_replicas_time_is_max_over_two_gloo_ranks():
    port = _free_port()
    procs = [subprocess.Popen([sys.executable, "-c", WORKER], env=_env(r, 2, port), stdout=subprocess.PIPE,
                              stderr=subprocess.PIPE, text=True) for r in range(2)]
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["t"] == 15.0                      # both ranks see the slowest rank's time
        assert o["rate"] == pytest.approx(200.0 / 15.0)


def test_max_over_ranks_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.whole_job_rate(10.0, 1, 2.0) == 5.0


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libtvm_ref.so")),
                    reason="reference harness not built")
def test_reference_arm_runs_on_rank0_only():
    args = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--log-n", "10",
            "--steps", "1", "--warmup", "0"]
    port = _free_port()
    r1 = subprocess.run(args, env=_env(1, 2, port), capture_output=True, text=True, timeout=300)
    assert r1.returncode == 0 and r1.stdout.strip() == ""
    r0 = subprocess.run(args, env=_env(0, 2, port), capture_output=True, text=True, timeout=300)
    assert r0.returncode == 0, r0.stderr[-2000:]
    line = json.loads(r0.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
