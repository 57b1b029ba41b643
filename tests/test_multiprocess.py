"""The N > 1 path of bench.py on CPU: independent replicas, one process per rank, whose
only collectives are the barrier and the max-over-ranks timing reduction (gloo here,
NCCL on GPUs), and the reference arm under torchrun (rank 0 alone runs and prints).
World size 2, rendezvous on 127.0.0.1."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _replica(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    try:
        # each replica times its own steps; the job's time is the slowest rank's
        local = [0.30 + 0.05 * rank, 0.25 - 0.01 * rank]
        ms, kms = bench.max_over_ranks(local, ws)
        dist.barrier()
        out[rank] = (ms, kms, bench.replica_value(ws, 1_000_000, ms))
    finally:
        dist.destroy_process_group()


def test_replica_timing_is_the_max_over_ranks():
    ws = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_replica, args=(ws, _free_port(), out), nprocs=ws, start_method="spawn", join=True)
    assert set(out.keys()) == {0, 1}
    for r in range(ws):
        ms, kms, value = out[r]
        assert ms == pytest.approx(0.35) and kms == pytest.approx(0.25)
        assert value == pytest.approx(2 * 1_000_000 / 0.35e-3)


def test_reference_arm_under_torchrun_prints_once():
    """`bench.py --impl reference` launched like the driver's N > 1 runs: rank 0 times the
    CPU restatement on a bounded sample and prints one JSON line, rank 1 exits 0."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "3", "--ref-sample", "2000"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
