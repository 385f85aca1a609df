"""The multi-process plumbing of bench.py on CPU: two ranks over gloo.

A solve does not shard (replicas only), so the data path has no collective; the
ranks meet only to time the steps, as the maximum over ranks, and the reference
arm runs on rank 0 alone.  Run as two spawned processes on 127.0.0.1.
"""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout
from types import SimpleNamespace

import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    sys.path.insert(0, REPO)
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    try:
        # every rank gets the largest of the ranks' timings
        got = bench.max_over_ranks(1.0 + 2.5 * rank, dist, device="cpu")
        # the reference arm: rank 0 prints one JSON line, the others return at once
        buf = io.StringIO()
        with redirect_stdout(buf):
            bench.run_reference(SimpleNamespace(n=32, steps=1, warmup=0, gpus=world), rank)
        dist.barrier()
        out[rank] = (got, buf.getvalue())
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    world = 2
    port = _free_port()
    with mp.Manager() as manager:
        out = manager.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for rank in range(world):
        assert res[rank][0] == 1.0 + 2.5 * (world - 1)
    assert res[1][1] == ""
    lines = [l for l in res[0][1].splitlines() if l.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == world and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"


def test_max_over_ranks_single_process():
    sys.path.insert(0, REPO)
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5
