"""Multi-GPU form of bench.py: independent replicas, one per rank, the job timed by its slowest
rank. Two gloo ranks on the CPU check the max-over-ranks reduction and the whole-job throughput
that bench.py reports, and that the reference arm prints from rank 0 only."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = [2.5, 3.5][rank]
        t = bench.max_over_ranks(local_ms, world, device="cpu")
        value = bench.job_throughput(262144, world, t / 1e3)
        buf = io.StringIO()

        class Args:
            precision, workload, steps, warmup = "f32", "plain", 1, 0

        if rank != 0:  # the reference arm: ranks other than 0 exit without work or output
            with redirect_stdout(buf):
                bench.run_reference(Args, rank, world)
        dist.barrier()
        out.put((rank, t, value, buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_replicas_max_over_ranks_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, value, printed in res:
        assert t == 3.5  # the slower rank
        assert value == pytest.approx(262144 * 2 / 3.5e-3)
        if rank != 0:
            assert printed == ""
