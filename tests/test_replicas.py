"""The replica path of bench.py on the CPU: world size 2 over gloo, as
`torchrun --nproc-per-node 2 bench.py` runs it (one independent instance per
rank, no data-path collective).  The device time of a step is the maximum
over the ranks; the reference arm runs on rank 0 alone, which prints the one
JSON line, and the other ranks exit 0 without work."""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist            # noqa: E402
import torch.multiprocessing as mp          # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from relax_b200.config import linear_maxwell
        # a tiny deck stands in for the benchmark workload
        bench.workload = lambda: linear_maxwell(sx=32, sz=32, dx=1.0, steps=4)
        v = bench.max_over_ranks(10.0 + rank, dist)

        class A:
            steps, warmup = 2, 3
        buf = io.StringIO()
        with redirect_stdout(buf):
            rc = bench.run_reference(A, rank, world)
        dist.barrier()
        out.put((rank, v, rc, buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_replicas_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    (r0, v0, rc0, out0), (r1, v1, rc1, out1) = res
    assert v0 == v1 == 11.0                   # the maximum over the two ranks
    assert rc0 == rc1 == 0
    assert out1 == ""                         # rank 1: no work, no line
    lines = [l for l in out0.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0
