"""Multi-GPU runs are independent replicas: the only exchange is the final
aggregate (max of the timed intervals, sum of the work). Checked with two
gloo ranks on the host."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        times, counts = bench.reduce_over_ranks([10.0 + rank, 5.0 * (rank + 1)], [100 * (rank + 1), 7])
        q.put((rank, times, counts))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_replicas_aggregate_max_time_and_summed_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=90) for _ in procs]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, times, counts in out:
        assert times == [11.0, 10.0]     # max over ranks of each interval
        assert counts == [300, 14]       # sum over ranks of each count


@pytest.mark.timeout(300)
def test_bench_gpus_two_starts_two_ranks():
    """``bench.py --gpus 2`` without a launcher starts two ranks itself (one
    process per GPU) and reports the aggregate with n_gpus from the world size;
    a host-only stand-in workload keeps the test off the GPU."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2",
                          "--workload", "replica-selftest", "--steps", "50", "--warmup", "3"],
                         capture_output=True, text=True, timeout=240, env=env, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1                      # rank 0 alone prints
    line = lines[0]
    assert line["n_gpus"] == 2 and line["config"]["ranks"] == 2
    assert line["steps"] == 50 and line["value"] > 0
