"""bench.py --gpus N runs N independent replicas (a direct solve does not shard:
elimination is level-synchronous with neighbour fill-ins and a dense root).
The only collective is the timing reduction: every rank reports its own time
and the slowest one counts.  Checked here with two gloo ranks on the CPU."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    t = bench.max_over_ranks(1.0 + rank, dist)  # rank 1 is the slower one
    out[rank] = (t, bench.replica_throughput(world, 1000, 3, t))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_replica_throughput_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        t, v = out[r]
        assert t == 2.0  # the slowest rank's time on every rank
        assert v == pytest.approx(2 * 1000 * 3 / 2.0)


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun the CPU reference arm prints from rank 0 alone; another rank exits 0 without work."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
