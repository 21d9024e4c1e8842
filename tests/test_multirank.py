"""The N>1 host logic of bench.py on CPU with two gloo ranks: replicas solve disjoint solutes,
every rank reports the slowest rank's time, and the whole-job rate counts all ranks' solutes.
The reference arm runs on rank 0 alone."""
import datetime
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    sys.path[:0] = [ROOT, os.path.join(ROOT, "mdft-dev_general_b200")]
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    t = bench.max_over_ranks(100.0 + 50.0 * rank, world, "cpu")       # rank 1 is the slower one
    seeds = bench.replica_seeds(rank, 9)
    every = [None] * world
    dist.all_gather_object(every, seeds)
    q.put((rank, t, bench.whole_job_rate(world, 6, t), every))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, rate, every in got:
        assert t == 150.0                       # the max over ranks, on every rank
        assert rate == 2 * 6 / 0.150            # all ranks' solutes over the slowest time
        assert not set(every[0]) & set(every[1])  # replicas solve different solutes


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def _rank_dies(rank, world, port, q):
    sys.path[:0] = [ROOT, os.path.join(ROOT, "mdft-dev_general_b200")]
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    import bench
    if rank == 1:
        os._exit(3)  # this replica dies between steps, before the timing reduction
    try:
        bench.max_over_ranks(100.0, world, "cpu")
        q.put((rank, "no error"))
    except Exception as e:  # noqa: BLE001 - the collective's error is the detection
        q.put((rank, type(e).__name__))


def test_a_dead_replica_ends_the_others_collective_with_an_error():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_dies, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    rank, what = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
    assert rank == 0 and what != "no error"
    assert procs[1].exitcode == 3
