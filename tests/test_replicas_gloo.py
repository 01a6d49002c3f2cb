"""The multi-GPU path is replicas only (independent posterior solves per
rank, no collective on the data path): its host-side plumbing — barrier,
max-over-ranks device time, whole-job value, per-rank seeds — checked with two
gloo ranks on the CPU."""
import datetime
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        bench.barrier(ws)
        # each rank's timed region (ms); the job's time is the slowest rank's
        ms = bench.max_over_ranks(ws, 100.0 + 50.0 * rank)
        steps = 3
        value = ws * steps / (ms / 1e3)
        wl = bench.make_workload("c1", seed=1234 + rank)
        q.put((rank, ms, value, wl["pts"][0].tolist()))
    finally:
        dist.destroy_process_group()


def test_two_replicas_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(2))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, ms0, v0, pts0), (r1, ms1, v1, pts1) = out
    assert ms0 == ms1 == 150.0  # max over ranks, the same on every rank
    assert v0 == v1 == 2 * 3 / 0.150  # whole-job throughput: all ranks' steps over the slowest time
    assert pts0 != pts1  # ranks work on independent (differently seeded) instances
