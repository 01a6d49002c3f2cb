"""Sharded batch of independent statFEM instances over two gloo ranks on the
CPU: the cost-balanced partition, each rank evaluating only its share, and
the all-gather that gives every rank all instances' log-likelihoods and
sensor-space posteriors, equal to the one-rank evaluation.  The per-instance
evaluation is the oracle's host restatement (SuperLU adjoint solves,
LikelihoodKOH in numpy) standing in for the device work, which on GPUs is
the persistent batch kernel over the rank's share."""
import datetime
import multiprocessing as mp
import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def evaluate(wl, k, Y):
    """One instance on the host: prior at the sensors, log-likelihood and
    posterior (the oracle's restatement of the batch kernel's outputs)."""
    from oracle import oracle as O
    from statfem_b200 import meshgen as mg
    from statfem_b200.workloads import C3_HP, REG
    mesh = wl["meshes"][k]
    P, pts = wl["sensors"][k]
    Pd = mg.projection_dense(mesh, *P)
    hp = C3_HP
    pr = O.statfem_prior(mesh, 3, np.array([1.0]), wl["bcs"][k], Pd, hp["forcing.sigma"], hp["forcing.length"], REG,
                         coeff=wl["coeffs"][k])
    Ks = O.mismatch_covariance(pts, hp["mismatch.sigma"], hp["mismatch.length"], hp["mismatch.sensorEps"])
    ll = O.koh_log_likelihood(pr["mean_s"], pr["C_s"], Ks, Y, hp["rho"])
    pm, pc = O.koh_proj_conditioned(pr["mean_s"], pr["C_s"], Ks, Y, hp["rho"])
    return ll, pm, pc


def readings(wl):
    rng = np.random.default_rng(77)
    return [0.05 + 0.01 * rng.standard_normal((wl["ns"], 1)) for _ in wl["meshes"]]


def _worker(rank, ws, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        from statfem_b200 import shard
        from statfem_b200.workloads import make_batch_workload
        # every rank generates the same batch (same seed) and keeps its share
        wl = make_batch_workload(99, n_inst=7, smin=4, smax=12, ns=6)
        parts = shard.partition(shard.instance_costs(wl["sides"]), ws)
        Ys = readings(wl)
        mine = [evaluate(wl, int(k), Ys[k]) for k in parts[rank]]
        local = {"loglik": np.array([m[0] for m in mine]), "post_mean": np.stack([m[1] for m in mine]),
                 "post_cov": np.stack([m[2] for m in mine])}
        full = shard.gather(local, parts, len(wl["sides"]))
        q.put((rank, [p.tolist() for p in parts], {k: v.tolist() for k, v in full.items()}))
    finally:
        dist.destroy_process_group()


def test_partition_balances_and_covers():
    from statfem_b200 import shard
    sides = np.random.default_rng(0).integers(32, 257, 512)
    for world in (1, 2, 3, 8):
        parts = shard.partition(shard.instance_costs(sides), world)
        allk = np.sort(np.concatenate(parts))
        assert np.array_equal(allk, np.arange(len(sides)))
        loads = [shard.instance_costs(sides[p]).sum() for p in parts]
        assert max(loads) - min(loads) <= shard.instance_costs([256])[0]


def test_two_ranks_gather_equals_one_rank():
    sys.path.insert(0, ROOT)
    from statfem_b200.workloads import make_batch_workload
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted((q.get(timeout=180) for _ in range(2)), key=lambda t: t[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, parts0, full0), (_, parts1, full1) = out
    assert parts0 == parts1 and sorted(parts0[0] + parts0[1]) == list(range(7))
    assert len(parts0[0]) > 0 and len(parts0[1]) > 0
    wl = make_batch_workload(99, n_inst=7, smin=4, smax=12, ns=6)
    Ys = readings(wl)
    ref = [evaluate(wl, k, Ys[k]) for k in range(7)]
    for full in (full0, full1):
        assert np.array_equal(np.array(full["loglik"]), np.array([r[0] for r in ref]))
        assert np.array_equal(np.array(full["post_mean"]), np.stack([r[1] for r in ref]))
        assert np.array_equal(np.array(full["post_cov"]), np.stack([r[2] for r in ref]))
