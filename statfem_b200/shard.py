"""Splitting independent statFEM units across ranks (one process per GPU).

The units are independent by construction: the MCMC proposals of a batch
(each its own mesh, material and hyperparameters; statX/infer/MCMC.hpp:123-160
evaluates them one after another) or the right-hand-side columns of a
multi-RHS solve.  Each rank takes a share of the units with no data-path
communication; the only exchange is the gather of the per-unit results
(log-likelihoods, sensor-space means and covariances) that the sampler on
rank 0 needs, done with one all-gather per result array over the process
group (NCCL on GPUs, gloo on the CPU).

Balancing: units are sorted by cost (largest first) and dealt out in snake
order (0, 1, ..., W-1, W-1, ..., 0, 0, 1, ...), which keeps every rank's total
within one unit of the mean cost for the uniform side distributions of the
batch workload.
"""
from __future__ import annotations

import numpy as np


def partition(costs, world):
    """Index arrays (ascending) of the units each of `world` ranks takes."""
    costs = np.asarray(costs, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    order = np.argsort(-costs, kind="stable")
    parts = [[] for _ in range(world)]
    for k, u in enumerate(order):
        rnd, pos = divmod(k, world)
        r = pos if rnd % 2 == 0 else world - 1 - pos
        parts[r].append(int(u))
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def instance_costs(sides):
    """Cost model of a 2-D Poisson instance of side s: dofs x iterations,
    with PCG iterations growing like s (the condition number like s^2)."""
    s = np.asarray(sides, dtype=np.float64)
    return (s + 1.0) ** 2 * s


def gather(local, parts, n_total, group=None):
    """All-gather per-unit result arrays.  `local` maps a name to an array
    whose first axis runs over this rank's units (parts[rank] order); returns
    the same names with the first axis over all n_total units in global
    order, on every rank.  Uses torch.distributed on the default group (or
    `group`); the tensors live on the current CUDA device under NCCL and on
    the CPU otherwise."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if len(parts) != world:
        raise ValueError("one part per rank expected")
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    cap = max(len(p) for p in parts)
    out = {}
    for name in sorted(local):
        a = np.ascontiguousarray(local[name])
        if a.shape[0] != len(parts[rank]):
            raise ValueError("%s: %d rows for %d local units" % (name, a.shape[0], len(parts[rank])))
        pad = np.zeros((cap,) + a.shape[1:], dtype=a.dtype)
        pad[: a.shape[0]] = a
        t = torch.from_numpy(pad).to(dev)
        bufs = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(bufs, t, group=group)
        full = np.zeros((n_total,) + a.shape[1:], dtype=a.dtype)
        for r, p in enumerate(parts):
            full[p] = bufs[r][: len(p)].cpu().numpy()
        out[name] = full
    return out
