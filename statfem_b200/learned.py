"""Training driver for the learned preconditioner (LearnedPreconditioner in
api.py) over many material samples.

The reference has no learned part: it factorises with Eigen::SparseLU
(corlib/SystemSolveEigenSparse.hpp).  Here a message-passing network is
trained on the GPU, one material sample at a time: for each sample the
library runs Jacobi-PCG on the sample's system, takes residual/error pairs
from its iterates and makes Adam steps on them.  After every epoch the
parameters and the Adam moments are written to a checkpoint (with the number
of finished epochs beside it), so an interrupted run resumes where it
stopped.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

from . import api
from . import meshgen as mg


class PoissonSamples:
    """3-D Poisson problems -div(k grad u) = f on the unit cube (n^3 hex8
    elements, 2x2x2 Gauss points, u = 0 on the boundary) whose
    log-conductivity is a Matérn nu = 3/2 field per element; sample k is
    drawn with seed seed0 + k.  One GPU system is reused: a sample only
    re-assembles the matrix values."""

    def __init__(self, ctx, n, sigma=1.0, length=0.1, seed0=0, load=1.0):
        self.ctx = ctx
        self.n = n
        self.sigma = sigma
        self.length = length
        self.seed0 = seed0
        self.mesh = mg.unit_cube_hex(n, mg.HEX8_POISSON)
        self.gm = api.Mesh(ctx, mg.HEX8_POISSON, 8, self.mesh.coords, self.mesh.conn)
        self.bc = mg.dirichlet_dofs(self.mesh, "all")
        self.load = np.array([load])
        self.system = api.SystemSolveCuda(ctx, self.mesh.num_dofs)

    def coefficients(self, k):
        rng = np.random.default_rng(self.seed0 + k)
        return np.exp(mg.matern32_field_cells(rng, self.n, self.sigma, self.length))

    def assemble(self, k, coeff=None):
        """Assemble sample k (or the given coefficients) into the system."""
        self.gm.set_coefficients(self.coefficients(k) if coeff is None else coeff)
        s = self.system
        s.assemble(self.gm)
        s.clearRhs()
        s.assemble_load(self.gm, self.load)
        s.applyConstraints((self.bc, np.zeros(len(self.bc))))
        return s


def train(net, samples, indices, epochs=1, steps_per_sample=40, checkpoint=None, resume=True, log=None,
          **opts):
    """Train `net` on samples.assemble(k) for k in indices, `epochs` times.
    opts go to LearnedPreconditioner.train (batch, lr, max_pairs, ...).
    Returns {"loss": per-step losses of this run, "seconds", "epochs"}."""
    start = 0
    if checkpoint and resume and os.path.exists(checkpoint) and os.path.exists(checkpoint + ".json"):
        net.load(checkpoint)
        with open(checkpoint + ".json") as f:
            start = int(json.load(f)["epochs"])
    hist = []
    t0 = time.perf_counter()
    for ep in range(start, epochs):
        for j, k in enumerate(indices):
            s = samples.assemble(k)
            h = net.train(s, steps=steps_per_sample, seed=ep * 1000003 + j, **opts)
            hist.append(h)
            if log:
                log("epoch %d sample %d loss %.4f -> %.4f" % (ep, k, h[:5].mean(), h[-5:].mean()))
        if checkpoint:
            net.save(checkpoint)
            with open(checkpoint + ".json", "w") as f:
                json.dump({"epochs": ep + 1, "samples": len(indices), "steps_per_sample": steps_per_sample}, f)
    return {"loss": np.concatenate(hist) if hist else np.zeros(0), "seconds": time.perf_counter() - t0,
            "epochs": epochs}
