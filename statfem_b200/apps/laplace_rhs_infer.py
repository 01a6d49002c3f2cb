"""laplaceRHSinfer on the GPU, reading the reference application's input
files unchanged (del2/apps/reference/laplaceRHSinfer: laplaceRHSinfer.cpp,
fem.hpp, inference.hpp, hyperParamLearning.hpp).

    python -m statfem_b200.apps.laplace_rhs_infer [--dir DIR] [--chains 64]
           [--fixed-hp rho=0.8,mismatch.sigma=0.02,mismatch.length=0.07]

DIR holds input.dat (meshFile, allParamFile, infInputFile), the SMF mesh
(2-node line elements, 3-point quadrature), the parameter map and the
inference properties (numReadings, phiMatFile, sensorPosFile, sensorValFile,
numSamples, enrichWithPrior, hpsMeanFile, sampleMCMCFile, feCondDataFile).
As the application: uniform conductivity from the parameter map, body force
pi^2/5 (fem.hpp:22-29), homogeneous Dirichlet where x = 0 or x = 1
(fem.hpp:36-45), ForwardGaussRHS with reg 0.001 (inference.hpp:136), MCMC
over log(rho, mismatch.sigma, mismatch.length) from the init.* values with
the propStDev.* proposal, posterior means after a 30 % burn-in written to
hpsMeanFile and used for the Woodbury posterior mean written to
feCondDataFile.  The sampler runs --chains chains side by side (numSamples
in total); --fixed-hp skips the sampling and uses the given values.
"""
from __future__ import annotations

import argparse
import math
import os
import sys

import numpy as np

from .. import api
from .. import io as sio
from .. import meshgen as mg
from ..mcmc import BatchedMetropolis

FREE = ("rho", "mismatch.sigma", "mismatch.length")


def run(directory, chains=64, fixed_hp=None, seed=0, log=print):
    def path(p):
        return os.path.join(directory, p)

    top = sio.read_properties(path("input.dat"))
    mesh = sio.read_smf(path(top["meshFile"]), kind=mg.LINE2_POISSON)
    hp = sio.read_param_map(path(top["allParamFile"]))
    inf = sio.read_properties(path(top["infInputFile"]))
    N = mesh.num_dofs
    ctx = api.Context(0)
    gm = api.Mesh(ctx, mg.LINE2_POISSON, 3, mesh.coords, mesh.conn)
    gm.set_coefficients(None, uniform=float(hp["conductivity"]))
    s = api.SystemSolveCuda(ctx, N)
    s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-13)
    x = mesh.coords[:, 0]
    bc = np.nonzero(mg.fuzzy_equal(x, 0.0) | mg.fuzzy_equal(x, 1.0))[0]
    s.assemble(gm)
    s.assemble_load(gm, math.pi * math.pi / 5.0)
    s.applyConstraints((bc, np.zeros(len(bc))))
    s.solveSystem()
    cf = api.CovarianceForcing(ctx, gm)
    cf.applyConstraints(bc)
    fg = api.ForwardGaussRHS(s, cf, 0.001)
    P = sio.read_matrix_phi(path(inf["phiMatFile"]), N)
    fg.setProjectionMatrix(P)
    fg.updateSolution(hp)
    pts = sio.read_coord_data(path(inf["sensorPosFile"]), mesh.dim)
    Y = sio.read_matrix_data(path(inf["sensorValFile"]))
    koh = api.LikelihoodKOH(fg, pts)
    koh.setSensorValues(Y)
    if fixed_hp is not None:
        hp.update(fixed_hp)
    else:
        n_samples = int(inf.get("numSamples", "20000"))
        steps = max(1, n_samples // chains)
        prior = None
        if int(inf.get("enrichWithPrior", "0")):
            prior = ([hp["priorMean." + k] for k in FREE], [hp["priorCov." + k] for k in FREE])
        mc = BatchedMetropolis(koh, hp, free=FREE, n_chains=chains, seed=seed, prior=prior)
        x0 = np.log([hp["init." + k] for k in FREE])
        std = [hp["propStDev." + k] for k in FREE]
        xs, ys, acc = mc.sample(steps, std, x0)
        mean = BatchedMetropolis.posterior_mean(xs)
        log("MCMC: %d chains x %d steps, acceptance %.3f" % (chains, steps, float(acc.mean())))
        for k, v in zip(FREE, mean):
            hp[k] = float(v)
        if "hpsMeanFile" in inf:
            with open(path(inf["hpsMeanFile"]), "w") as f:
                for k in FREE:
                    f.write("%s  %g\n" % (k, hp[k]))
        if "sampleMCMCFile" in inf:
            with open(path(inf["sampleMCMCFile"]), "w") as f:
                b = int(steps * 0.3)
                for i in range(b, steps):
                    for c in range(chains):
                        f.write("  ".join("%g" % v for v in np.exp(xs[i, c])) + "  %g\n" % ys[i, c])
    fg.updateSolution(hp)
    mean, _ = koh.giveFEconditionedDataWoodbury(hp, with_cov=False) if N <= 8192 else \
        (koh.giveFEconditionedMeanWoodbury(hp), None)
    if "feCondDataFile" in inf:
        sio.write_vector(path(inf["feCondDataFile"]), mean)
    return dict(hp={k: hp[k] for k in FREE}, mean=mean)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--dir", default=".")
    ap.add_argument("--chains", type=int, default=64)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--fixed-hp", default=None, help="name=value,... instead of sampling")
    a = ap.parse_args(argv)
    fixed = None
    if a.fixed_hp:
        fixed = {k: float(v) for k, v in (t.split("=") for t in a.fixed_hp.split(","))}
    out = run(a.dir, a.chains, fixed, a.seed)
    print(" ".join("%s=%g" % kv for kv in out["hp"].items()))
    return 0


if __name__ == "__main__":
    sys.exit(main())
