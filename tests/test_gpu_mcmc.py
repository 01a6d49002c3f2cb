"""Batched log-likelihood and the many-chain hyperparameter sampler."""
import numpy as np
import pytest

from statfem_b200 import api
from statfem_b200 import meshgen as mg
from statfem_b200.mcmc import BatchedMetropolis
from tests.test_gpu_statfem import HP, gpu_prior
from tests.problems import statfem_problem

pytestmark = pytest.mark.gpu


def _koh(ctx, seed=5):
    prob = statfem_problem(mg.TRI3_POISSON, 12, 10, seed=seed)
    g = gpu_prior(ctx, prob, HP, 1e-3, 1.0, api.SFC_SOLVER_PCG_FP64, tol=1e-12)
    rng = np.random.default_rng(seed)
    # readings from the model with rho 1.2 plus a mismatch of scale 0.01
    C = 0.01 ** 2 * np.eye(10) + 1.2 ** 2 * g["cov"]
    Y = 1.2 * g["mean"][:, None] + np.linalg.cholesky(C) @ rng.standard_normal((10, 4))
    koh = api.LikelihoodKOH(g["fg"], prob["pts"])
    koh.setSensorValues(Y)
    return koh, g


def test_batched_loglik_matches_single(ctx):
    koh, g = _koh(ctx)
    rng = np.random.default_rng(0)
    hps = [dict(HP, **{"rho": rng.uniform(0.5, 2), "mismatch.sigma": rng.uniform(0.001, 0.05),
                       "mismatch.length": rng.uniform(0.05, 0.5)}) for _ in range(37)]
    batch = koh.giveLogLikelihoodBatch(hps)
    single = np.array([koh.giveLogLikelihood(h) for h in hps])
    np.testing.assert_allclose(batch, single, rtol=1e-11, atol=1e-9)


def test_many_chain_sampler_matches_quadrature(ctx):
    """One free parameter (rho): the pooled posterior mean of exp(x) from 64
    chains against a quadrature of the same (flat-in-log) target."""
    koh, g = _koh(ctx, seed=7)
    hp = dict(HP, **{"mismatch.sigma": 0.01, "mismatch.length": 0.2})
    mc = BatchedMetropolis(koh, hp, free=["rho"], n_chains=64, seed=3)
    xs, ys, acc = mc.sample(300, prop_std=[0.05], x_init=[np.log(1.0)])
    assert 0.1 < acc.mean() < 0.9
    est = BatchedMetropolis.posterior_mean(xs)[0]
    grid = np.linspace(np.log(0.5), np.log(2.5), 2001)
    f = mc.log_target(grid[:, None])
    w = np.exp(f - f.max())
    ref = np.sum(np.exp(grid) * w) / np.sum(w)
    sd = np.sqrt(np.sum((np.exp(grid) - ref) ** 2 * w) / np.sum(w))
    assert abs(est - ref) < max(0.2 * sd, 1e-3 * ref), (est, ref, sd)
