"""Hyperparameter MCMC with many proposals per GPU launch.

The reference samples the free hyperparameters (rho, mismatch.sigma,
mismatch.length) in log space with a random-walk Metropolis chain
(statX::infer::MCMC::sample, statX/infer/MCMC.hpp:123-160, driven by
hyperParamLearning, del2/apps/reference/laplaceRHSinfer/hyperParamLearning.hpp:
90-249): proposal x' ~ N(x, diag(prop_std^2)), accept when
log u <= min(0, f(x') - f(x)), f = log-likelihood (+ log prior when
enrichWithPrior); the estimate is the mean of exp(x) over the samples after a
30 % burn-in.  Here n_chains such chains run side by side; every step
evaluates all proposals with one batched log-likelihood launch
(LikelihoodKOH.giveLogLikelihoodBatch).  The random numbers come from numpy
on the host (seeded); the reference's Boost mt19937 streams are not
reproduced, so individual draws differ from the reference's while the
sampled distribution is the same.
"""
from __future__ import annotations

import numpy as np

FREE_DEFAULT = ("rho", "mismatch.sigma", "mismatch.length")


class BatchedMetropolis:
    """n_chains random-walk Metropolis chains over log hyperparameters.

    likelihood: an api.LikelihoodKOH whose forward model has been updated.
    hp: the full hyperparameter map (values of the parameters not sampled).
    free: names of the sampled parameters.
    prior: optional (mean, var) per free parameter, used as the reference
    does (MultiVariateNormalPDF with the log of the prior means, evaluated at
    the exponentiated sample, hyperParamLearning.hpp:46-61, 92-98)."""

    def __init__(self, likelihood, hp, free=FREE_DEFAULT, n_chains=64, seed=0, prior=None):
        self.lik = likelihood
        self.hp = dict(hp)
        self.free = list(free)
        self.n = int(n_chains)
        self.rng = np.random.default_rng(seed)
        self.prior = prior

    def log_target(self, X):
        """f for each row of X (n x len(free), log space)."""
        E = np.exp(X)
        maps = []
        for row in E:
            h = dict(self.hp)
            for name, v in zip(self.free, row):
                h[name] = float(v)
            maps.append(h)
        f = self.lik.giveLogLikelihoodBatch(maps)
        if self.prior is not None:
            mean = np.log(np.array([self.prior[0][k] for k in range(len(self.free))]))
            var = np.array(self.prior[1], dtype=np.float64)
            d = E - mean
            f = f + (-0.5 * np.sum(d * d / var, axis=1) - 0.5 * np.sum(np.log(2 * np.pi * var)))
        return np.where(np.isfinite(f), f, -np.inf)

    def sample(self, n_samples, prop_std, x_init):
        """Run n_samples steps of every chain from x_init (log space, one row
        or one per chain).  Returns (samples n_samples x n x d, values
        n_samples x n, acceptance ratio per chain)."""
        d = len(self.free)
        x = np.broadcast_to(np.asarray(x_init, dtype=np.float64), (self.n, d)).copy()
        y = self.log_target(x)
        std = np.broadcast_to(np.asarray(prop_std, dtype=np.float64), (d,))
        xs = np.empty((n_samples, self.n, d))
        ys = np.empty((n_samples, self.n))
        acc = np.zeros(self.n)
        for i in range(n_samples):
            xp = x + std * self.rng.standard_normal((self.n, d))
            yp = self.log_target(xp)
            ratio = np.minimum(0.0, yp - y)
            ok = np.log(self.rng.random(self.n)) <= ratio
            x[ok] = xp[ok]
            y[ok] = yp[ok]
            acc += ok
            xs[i] = x
            ys[i] = y
        return xs, ys, acc / n_samples

    @staticmethod
    def posterior_mean(xs, burn_in=0.3):
        """Mean of exp(samples) after the burn-in fraction, pooled over the
        chains (hyperParamLearning.hpp:121-158)."""
        b = int(xs.shape[0] * burn_in)
        return np.exp(xs[b:]).reshape(-1, xs.shape[2]).mean(axis=0)
