"""Generates tests/golden/c2_oracle.npz: the FP64 oracle's prior and
posterior at the sensors for the 48^3 elasticity statFEM workload (352,947
dofs, 256 sensors; statfem_b200.workloads.make_workload("c2", seed=1234)).

The reference's Eigen SparseLU cannot factor this system in any reasonable
time (a 117k-dof 3-D Poisson matrix already takes minutes in SuperLU), so the
oracle solves the forward system and the 256 adjoint systems by FP64
Jacobi-PCG (oracle.statfem_prior_iterative, OpenMP over matrix rows), first to
the relative residual 1e-11 and then, restarted from that solution, to 1e-13.
The change of every output between the two runs is stored as the oracle's
own error estimate (the 1e-13 solution is about a hundred times closer).
On small meshes the same iterative oracle agrees with the SuperLU oracle to
1e-13 (tests/test_oracle_iterative.py).

Observations: one reading per sensor drawn from the oracle's prior plus
noise (LikelihoodKOH::giveTypicalReadings), numpy seed 97531.  Stored: the
inputs' fingerprints, prior mean and covariance, readings, KOH
log-likelihood, sensor-space posterior mean and covariance (upper triangles
of the symmetric matrices).

    python tests/golden/make_c2_oracle.py      # about half an hour on 8 cores
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from statfem_b200 import meshgen as mg  # noqa: E402
from statfem_b200.workloads import REG, draw_readings, fingerprint, make_workload  # noqa: E402


def outputs(pr, wl, Y):
    hp = wl["hp"]
    Ks = O.mismatch_covariance(wl["pts"], hp["mismatch.sigma"], hp["mismatch.length"], hp["mismatch.sensorEps"])
    ll = O.koh_log_likelihood(pr["mean_s"], pr["C_s"], Ks, Y, hp["rho"])
    pm, pc = O.koh_proj_conditioned(pr["mean_s"], pr["C_s"], Ks, Y, hp["rho"])
    return dict(mean_s=pr["mean_s"], C_s=pr["C_s"], loglik=ll, post_mean=pm, post_cov=pc)


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def main():
    wl = make_workload("c2", seed=1234)
    mesh, hp = wl["mesh"], wl["hp"]
    Pd = mg.projection_dense(mesh, *wl["P"])
    t0 = time.time()
    args = (mesh, wl["qps"], wl["f"], wl["bc"], Pd, hp["forcing.sigma"], hp["forcing.length"], REG)
    p11 = O.statfem_prior_iterative(*args, coeff=wl["coeff"], nu=0.3, tol=1e-11)
    t1 = time.time()
    p13 = O.statfem_prior_iterative(*args, coeff=wl["coeff"], nu=0.3, tol=1e-13, X0=p11["X"])
    t2 = time.time()
    Y = draw_readings(np.random.default_rng(97531), p13["mean_s"], p13["C_s"], hp)
    o11, o13 = outputs(p11, wl, Y), outputs(p13, wl, Y)
    diff = {k: rel(o11[k], o13[k]) for k in o13}
    iu = np.triu_indices(wl["ns"])
    np.savez_compressed(
        os.path.join(HERE, "c2_oracle.npz"),
        fingerprint=fingerprint(wl), mean_s=o13["mean_s"], C_s_upper=o13["C_s"][iu], Y=Y,
        loglik=np.float64(o13["loglik"]), post_mean=o13["post_mean"], post_cov_upper=o13["post_cov"][iu],
        tol=np.float64(1e-13), its_1e11=p11["its"], its_1e13_restart=p13["its"],
        est_names=np.array(sorted(diff)), est_rel_change_1e11_to_1e13=np.array([diff[k] for k in sorted(diff)]))
    print("solves: %.0f s to 1e-11 (max %d it), %.0f s more to 1e-13 (max %d it)"
          % (t1 - t0, p11["its"].max(), t2 - t1, p13["its"].max()))
    print("relative change 1e-11 -> 1e-13:", diff)


if __name__ == "__main__":
    main()
