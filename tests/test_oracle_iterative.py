"""The oracle's large-mesh forms against its direct forms on small meshes:
FP64 block Jacobi-PCG (the stand-in for SparseLU where the direct solve is
out of reach) against SuperLU, and the Kronecker-factor application of the
nodal forcing covariance against the dense C restatement of
CovarianceForcing::giveProjectedCovar (statX/infer/CovarianceForcing.ipp:38-109)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from statfem_b200 import meshgen as mg
from tests.problems import QPS, statfem_problem

CASES = [(mg.HEX8_ELASTIC, 4, "x0", [0.0, 0.0, -1.0]), (mg.TRI3_POISSON, 12, "all", [1.0]),
         (mg.LINE2_POISSON, 30, "x", [1.0]), (mg.HEX8_POISSON, 5, "all", [1.0])]


@pytest.mark.parametrize("kind,n,faces,f", CASES)
def test_iterative_prior_matches_direct(kind, n, faces, f):
    prob = statfem_problem(kind, n, 7, seed=3, faces=faces)
    mesh = prob["mesh"]
    Pd = mg.projection_dense(mesh, *prob["P"])
    f = np.array(f)
    d = O.statfem_prior(mesh, QPS[kind], f, prob["bc"], Pd, 0.1, 0.2, 0.001, coeff=prob["coeff"])
    it = O.statfem_prior_iterative(mesh, QPS[kind], f, prob["bc"], Pd, 0.1, 0.2, 0.001, coeff=prob["coeff"])
    assert np.abs(it["mean_s"] - d["mean_s"]).max() <= 1e-12 * np.abs(d["mean_s"]).max()
    assert np.abs(it["C_s"] - d["C_s"]).max() <= 1e-12 * np.abs(d["C_s"]).max()
    assert (it["its"] > 0).all()


@pytest.mark.parametrize("kind,n,faces,f", CASES)
def test_grid_covariance_matches_dense(kind, n, faces, f):
    prob = statfem_problem(kind, n, 3, seed=5, faces=faces)
    mesh = prob["mesh"]
    phibar = O.unit_load(mesh, QPS[kind], prob["bc"])
    Cf = O.forcing_covariance_dense(mesh.dim, mesh.dof, mesh.coords, phibar, 0.07, 0.3)
    W = np.random.default_rng(0).standard_normal((mesh.num_dofs, 4))
    got = O.forcing_covariance_apply_grid(mesh, phibar, 0.07, 0.3, W)
    assert np.abs(got - Cf @ W).max() <= 1e-13 * np.abs(Cf @ W).max()


def test_block_pcg_restart_from_x0():
    """A restart from a converged block changes it by less than its tolerance
    allows, and stops at once when the start already satisfies the test."""
    prob = statfem_problem(mg.HEX8_ELASTIC, 3, 4, seed=9, faces="x0")
    mesh = prob["mesh"]
    rp, col, val, F = O.fem(mesh, 8, np.array([0.0, 0.0, -1.0]), prob["bc"], coeff=prob["coeff"])
    mask = np.zeros(mesh.num_dofs, dtype=np.uint8)
    mask[prob["bc"]] = 1
    B = np.vstack([F, mg.projection_dense(mesh, *prob["P"])])
    X1, its1 = O.block_pcg(rp, col, val, mask, B, 1e-8)
    X2, its2 = O.block_pcg(rp, col, val, mask, B, 1e-13, X0=X1)
    X3, its3 = O.block_pcg(rp, col, val, mask, B, 1e-13, X0=X2)
    assert (its1 > 0).all() and (its2 > 0).all() and (its3 == 0).all()
    assert np.abs(X3 - X2).max() == 0.0
    assert np.abs(X1 - X2).max() <= 1e-5 * np.abs(X2).max()


GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "c2_oracle.npz")


@pytest.mark.skipif(not os.path.exists(GOLDEN), reason="c2 oracle fixture not generated")
def test_c2_fixture_is_consistent():
    """The committed 48^3 elasticity oracle fixture: its inputs are the
    workload generator's, its oracle error estimate is far below the 1e-7
    parity bound, and its posterior follows from its prior (recomputed here
    with the numpy restatement of LikelihoodKOH)."""
    from statfem_b200.workloads import fingerprint
    from statfem_b200.workloads import make_workload
    g = np.load(GOLDEN)
    wl = make_workload("c2", seed=1234)
    assert np.allclose(g["fingerprint"], fingerprint(wl), rtol=1e-12, atol=0)
    assert g["est_rel_change_1e11_to_1e13"].max() < 1e-8
    ns = wl["ns"]
    iu = np.triu_indices(ns)
    C = np.zeros((ns, ns))
    C[iu] = g["C_s_upper"]
    C = C + np.triu(C, 1).T
    hp = wl["hp"]
    Ks = O.mismatch_covariance(wl["pts"], hp["mismatch.sigma"], hp["mismatch.length"], hp["mismatch.sensorEps"])
    pm, pc = O.koh_proj_conditioned(g["mean_s"], C, Ks, g["Y"], hp["rho"])
    assert np.abs(pm - g["post_mean"]).max() <= 1e-12 * np.abs(pm).max()
    ll = O.koh_log_likelihood(g["mean_s"], C, Ks, g["Y"], hp["rho"])
    assert abs(ll - float(g["loglik"])) <= 1e-10 * abs(ll)


GOLDEN_C4 = os.path.join(os.path.dirname(__file__), "golden", "c4_oracle.npz")


@pytest.mark.skipif(not os.path.exists(GOLDEN_C4), reason="c4 oracle fixture not generated")
def test_c4_fixture_is_consistent():
    """The multi-RHS oracle fixture was made from the workload generator's
    columns, and its oracle error estimate is far below 1e-7."""
    from statfem_b200.workloads import fingerprint, make_workload, multi_rhs_columns
    f = np.load(GOLDEN_C4)
    wl = make_workload("c2", seed=1234)
    assert np.allclose(f["fingerprint"], fingerprint(wl), rtol=1e-12, atol=0)
    wl["phibar"] = O.unit_load(wl["mesh"], wl["qps"], wl["bc"])
    B = multi_rhs_columns(wl, 1024, wl["hp"]["forcing.sigma"], wl["hp"]["forcing.length"], cols=f["pick"])
    assert np.allclose(f["b_sums"], B.sum(axis=1), rtol=1e-12, atol=0)
    assert np.allclose(f["b_norms"], np.linalg.norm(B, axis=1), rtol=1e-12, atol=0)
    assert float(f["est_rel_change_1e11_to_1e13"]) < 1e-9
    assert (f["energy"] > 0).all()
