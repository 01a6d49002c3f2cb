"""Batched instances (persistent cluster kernel in a CUDA graph) against the
oracle, instance by instance: SuperLU adjoint solves of the reference's
row-zeroed system, the dense forcing covariance, and the numpy restatements
of LikelihoodKOH::giveLogLikelihood / giveProjFEconditionedData."""
import numpy as np
import pytest

from oracle import oracle as O
from statfem_b200 import api
from statfem_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


def make_batch(sides, ns, seed, poison=None):
    rng = np.random.default_rng(seed)
    meshes, coeffs, bcs, sensors, hps, Ys = [], [], [], [], [], []
    for k, (s, m) in enumerate(zip(sides, ns)):
        mesh = mg.unit_square_tri(s)
        c = np.exp(0.5 * rng.standard_normal(mesh.num_elems))
        if poison == k:
            c[3] = np.nan
        pts = mg.interior_points(rng, m, 2, margin=0.05)
        P = mg.projection_matrix(mesh, pts)
        meshes.append(mesh)
        coeffs.append(c)
        bcs.append(mg.dirichlet_dofs(mesh, "all"))
        sensors.append((P, pts))
        hps.append({"forcing.sigma": rng.uniform(0.05, 0.2), "forcing.length": rng.uniform(0.1, 0.4),
                    "rho": rng.uniform(0.8, 1.2), "mismatch.sigma": rng.uniform(0.0, 0.01),
                    "mismatch.length": rng.uniform(0.1, 0.3), "mismatch.sensorEps": 1e-3})
        Ys.append(0.05 + 0.01 * rng.standard_normal((m, 2)))
    union, off = mg.disjoint_union(meshes)
    bc = np.concatenate([b + off[k] for k, b in enumerate(bcs)])
    return dict(meshes=meshes, coeffs=coeffs, bcs=bcs, sensors=sensors, hps=hps, Ys=Ys, union=union, off=off,
                bc=bc, sides=sides)


def oracle_instance(pb, k, reg, f=1.0):
    mesh = pb["meshes"][k]
    P, pts = pb["sensors"][k]
    Pd = mg.projection_dense(mesh, *P)
    hp = pb["hps"][k]
    r = O.statfem_prior(mesh, 3, np.array([f]), pb["bcs"][k], Pd, hp["forcing.sigma"], hp["forcing.length"], reg,
                        coeff=pb["coeffs"][k])
    Ks = O.mismatch_covariance(pts, hp["mismatch.sigma"], hp["mismatch.length"], hp["mismatch.sensorEps"])
    Y = pb["Ys"][k]
    ll = O.koh_log_likelihood(r["mean_s"], r["C_s"], Ks, Y, hp["rho"])
    pm, pc = O.koh_proj_conditioned(r["mean_s"], r["C_s"], Ks, Y, hp["rho"])
    return r["mean_s"], r["C_s"], ll, pm, pc


def run_gpu(ctx, pb, reg, cluster=0, tol=1e-10):
    gm = api.Mesh(ctx, mg.TRI3_POISSON, 3, pb["union"].coords, pb["union"].conn)
    b = api.BatchStatFEM(ctx, gm, pb["off"], pb["sides"], pb["bc"], pb["sensors"], 1.0, cluster)
    b.set_solver(tol=tol)
    b.set_coefficients(np.concatenate(pb["coeffs"]))
    b.set_hparams(pb["hps"], reg)
    b.set_readings(pb["Ys"])
    b.run()
    return b, gm


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


SIDES = [4, 9, 6, 14, 11, 3, 20]
NS = [5, 8, 3, 12, 7, 1, 32]


def test_batch_matches_oracle(ctx):
    reg = 1e-3
    pb = make_batch(SIDES, NS, 3)
    b, gm = run_gpu(ctx, pb, reg)
    res = b.results()
    assert (res["status"] == 0).all(), res["status"]
    for k in range(len(SIDES)):
        m = NS[k]
        mean, C, ll, pm, pc = oracle_instance(pb, k, reg)
        assert rel(res["mean_s"][k, :m], mean) < 1e-8
        assert rel(res["cov_s"][k, :m, :m], C) < 1e-8
        assert abs(res["loglik"][k] - ll) < 1e-8 * max(1.0, abs(ll))
        assert rel(res["post_mean"][k, :m], pm) < 1e-7
        assert rel(res["post_cov"][k, :m, :m], pc) < 1e-7
        # unused sensor slots stay zero
        assert not res["cov_s"][k, m:, :].any() and not res["post_mean"][k, m:].any()
    b.close()


@pytest.mark.parametrize("cluster", [1, 2, 4, 16])
def test_batch_cluster_sizes_agree(ctx, cluster):
    """Any cluster shape gives the same results (to the solver tolerance)."""
    reg = 1e-3
    pb = make_batch(SIDES[:5], NS[:5], 4)
    b8, _ = run_gpu(ctx, pb, reg, cluster=8)
    r8 = b8.results()
    b, _ = run_gpu(ctx, pb, reg, cluster=cluster)
    cs, grid = b.launch_shape()
    assert cs <= max(cluster, 1) and grid % cs == 0
    r = b.results()
    assert (r["status"] == 0).all()
    assert rel(r["cov_s"], r8["cov_s"]) < 1e-8
    assert np.allclose(r["loglik"], r8["loglik"], rtol=1e-8, atol=1e-8)
    b.close()
    b8.close()


def test_batch_poisoned_instance_fails_alone(ctx):
    """A NaN conductivity in one instance gives that instance an error status;
    every other instance still matches the oracle."""
    reg = 1e-3
    pb = make_batch(SIDES[:4], NS[:4], 5, poison=2)
    b, _ = run_gpu(ctx, pb, reg)
    res = b.results()
    assert res["status"][2] != 0
    for k in (0, 1, 3):
        assert res["status"][k] == 0
        mean, C, ll, pm, pc = oracle_instance(pb, k, reg)
        assert rel(res["cov_s"][k, :NS[k], :NS[k]], C) < 1e-8
        assert abs(res["loglik"][k] - ll) < 1e-8 * max(1.0, abs(ll))
    b.close()


def test_batch_rerun_with_new_proposals(ctx):
    """The captured graph is relaunched with new coefficients and
    hyperparameters (the MCMC use): results follow the new inputs."""
    reg = 1e-3
    pb = make_batch(SIDES[:3], NS[:3], 6)
    b, _ = run_gpu(ctx, pb, reg)
    rng = np.random.default_rng(1)
    pb["coeffs"] = [np.exp(0.5 * rng.standard_normal(m.num_elems)) for m in pb["meshes"]]
    pb["hps"] = [dict(h, **{"forcing.length": h["forcing.length"] * 1.3, "rho": 1.1}) for h in pb["hps"]]
    b.set_coefficients(np.concatenate(pb["coeffs"]))
    b.set_hparams(pb["hps"], reg)
    b.run()
    res = b.results()
    for k in range(3):
        mean, C, ll, pm, pc = oracle_instance(pb, k, reg)
        assert rel(res["mean_s"][k, :NS[k]], mean) < 1e-8
        assert abs(res["loglik"][k] - ll) < 1e-8 * max(1.0, abs(ll))
    b.close()


def test_batch_rejects_non_grid_instances(ctx):
    pb = make_batch([4, 5], [2, 2], 7)
    gm = api.Mesh(ctx, mg.TRI3_POISSON, 3, pb["union"].coords, pb["union"].conn)
    with pytest.raises(api.SfcError):
        api.BatchStatFEM(ctx, gm, pb["off"], [4, 6], pb["bc"], pb["sensors"])
