"""Parity at the benchmark configurations themselves, with the benchmark's
solver settings (relative residual 1e-8): prior mean and covariance at the
sensors, KOH log-likelihood and sensor-space posterior mean and covariance,
each within 1e-7 relative of the FP64 oracle.

c1 (64^2 P1 Poisson, 16 sensors): SuperLU oracle, dense forcing covariance.
c3 (Poisson instances with sides across 32..256, 32 sensors each): SuperLU
    oracle per instance, forcing covariance through its Kronecker factors.
c2 (48^3 hex8 elasticity, 352,947 dofs, 256 sensors): the committed oracle
    fixture tests/golden/c2_oracle.npz (FP64 Jacobi-PCG to 1e-13; made by
    tests/golden/make_c2_oracle.py), with the fixture's readings.
The reference formulas: ForwardGaussRHS.hpp:95-139, LikelihoodKOH.ipp:75-120
and 311-361."""
import os

import numpy as np
import pytest

import bench
from oracle import oracle as O
from statfem_b200 import api
from statfem_b200 import meshgen as mg
from statfem_b200.workloads import C3_HP, REG, draw_readings, make_batch_workload, make_workload

pytestmark = pytest.mark.gpu

REL = 1e-7  # north_star's bound on the posterior mean / covariance
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "c2_oracle.npz")


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def koh_oracle(mean_s, C_s, pts, Y, hp):
    Ks = O.mismatch_covariance(pts, hp["mismatch.sigma"], hp["mismatch.length"], hp["mismatch.sensorEps"])
    ll = O.koh_log_likelihood(mean_s, C_s, Ks, Y, hp["rho"])
    pm, pc = O.koh_proj_conditioned(mean_s, C_s, Ks, Y, hp["rho"])
    return ll, pm, pc


def check_all(got, ref):
    errs = {k: rel(got[k], ref[k]) for k in ("mean_s", "C_s", "post_mean", "post_cov")}
    errs["loglik"] = abs(got["loglik"] - ref["loglik"]) / max(1.0, abs(ref["loglik"]))
    bad = {k: v for k, v in errs.items() if not v < REL}
    assert not bad, "relative errors above 1e-7: %s (all: %s)" % (bad, errs)
    return errs


@pytest.mark.parametrize("method,precond", [("fp64", "jacobi"), ("mixed", "two-level"), ("mixed", "jacobi")])
def test_c1_at_config_size(method, precond):
    wl = make_workload("c1", seed=1234)
    mesh, hp = wl["mesh"], wl["hp"]
    Pd = mg.projection_dense(mesh, *wl["P"])
    pr = O.statfem_prior(mesh, wl["qps"], wl["f"], wl["bc"], Pd, hp["forcing.sigma"], hp["forcing.length"], REG,
                         coeff=wl["coeff"])
    Y = draw_readings(np.random.default_rng(5), pr["mean_s"], pr["C_s"], hp)
    ll, pm, pc = koh_oracle(pr["mean_s"], pr["C_s"], wl["pts"], Y, hp)
    m = api.SFC_SOLVER_PCG_MIXED if method == "mixed" else api.SFC_SOLVER_PCG_FP64
    g = bench.GpuStatFEM(wl, 0, m, 128, bench.precond_code(api, precond))
    g.koh.setSensorValues(Y)
    gll, gpm, gpc = g.step()
    got = dict(mean_s=g.fg.giveProjectedMeanU(), C_s=g.fg.giveProjectedCovarU(), loglik=gll, post_mean=gpm,
               post_cov=gpc)
    check_all(got, dict(mean_s=pr["mean_s"], C_s=pr["C_s"], loglik=ll, post_mean=pm, post_cov=pc))


def test_c3_sides_32_to_256():
    """Instances at both ends and inside the config's side range, through the
    persistent batch kernel with the benchmark's tolerances (rel. residual
    1e-9, FP32 reduction 1e-2 between FP64 residuals)."""
    sides = [32, 256, 77, 141, 203, 45]
    wl = make_batch_workload(4321, sides=sides)
    ctx = api.Context(0)
    gm = api.Mesh(ctx, mg.TRI3_POISSON, 3, wl["union"].coords, wl["union"].conn)
    b = api.BatchStatFEM(ctx, gm, wl["off"], wl["sides"], wl["bc"], wl["sensors"], 1.0)
    b.set_solver(tol=1e-9, inner_tol=1e-2)  # the bench's c3 setting (at 1e-8 the worst instance is at 1.1e-7)
    b.set_coefficients(wl["coeff"])
    b.set_hparams(C3_HP, REG)
    refs, Ys = [], []
    rng = np.random.default_rng(11)
    for k, mesh in enumerate(wl["meshes"]):
        P, pts = wl["sensors"][k]
        Pd = mg.projection_dense(mesh, *P)
        rp, col, val, F = O.fem(mesh, 3, np.array([1.0]), wl["bcs"][k], coeff=wl["coeffs"][k])
        R = O.DirectSolver(rp, col, val).solve_transpose(Pd.T).T
        phibar = O.unit_load(mesh, 3, wl["bcs"][k])
        mean_s, C_s = O.forward_gauss_rhs_grid(R, F, Pd, mesh, phibar, C3_HP["forcing.sigma"],
                                               C3_HP["forcing.length"], REG)
        Y = draw_readings(rng, mean_s, C_s, C3_HP)
        ll, pm, pc = koh_oracle(mean_s, C_s, pts, Y, C3_HP)
        refs.append(dict(mean_s=mean_s, C_s=C_s, loglik=ll, post_mean=pm, post_cov=pc))
        Ys.append(Y)
    b.set_readings(Ys)
    b.run()
    res = b.results()
    assert (res["status"] == 0).all(), res["status"]
    for k in range(len(sides)):
        got = dict(mean_s=res["mean_s"][k], C_s=res["cov_s"][k], loglik=res["loglik"][k],
                   post_mean=res["post_mean"][k], post_cov=res["post_cov"][k])
        check_all(got, refs[k])
    b.close()
    gm.close()
    ctx.close()


@pytest.mark.skipif(not os.path.exists(GOLDEN), reason="c2 oracle fixture not generated")
def test_c2_headline_against_fp64_oracle():
    """The benchmark's default workload and solver (mixed FP32 block PCG with
    FP64 residuals, two-level preconditioner, rel. residual 1e-8) against the
    committed FP64 oracle."""
    from statfem_b200.workloads import fingerprint
    g0 = np.load(GOLDEN)
    wl = make_workload("c2", seed=1234)
    assert np.allclose(g0["fingerprint"], fingerprint(wl), rtol=1e-12, atol=0), "workload generator changed"
    ns = wl["ns"]
    iu = np.triu_indices(ns)

    def sym(u):
        M = np.zeros((ns, ns))
        M[iu] = u
        return M + np.triu(M, 1).T

    ref = dict(mean_s=g0["mean_s"], C_s=sym(g0["C_s_upper"]), loglik=float(g0["loglik"]),
               post_mean=g0["post_mean"], post_cov=sym(g0["post_cov_upper"]))
    g = bench.GpuStatFEM(wl, 0, api.SFC_SOLVER_PCG_MIXED, 128, api.SFC_PRECOND_TWO_LEVEL)
    g.koh.setSensorValues(g0["Y"])
    ll, pm, pc = g.step()
    got = dict(mean_s=g.fg.giveProjectedMeanU(), C_s=g.fg.giveProjectedCovarU(), loglik=ll, post_mean=pm,
               post_cov=pc)
    errs = check_all(got, ref)
    print("c2 relative errors against the FP64 oracle:", errs)


GOLDEN_C4 = os.path.join(os.path.dirname(__file__), "golden", "c4_oracle.npz")


@pytest.mark.skipif(not os.path.exists(GOLDEN_C4), reason="c4 oracle fixture not generated")
def test_c4_columns_against_fp64_oracle():
    """Multi-RHS prior covariance columns on the 48^3 elasticity mesh (mixed
    block PCG with the two-level preconditioner, rel. residual 1e-10): the
    oracle fixture's 16 columns, compared through the functionals it keeps
    (values at the 256 sensor rows, energy u^T b)."""
    from statfem_b200.workloads import fingerprint, multi_rhs_columns
    f = np.load(GOLDEN_C4)
    wl = make_workload("c2", seed=1234)
    assert np.allclose(f["fingerprint"], fingerprint(wl), rtol=1e-12, atol=0), "workload generator changed"
    g = bench.GpuStatFEM(wl, 0, api.SFC_SOLVER_PCG_MIXED, 128, api.SFC_PRECOND_TWO_LEVEL)
    wl["phibar"] = g.cf.phibar()
    pick = f["pick"]
    B = multi_rhs_columns(wl, 1024, wl["hp"]["forcing.sigma"], wl["hp"]["forcing.length"], cols=pick)
    assert np.allclose(f["b_sums"], B.sum(axis=1), rtol=1e-12, atol=0)
    g.s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-10, max_iter=30000, inner_tol=1e-4, block_width=128,
                    check_every=32, precond=api.SFC_PRECOND_TWO_LEVEL)
    U = g.s.solveSystemMulti(B)
    st = g.s.last_stats()
    assert st["converged"] == 1 and st["max_rel_residual"] <= 1e-10
    Pd = mg.projection_dense(wl["mesh"], *wl["P"])
    pu = Pd @ U.T
    en = np.einsum("ij,ij->i", U, B)
    sens = (np.abs(pu - f["Pu"]).max(axis=0) / np.abs(f["Pu"]).max(axis=0)).max()
    ener = (np.abs(en - f["energy"]) / np.abs(f["energy"])).max()
    assert sens < 1e-7 and ener < 1e-7, (sens, ener)
