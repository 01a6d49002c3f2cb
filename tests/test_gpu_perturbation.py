"""First-order material uncertainty (ForwardPerturbation) on the GPU against
the oracle's dense restatement of the reference's double sum over element
pairs."""
import numpy as np
import pytest

from oracle import oracle as O
from statfem_b200 import api
from statfem_b200 import meshgen as mg
from tests.problems import QPS, statfem_problem

pytestmark = pytest.mark.gpu

HP = {"forcing.sigma": 0.1, "forcing.length": 0.2, "rho": 1.0, "mismatch.sigma": 0.0,
      "mismatch.length": 0.2, "mismatch.sensorEps": 1e-3, "material.sigma": 0.4, "material.length": 0.3}


@pytest.mark.parametrize("kind,n,ns,amount", [(mg.TRI3_POISSON, 6, 5, 0.0), (mg.TRI3_POISSON, 5, 4, 0.25),
                                              (mg.HEX8_POISSON, 3, 6, 0.0)])
@pytest.mark.parametrize("method", [api.SFC_SOLVER_PCG_FP64, api.SFC_SOLVER_PCG_MIXED])
def test_perturbation_matches_oracle(ctx, kind, n, ns, amount, method):
    pr = statfem_problem(kind, n, ns, seed=17 + n, amount=amount)
    mesh = pr["mesh"]
    qps = QPS[kind]
    gm = api.Mesh(ctx, kind, qps, mesh.coords, mesh.conn)
    gm.set_coefficients(pr["coeff"])
    s = api.SystemSolveCuda(ctx, mesh.num_dofs)
    s.set_options(method=method, tol=1e-12)
    s.assemble(gm)
    s.assemble_load(gm, 1.0)
    s.applyConstraints((pr["bc"], np.zeros(len(pr["bc"]))))
    cf = api.CovarianceForcing(ctx, gm)
    cf.applyConstraints(pr["bc"])
    fg = api.ForwardGaussRHS(s, cf, 1e-3)
    fg.setProjectionMatrix(pr["P"])
    pt = api.ForwardPerturbation(fg, reg=1e-4)
    pt.updateSolution(HP, factor_tol=1e-15)
    assert 0 < pt.rank <= mesh.num_elems
    m = pt.giveProjectedMeanU()
    C = pt.giveProjectedCovarU()
    rp, col, val, F = O.fem(mesh, qps, 1.0, pr["bc"], coeff=pr["coeff"])
    phibar = O.unit_load(mesh, qps, pr["bc"])
    Pd = mg.projection_dense(mesh, *pr["P"])
    m_ref, C_ref = O.forward_perturbation(mesh, qps, F, rp, col, val, pr["bc"], Pd, phibar,
                                          HP["forcing.sigma"], HP["forcing.length"], HP["material.sigma"],
                                          HP["material.length"], 1e-4)
    np.testing.assert_allclose(m, m_ref, rtol=1e-8, atol=1e-14)
    assert np.abs(C - C_ref).max() <= 1e-7 * np.abs(C_ref).max()
    pt.close()


def test_perturbation_low_rank_factor(ctx):
    """A coarser factor tolerance uses fewer columns and stays close."""
    pr = statfem_problem(mg.TRI3_POISSON, 8, 6, seed=3)
    mesh = pr["mesh"]
    gm = api.Mesh(ctx, mg.TRI3_POISSON, 3, mesh.coords, mesh.conn)
    gm.set_coefficients(pr["coeff"])
    s = api.SystemSolveCuda(ctx, mesh.num_dofs)
    s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-12)
    s.assemble(gm)
    s.assemble_load(gm, 1.0)
    s.applyConstraints((pr["bc"], np.zeros(len(pr["bc"]))))
    cf = api.CovarianceForcing(ctx, gm)
    cf.applyConstraints(pr["bc"])
    fg = api.ForwardGaussRHS(s, cf, 1e-3)
    fg.setProjectionMatrix(pr["P"])
    pt = api.ForwardPerturbation(fg)
    pt.updateSolution(HP, factor_tol=1e-15)
    full_rank, C_full = pt.rank, pt.giveProjectedCovarU()
    pt.updateSolution(HP, factor_tol=1e-6)
    assert pt.rank < full_rank
    assert np.abs(pt.giveProjectedCovarU() - C_full).max() <= 1e-4 * np.abs(C_full).max()
    pt.close()
