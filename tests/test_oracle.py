"""CPU tests: the oracle against the reference's golden vectors and against
properties the reference's arithmetic guarantees."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from statfem_b200 import meshgen as mg

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_kat2_gaussian_process():
    """statX/apps/reference/gaussianProcess watchdog: ExpKernel + LLT log-det
    (watchDog.0.mk ERRTOL = 1e-8)."""
    g = np.load(os.path.join(GOLDEN, "kat2_gaussianProcess.npz"))
    m, v, ll = O.gp_regression(g["x_train"], g["y_train"], g["x_pred"][:, None], float(g["sigma"]),
                               float(g["length"]), float(g["eps"]))
    assert np.max(np.abs(m - g["expected_mean"])) < 1e-8
    assert np.max(np.abs(v - g["expected_var"])) < 1e-8
    assert abs(ll - float(g["expected_loglik"])) < 1e-8


def kat1_oracle():
    k = np.load(os.path.join(GOLDEN, "kat1_laplaceRHSinfer.npz"))
    mesh = mg.Mesh(mg.LINE2_POISSON, k["coords"], k["conn"], grid=(len(k["conn"]),))
    bc = mg.dirichlet_dofs(mesh, "x")
    coeff = np.full(mesh.num_elems, float(k["conductivity"]))
    pr = O.statfem_prior(mesh, 3, float(k["force"]), bc, k["P"], float(k["forcing_sigma"]),
                         float(k["forcing_length"]), float(k["reg"]), coeff=coeff)
    Ks = O.mismatch_covariance(k["sensor_coords"], float(k["mismatch_sigma"]), float(k["mismatch_length"]),
                               float(k["sensor_eps"]))
    N = mesh.num_dofs
    meanU, Cu, _ = O.forward_gauss_rhs(pr["solver"], pr["F"], np.eye(N), mesh.coords, pr["phibar"], 1, 1,
                                       float(k["forcing_sigma"]), float(k["forcing_length"]), float(k["reg"]))
    mean, cov = O.koh_woodbury(pr["C_s"], Ks, k["Y"], float(k["rho"]), k["P"], Cu, meanU)
    return k, mean


def test_kat1_laplace_rhs_infer():
    """laplaceRHSinfer watchdog posterior mean (33 values printed to 6 digits;
    the hyperparameters are the watchdog's 6-digit means) -> tol 1e-6 abs."""
    k, mean = kat1_oracle()
    assert np.max(np.abs(mean - k["expected_mean"])) < 1e-6


@pytest.mark.parametrize("kind,qps,total", [(mg.LINE2_POISSON, 3, 1.0), (mg.TRI3_POISSON, 3, 0.5),
                                            (mg.HEX8_POISSON, 8, 1.0), (mg.HEX8_ELASTIC, 8, 1.0)])
def test_quadrature_tables(kind, qps, total):
    w, pts = O.quadrature(kind, qps)
    assert len(w) == qps
    assert abs(w.sum() - total) < 1e-14
    if kind == mg.TRI3_POISSON:
        assert w[0] == 0.166666666666666  # truncated literal, corlib/SimplexQuadrature.hpp:181
    if kind in (mg.HEX8_POISSON, mg.HEX8_ELASTIC):
        assert pts[0, 0] == 0.788675134594813 and pts[1, 0] == 0.211324865405187  # x fastest, descending


@pytest.mark.parametrize("kind", [mg.LINE2_POISSON, mg.TRI3_POISSON, mg.HEX8_POISSON, mg.HEX8_ELASTIC])
def test_element_matrix_properties(kind):
    rng = np.random.default_rng(1)
    m = mg.bar(1) if kind == 1 else mg.unit_square_tri(1) if kind == 2 else mg.unit_cube_hex(1, kind)
    X = m.coords[m.conn[0]] + 0.05 * rng.standard_normal((m.conn.shape[1], 3))
    if m.dim < 3:
        X[:, m.dim:] = 0
    Ke = O.element_matrix(kind, {1: 3, 2: 3, 3: 8, 4: 8}[kind], X, coeff=1.7, nu=0.3)
    assert np.allclose(Ke, Ke.T, rtol=0, atol=1e-12 * np.abs(Ke).max())
    # constants (and, for elasticity, rigid translations) are in the kernel
    d = m.dof
    for c in range(d):
        v = np.zeros(Ke.shape[0])
        v[c::d] = 1.0
        assert np.abs(Ke @ v).max() < 1e-12 * np.abs(Ke).max()
    assert np.linalg.eigvalsh(0.5 * (Ke + Ke.T)).min() > -1e-10 * np.abs(Ke).max()


def test_c1_pattern_size_matches_formula():
    m = mg.unit_square_tri(8)
    rp, col, val = O.assemble_csr(m, 3)
    n = 9
    assert len(col) == n * n + 2 * (2 * n * (n - 1) + (n - 1) ** 2)
    for i in range(m.num_dofs):  # sorted, unique columns per row
        c = col[rp[i]:rp[i + 1]]
        assert np.all(np.diff(c) > 0)


def test_row_zero_constraints_and_transpose_solve():
    """Row-zeroed system vs symmetric elimination: same u, and A^-T p differs
    only on constrained dofs (SystemSolveEigenSparse.hpp:197-215, 364-404)."""
    m = mg.unit_square_tri(6)
    bc = mg.dirichlet_dofs(m, "all")
    rp, col, val, F = O.fem(m, 3, 1.0, bc)
    for c in bc:
        row = col[rp[c]:rp[c + 1]]
        v = val[rp[c]:rp[c + 1]]
        assert np.all(v[row != c] == 0) and v[row == c][0] == 1.0
        assert F[c] == 0.0
    ds = O.DirectSolver(rp, col, val)
    u = ds.solve(F)
    mask = np.zeros(m.num_dofs, dtype=np.uint8)
    mask[bc] = 1
    x, it = O.pcg(rp, col, val, mask, F, tol=1e-13)
    assert it > 0 and np.abs(x - u).max() < 1e-11


def test_meshgen_projection_rows_sum_to_one():
    rng = np.random.default_rng(3)
    for m in (mg.unit_square_tri(5), mg.unit_cube_hex(4), mg.bar(7)):
        pts = mg.interior_points(rng, 11, m.dim)
        ip, ix, dv = mg.projection_matrix(m, pts)
        P = mg.projection_dense(m, ip, ix, dv)
        assert np.allclose(P.sum(axis=1), 1.0)
        # the projection reproduces linear fields exactly
        assert np.allclose(P @ m.coords[:, 0], pts[:, 0])


def test_se_field_tensor_matches_kernel_covariance():
    rng = np.random.default_rng(0)
    ax = [np.linspace(0, 1, 5), np.linspace(0, 1, 4)]
    S = np.stack([mg.se_field_tensor(rng, ax, 0.7, 0.3) for _ in range(20000)])
    X = np.stack(np.meshgrid(ax[0], ax[1], indexing="xy"), axis=-1).reshape(-1, 2)
    K = O.se_matrix(X, X, 0.7, 0.3)
    assert np.abs(np.cov(S.T) - K).max() < 0.03


def test_perturbation_oracle_reduces_to_forcing_only():
    """With zero material variance the perturbation covariance is the
    ForwardGaussRHS covariance without its regularisation term; it is
    symmetric positive semidefinite otherwise."""
    from tests.problems import statfem_problem
    pr = statfem_problem(mg.TRI3_POISSON, 5, 4, seed=2)
    mesh = pr["mesh"]
    rp, col, val, F = O.fem(mesh, 3, 1.0, pr["bc"], coeff=pr["coeff"])
    phibar = O.unit_load(mesh, 3, pr["bc"])
    Pd = mg.projection_dense(mesh, *pr["P"])
    solver = O.DirectSolver(rp, col, val)
    mean0, C0, _ = O.forward_gauss_rhs(solver, F, Pd, mesh.coords, phibar, 2, 1, 0.1, 0.2, 0.0)
    m, C = O.forward_perturbation(mesh, 3, F, rp, col, val, pr["bc"], Pd, phibar, 0.1, 0.2, 0.0, 0.3, 1e-4)
    np.testing.assert_allclose(m, mean0, rtol=1e-10)
    np.testing.assert_allclose(C, C0, rtol=1e-9, atol=1e-14)
    m, C = O.forward_perturbation(mesh, 3, F, rp, col, val, pr["bc"], Pd, phibar, 0.1, 0.2, 0.5, 0.3, 1e-4)
    assert np.allclose(C, C.T, rtol=1e-10, atol=1e-16)
    assert np.linalg.eigvalsh(C).min() > -1e-12 * np.abs(C).max()
    assert (np.diag(C) > np.diag(C0)).all()
