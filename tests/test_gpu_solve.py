"""GPU solves against the oracle's direct solve of the reference's row-zeroed
system (SuperLU on A and A^T, the Eigen::SparseLU stand-in)."""
import numpy as np
import pytest

from oracle import oracle as O
from statfem_b200 import api
from statfem_b200 import meshgen as mg
from tests.problems import QPS, coefficients, small_mesh

pytestmark = pytest.mark.gpu


def setup(ctx, kind, n, seed, amount=0.3, faces="all", bc_vals=None):
    rng = np.random.default_rng(seed)
    mesh = small_mesh(kind, n, rng, amount)
    coeff = coefficients(mesh, rng, kind)
    gm = api.Mesh(ctx, kind, QPS[kind], mesh.coords, mesh.conn)
    gm.set_coefficients(coeff)
    s = api.SystemSolveCuda(ctx, mesh.num_dofs)
    s.assemble(gm)
    f = np.array([1.0, -0.5, 0.25])[: mesh.dof]
    s.assemble_load(gm, f)
    bc = mg.dirichlet_dofs(mesh, faces)
    vals = np.zeros(len(bc)) if bc_vals is None else bc_vals(rng, len(bc))
    s.applyConstraints((bc, vals))
    rp, col, val, F = O.fem(mesh, QPS[kind], f, bc, coeff=coeff, bc_values=vals)
    return mesh, s, O.DirectSolver(rp, col, val), F, bc


CASES = [(mg.TRI3_POISSON, 12, "all"), (mg.HEX8_POISSON, 6, "all"), (mg.HEX8_ELASTIC, 4, "x0"),
         (mg.LINE2_POISSON, 40, "x")]


@pytest.mark.parametrize("kind,n,faces", CASES)
@pytest.mark.parametrize("inhom", [False, True])
def test_forward_solve_fp64(ctx, kind, n, faces, inhom):
    bcv = (lambda rng, k: rng.standard_normal(k)) if inhom else None
    mesh, s, ds, F, bc = setup(ctx, kind, n, 1 + kind, faces=faces, bc_vals=bcv)
    s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-12)
    s.solveSystem()
    u = s.giveSolution()
    u_ref = ds.solve(F)
    st = s.last_stats()
    assert st["converged"] == 1 and st["max_rel_residual"] < 1e-11
    assert np.abs(u - u_ref).max() <= 1e-9 * np.abs(u_ref).max()


@pytest.mark.parametrize("kind,n,faces", CASES)
@pytest.mark.parametrize("method", [api.SFC_SOLVER_PCG_FP64, api.SFC_SOLVER_PCG_MIXED])
def test_transpose_solves(ctx, kind, n, faces, method):
    """solveSystemTranspose for many RHS including constrained-dof entries:
    r_c = (p_c - K_cf r_f) / scalar must match the LU solve of A^T."""
    mesh, s, ds, F, bc = setup(ctx, kind, n, 5 + kind, faces=faces)
    rng = np.random.default_rng(9)
    nr = 37
    Rhs = rng.standard_normal((nr, mesh.num_dofs))
    s.set_options(method=method, tol=1e-10, inner_tol=1e-3)
    U = s.solveSystemTranspose(Rhs)
    st = s.last_stats()
    assert st["converged"] == 1
    if method == api.SFC_SOLVER_PCG_MIXED:
        assert st["max_rel_residual"] <= 1e-10 and st["refinements"] >= 2
    for a in range(nr):
        ref = ds.solve_transpose(Rhs[a])
        assert np.abs(U[a] - ref).max() <= 1e-7 * np.abs(ref).max(), a


@pytest.mark.parametrize("bw", [32, 64, 128])
def test_block_jacobi_elasticity(ctx, bw):
    """Mixed solver with the nodal 3x3 block-Jacobi preconditioner: same
    A^-T solutions as the LU of A^T, true residual below tol."""
    mesh, s, ds, F, bc = setup(ctx, mg.HEX8_ELASTIC, 4, 17, faces="x0")
    rng = np.random.default_rng(4)
    Rhs = rng.standard_normal((45, mesh.num_dofs))
    s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-10, block_width=bw, precond=api.SFC_PRECOND_BLOCK_JACOBI)
    U = s.solveSystemTranspose(Rhs)
    st = s.last_stats()
    assert st["converged"] == 1 and st["max_rel_residual"] <= 1e-10
    refs = np.stack([ds.solve_transpose(r) for r in Rhs])
    assert np.abs(U - refs).max() <= 1e-7 * np.abs(refs).max()


def test_mixed_block_width_variants(ctx):
    mesh, s, ds, F, bc = setup(ctx, mg.TRI3_POISSON, 16, 3)
    rng = np.random.default_rng(2)
    Rhs = rng.standard_normal((130, mesh.num_dofs))
    refs = np.stack([ds.solve_transpose(r) for r in Rhs])
    for bw in (32, 64, 128):
        s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-9, block_width=bw)
        U = s.solveSystemTranspose(Rhs)
        assert np.abs(U - refs).max() <= 1e-6 * np.abs(refs).max(), bw


def test_not_converged_is_reported(ctx):
    mesh, s, ds, F, bc = setup(ctx, mg.HEX8_POISSON, 6, 4)
    s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-12, max_iter=3)
    with pytest.raises(api.SfcError) as e:
        s.solveSystem()
    assert e.value.code == -4


def test_zero_rhs_gives_zero(ctx):
    mesh, s, ds, F, bc = setup(ctx, mg.TRI3_POISSON, 6, 6)
    s.clearRhs()
    s.solveSystem()
    assert np.all(s.giveSolution() == 0.0)


@pytest.mark.parametrize("kind,n,faces", CASES)
@pytest.mark.parametrize("method", [api.SFC_SOLVER_PCG_FP64, api.SFC_SOLVER_PCG_MIXED])
def test_multi_rhs_forward(ctx, kind, n, faces, method):
    """A U = B for many right-hand sides (constrained rows included) against
    the LU solve of the row-zeroed A, for both solvers."""
    mesh, s, ds, F, bc = setup(ctx, kind, n, 7 + kind, faces=faces,
                               bc_vals=lambda rng, k: rng.standard_normal(k))
    rng = np.random.default_rng(4)
    R = rng.standard_normal((41, mesh.num_dofs))
    s.set_options(method=method, tol=1e-11, inner_tol=1e-3)
    U = s.solveSystemMulti(R)
    U_ref = np.stack([ds.solve(r) for r in R])
    assert np.abs(U - U_ref).max() <= 1e-8 * np.abs(U_ref).max()
