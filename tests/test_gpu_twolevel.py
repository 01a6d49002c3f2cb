"""Two-level preconditioner (nodal block Jacobi + rigid-body-mode coarse
correction on box aggregates): the solutions are those of the oracle's direct
solve of the reference's row-zeroed system, only the iteration counts change."""
import numpy as np
import pytest

from oracle import oracle as O
from statfem_b200 import api
from statfem_b200 import meshgen as mg
from tests.problems import QPS, coefficients, small_mesh, statfem_problem

pytestmark = pytest.mark.gpu

EL = mg.HEX8_ELASTIC


def elastic_system(ctx, n, seed, amount=0.0, bc=None, bc_vals=None, coeff=None):
    rng = np.random.default_rng(seed)
    mesh = small_mesh(EL, n, rng, amount)
    if coeff is None:
        coeff = coefficients(mesh, rng, EL)
    gm = api.Mesh(ctx, EL, QPS[EL], mesh.coords, mesh.conn)
    gm.set_coefficients(coeff)
    s = api.SystemSolveCuda(ctx, mesh.num_dofs)
    s.assemble(gm)
    f = np.array([0.3, -0.5, 1.0])
    s.assemble_load(gm, f)
    if bc is None:
        bc = mg.dirichlet_dofs(mesh, "x0")
    vals = np.zeros(len(bc)) if bc_vals is None else bc_vals
    s.applyConstraints((bc, vals))
    rp, col, val, F = O.fem(mesh, QPS[EL], f, bc, coeff=coeff, bc_values=vals)
    return mesh, gm, s, O.DirectSolver(rp, col, val), F, f


@pytest.mark.parametrize("amount", [0.0, 0.3])
def test_forward_fp64_two_level(ctx, amount):
    mesh, gm, s, ds, F, f = elastic_system(ctx, 12, 3, amount)
    u_ref = ds.solve(F)
    s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-12, precond=api.SFC_PRECOND_JACOBI)
    s.solveSystem()
    it_jacobi = s.last_stats()["iterations"]
    s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-12, precond=api.SFC_PRECOND_TWO_LEVEL, coarse_size=4)
    s.solveSystem()
    st = s.last_stats()
    u = s.giveSolution()
    assert st["converged"] == 1 and st["max_rel_residual"] < 1e-11
    assert st["coarse_dofs"] > 0 and st["coarse_dofs"] % 6 == 0
    assert np.abs(u - u_ref).max() <= 1e-9 * np.abs(u_ref).max()
    assert st["iterations"] < 0.6 * it_jacobi, (st["iterations"], it_jacobi)


@pytest.mark.parametrize("bw", [32, 128])
def test_transpose_mixed_two_level(ctx, bw):
    mesh, gm, s, ds, F, f = elastic_system(ctx, 12, 5)
    rng = np.random.default_rng(4)
    Rhs = rng.standard_normal((45, mesh.num_dofs))
    refs = np.stack([ds.solve_transpose(r) for r in Rhs])
    s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-10, block_width=bw, precond=api.SFC_PRECOND_BLOCK_JACOBI)
    s.solveSystemTranspose(Rhs)
    it_bj = s.last_stats()["iterations"]
    s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-10, block_width=bw, precond=api.SFC_PRECOND_TWO_LEVEL,
                  coarse_size=4)
    U = s.solveSystemTranspose(Rhs)
    st = s.last_stats()
    assert st["converged"] == 1 and st["max_rel_residual"] <= 1e-10
    assert st["coarse_dofs"] > 0
    assert np.abs(U - refs).max() <= 1e-7 * np.abs(refs).max()
    assert st["iterations"] < it_bj, (st["iterations"], it_bj)


@pytest.mark.parametrize("amount,bw", [(0.0, 128), (0.3, 64), (0.3, 32)])
def test_fused_r_update_and_restriction(ctx, amount, bw):
    """The r update fused with the coarse restriction (the default) and the
    two separate kernels (SFC_RESTRICT=separate) both give the direct solve's
    answer; their FP32 sums differ only in order, so the iteration counts
    stay close."""
    import os

    mesh, gm, s, ds, F, f = elastic_system(ctx, 11, 6, amount)
    rng = np.random.default_rng(2)
    Rhs = rng.standard_normal((70, mesh.num_dofs))
    refs = np.stack([ds.solve_transpose(r) for r in Rhs])
    out = {}
    for mode in ("fused", "separate"):
        if mode == "separate":
            os.environ["SFC_RESTRICT"] = "separate"
        try:
            s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-10, block_width=bw,
                          precond=api.SFC_PRECOND_TWO_LEVEL, coarse_size=4)
            out[mode] = (s.solveSystemTranspose(Rhs), s.last_stats())
        finally:
            os.environ.pop("SFC_RESTRICT", None)
    for U, st in out.values():
        assert st["converged"] == 1 and st["max_rel_residual"] <= 1e-10
        assert st["coarse_dofs"] > 0
        assert np.abs(U - refs).max() <= 1e-7 * np.abs(refs).max()
    itf, its = out["fused"][1]["iterations"], out["separate"][1]["iterations"]
    assert abs(itf - its) <= max(8, its // 5), (itf, its)


@pytest.mark.parametrize("precond", [api.SFC_PRECOND_BLOCK_JACOBI, api.SFC_PRECOND_TWO_LEVEL])
def test_convergence_inside_a_check_interval(ctx, precond):
    """With a check interval longer than a whole FP32 stretch, the
    per-iteration convergence test stops each captured interval where the
    columns' recurrence converges (the reliable update then follows): the
    iteration count is the one that ran, not a multiple of the interval, close
    between the graph and separate launches (their FP64 column sums add in
    different orders), and the answer is the direct solve's."""
    import os

    mesh, gm, s, ds, F, f = elastic_system(ctx, 8, 9)
    rng = np.random.default_rng(5)
    Rhs = rng.standard_normal((40, mesh.num_dofs))
    refs = np.stack([ds.solve_transpose(r) for r in Rhs])
    check = 400
    out = {}
    for mode in ("graph", "eager"):
        if mode == "eager":
            os.environ["SFC_BLOCK_GRAPH"] = "0"
        try:
            s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-9, block_width=64, precond=precond,
                          coarse_size=4, check_every=check)
            out[mode] = (s.solveSystemTranspose(Rhs), s.last_stats())
        finally:
            os.environ.pop("SFC_BLOCK_GRAPH", None)
    for U, st in out.values():
        assert st["converged"] == 1 and st["max_rel_residual"] <= 1e-9, st
        assert st["iterations"] > 0 and st["iterations"] % check != 0, st
        assert np.abs(U - refs).max() <= 1e-6 * np.abs(refs).max()
    assert abs(out["graph"][1]["iterations"] - out["eager"][1]["iterations"]) <= 4


def test_multi_rhs_inhomogeneous_two_level(ctx):
    rng = np.random.default_rng(8)
    mesh = small_mesh(EL, 10)
    bc = mg.dirichlet_dofs(mesh, "x0")
    mesh, gm, s, ds, F, f = elastic_system(ctx, 10, 8, 0.2, bc=bc, bc_vals=rng.standard_normal(len(bc)))
    R = rng.standard_normal((40, mesh.num_dofs))
    s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-11, inner_tol=1e-3, precond=api.SFC_PRECOND_TWO_LEVEL,
                  coarse_size=3)
    U = s.solveSystemMulti(R)
    U_ref = np.stack([ds.solve(r) for r in R])
    assert np.abs(U - U_ref).max() <= 1e-8 * np.abs(U_ref).max()
    s.solveSystem()
    u_ref = ds.solve(F)
    assert np.abs(s.giveSolution() - u_ref).max() <= 1e-7 * np.abs(u_ref).max()


def test_fully_constrained_aggregates_are_dropped(ctx):
    """A slab of fully constrained nodes leaves aggregates whose modes vanish:
    their coarse dofs are dropped from the inverse and the solve is unchanged."""
    mesh = small_mesh(EL, 12)
    s0 = elastic_system(ctx, 12, 11)[2]
    s0.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-11, precond=api.SFC_PRECOND_TWO_LEVEL, coarse_size=4)
    s0.solveSystem()
    full = s0.last_stats()["coarse_dofs"]
    slab = np.nonzero(mesh.coords[:, 0] < 0.34)[0]
    bc = np.sort(np.concatenate([3 * slab, 3 * slab + 1, 3 * slab + 2]))
    mesh, gm, s, ds, F, f = elastic_system(ctx, 12, 11, bc=bc)
    for method in (api.SFC_SOLVER_PCG_FP64, api.SFC_SOLVER_PCG_MIXED):
        s.set_options(method=method, tol=1e-11, precond=api.SFC_PRECOND_TWO_LEVEL, coarse_size=4)
        s.solveSystem()
        st = s.last_stats()
        assert 0 < st["coarse_dofs"] < full
        u_ref = ds.solve(F)
        assert np.abs(s.giveSolution() - u_ref).max() <= 1e-8 * np.abs(u_ref).max()


@pytest.mark.parametrize("size", [2, 5, 100])
def test_coarse_sizes(ctx, size):
    """From many small aggregates to a single one (six global modes)."""
    mesh, gm, s, ds, F, f = elastic_system(ctx, 8, 12)
    s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-12, precond=api.SFC_PRECOND_TWO_LEVEL, coarse_size=size)
    s.solveSystem()
    st = s.last_stats()
    u_ref = ds.solve(F)
    assert st["converged"] == 1 and np.abs(s.giveSolution() - u_ref).max() <= 1e-9 * np.abs(u_ref).max()
    if size == 100:
        assert st["coarse_dofs"] == 6


def test_rebuilt_after_coefficient_change(ctx):
    """The coarse inverse follows the operator: new coefficients, new answer."""
    mesh, gm, s, ds, F, f = elastic_system(ctx, 10, 13)
    s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-10, precond=api.SFC_PRECOND_TWO_LEVEL, coarse_size=4)
    s.solveSystem()
    rng = np.random.default_rng(14)
    coeff2 = np.exp(0.8 * rng.standard_normal(mesh.num_elems))
    gm.set_coefficients(coeff2)
    s.assemble(gm)
    s.clearRhs()
    s.assemble_load(gm, f)
    bc = mg.dirichlet_dofs(mesh, "x0")
    s.applyConstraints((bc, np.zeros(len(bc))))
    s.solveSystem()
    rp, col, val, F2 = O.fem(mesh, QPS[EL], f, bc, coeff=coeff2)
    u_ref = O.DirectSolver(rp, col, val).solve(F2)
    assert np.abs(s.giveSolution() - u_ref).max() <= 1e-8 * np.abs(u_ref).max()


SCALAR = [(mg.LINE2_POISSON, 200, "x"), (mg.TRI3_POISSON, 24, "all"), (mg.HEX8_POISSON, 10, "all")]


def poisson_system(ctx, kind, n, faces, seed):
    rng = np.random.default_rng(seed)
    mesh = small_mesh(kind, n, rng, 0.2 if kind != mg.LINE2_POISSON else 0.0)
    coeff = coefficients(mesh, rng, kind)
    gm = api.Mesh(ctx, kind, QPS[kind], mesh.coords, mesh.conn)
    gm.set_coefficients(coeff)
    s = api.SystemSolveCuda(ctx, mesh.num_dofs)
    s.assemble(gm)
    s.assemble_load(gm, np.array([1.0]))
    bc = mg.dirichlet_dofs(mesh, faces)
    s.applyConstraints((bc, np.zeros(len(bc))))
    rp, col, val, F = O.fem(mesh, QPS[kind], np.array([1.0]), bc, coeff=coeff)
    return mesh, s, O.DirectSolver(rp, col, val), F


@pytest.mark.parametrize("kind,n,faces", SCALAR)
def test_scalar_two_level_forward_and_transpose(ctx, kind, n, faces):
    """Scalar (Poisson) meshes: point Jacobi plus one constant mode per box
    aggregate, in the FP64 PCG and in the mixed block solver."""
    mesh, s, ds, F = poisson_system(ctx, kind, n, faces, 30 + kind)
    u_ref = ds.solve(F)
    s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-12, precond=api.SFC_PRECOND_JACOBI)
    s.solveSystem()
    it_jacobi = s.last_stats()["iterations"]
    s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-12, precond=api.SFC_PRECOND_TWO_LEVEL, coarse_size=4)
    s.solveSystem()
    st = s.last_stats()
    assert st["converged"] == 1 and st["coarse_dofs"] > 0
    assert np.abs(s.giveSolution() - u_ref).max() <= 1e-9 * np.abs(u_ref).max()
    assert st["iterations"] < it_jacobi, (st["iterations"], it_jacobi)
    rng = np.random.default_rng(5)
    Rhs = rng.standard_normal((40, mesh.num_dofs))
    s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-10, inner_tol=1e-3, precond=api.SFC_PRECOND_TWO_LEVEL,
                  coarse_size=4)
    U = s.solveSystemTranspose(Rhs)
    st = s.last_stats()
    assert st["converged"] == 1 and st["coarse_dofs"] > 0 and st["max_rel_residual"] <= 1e-10
    refs = np.stack([ds.solve_transpose(r) for r in Rhs])
    assert np.abs(U - refs).max() <= 1e-7 * np.abs(refs).max()


def test_scalar_coarse_size_matches_oracle_boxes(ctx):
    from oracle import coarse_ref as C
    mesh, s, ds, F = poisson_system(ctx, mg.HEX8_POISSON, 12, "all", 41)
    s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-10, precond=api.SFC_PRECOND_TWO_LEVEL, coarse_size=3)
    s.solveSystem()
    agg, _ = C.box_aggregates(mesh.coords, 3, max_aggs=2048)
    assert s.last_stats()["coarse_dofs"] == int(agg.max()) + 1


def test_triplet_system_has_no_coarse_space(ctx):
    """A system assembled from element triplets (no mesh attached) has no
    aggregates: the solver runs its one-level preconditioner and reports no
    coarse dofs."""
    rng = np.random.default_rng(2)
    kind = mg.TRI3_POISSON
    mesh = small_mesh(kind, 8, rng, 0.2)
    coeff = coefficients(mesh, rng, kind)
    s = api.SystemSolveCuda(ctx, mesh.num_dofs)
    for e in range(mesh.num_elems):
        Ke = O.element_matrix(kind, QPS[kind], mesh.coords[mesh.conn[e]], coeff[e], 0.3)
        dofs = mesh.conn[e].astype(np.int64)
        s.insertToMatrix(Ke, dofs, dofs)
        s.insertToRhs(np.full(len(dofs), 0.25), dofs)
    s.finishAssembly()
    bc = mg.dirichlet_dofs(mesh, "all")
    s.applyConstraints((bc, np.zeros(len(bc))))
    s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-10, precond=api.SFC_PRECOND_TWO_LEVEL)
    s.solveSystem()
    st = s.last_stats()
    rp, col, val = O.assemble_csr(mesh, QPS[kind], coeff=coeff, nu=0.3)
    F = 0.25 * np.bincount(mesh.conn.ravel(), minlength=mesh.num_nodes).astype(np.float64)
    O.apply_constraints(rp, col, val, F, bc)
    u_ref = O.DirectSolver(rp, col, val).solve(F)
    assert st["coarse_dofs"] == 0
    assert np.abs(s.giveSolution() - u_ref).max() <= 1e-8 * np.abs(u_ref).max()


def test_statfem_posterior_two_level(ctx):
    """ForwardGaussRHS / LikelihoodKOH on elasticity: the sensor-space prior and
    posterior do not depend on the preconditioner."""
    pb = statfem_problem(EL, 8, 24, seed=21, faces="x0")
    mesh = pb["mesh"]
    hp = {"forcing.sigma": 0.05, "forcing.length": 0.3, "rho": 1.0, "mismatch.sigma": 0.01,
          "mismatch.length": 0.25, "mismatch.sensorEps": 1e-4}
    out = []
    for precond in (api.SFC_PRECOND_BLOCK_JACOBI, api.SFC_PRECOND_TWO_LEVEL):
        gm = api.Mesh(ctx, EL, 8, mesh.coords, mesh.conn)
        gm.set_coefficients(pb["coeff"])
        s = api.SystemSolveCuda(ctx, mesh.num_dofs)
        s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-10, precond=precond, coarse_size=3)
        s.assemble(gm)
        s.assemble_load(gm, np.array([0.0, 0.0, -1.0]))
        s.applyConstraints((pb["bc"], np.zeros(len(pb["bc"]))))
        s.solveSystem()
        cf = api.CovarianceForcing(ctx, gm)
        cf.applyConstraints(pb["bc"])
        fg = api.ForwardGaussRHS(s, cf, 1e-3)
        fg.setProjectionMatrix(pb["P"])
        fg.updateSolution(hp)
        if precond == api.SFC_PRECOND_TWO_LEVEL:
            assert s.last_stats()["coarse_dofs"] > 0
        out.append((fg.giveProjectedMeanU(), fg.giveProjectedCovarU()))
    (m0, c0), (m1, c1) = out
    assert np.abs(m1 - m0).max() <= 1e-8 * np.abs(m0).max()
    assert np.abs(c1 - c0).max() <= 1e-7 * np.abs(c0).max()


@pytest.mark.parametrize("size", [3, 4, 6])
def test_coarse_space_size_matches_oracle_boxes(ctx, size):
    """The library's box grid is the oracle's (oracle/coarse_ref.py): six
    coarse dofs per non-empty box when no box is fully constrained."""
    from oracle import coarse_ref as C
    mesh, gm, s, ds, F, f = elastic_system(ctx, 12, 15)
    s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-10, precond=api.SFC_PRECOND_TWO_LEVEL, coarse_size=size)
    s.solveSystem()
    agg, _ = C.box_aggregates(mesh.coords, size)
    assert s.last_stats()["coarse_dofs"] == 6 * (int(agg.max()) + 1)
