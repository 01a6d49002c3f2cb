"""GPU parity of element matrices, sparse assembly, loads and constraints
against the oracle: CSR pattern and values bit-exact (the kernels evaluate
the reference's expressions in the same order, without FMA contraction)."""
import numpy as np
import pytest

from oracle import oracle as O
from statfem_b200 import api
from statfem_b200 import meshgen as mg
from tests.problems import QPS, coefficients, small_mesh

pytestmark = pytest.mark.gpu

CASES = [(mg.LINE2_POISSON, 17), (mg.TRI3_POISSON, 9), (mg.HEX8_POISSON, 4), (mg.HEX8_ELASTIC, 3)]


def gpu_system(ctx, mesh, coeff, nu=0.3):
    gm = api.Mesh(ctx, mesh.kind, QPS[mesh.kind], mesh.coords, mesh.conn)
    gm.set_coefficients(coeff, poisson_ratio=nu)
    s = api.SystemSolveCuda(ctx, mesh.num_dofs)
    return gm, s


@pytest.mark.parametrize("kind,n", CASES)
@pytest.mark.parametrize("amount", [0.0, 0.4])
def test_assembly_bit_exact(ctx, kind, n, amount):
    rng = np.random.default_rng(10 + kind)
    mesh = small_mesh(kind, n, rng, amount)
    coeff = coefficients(mesh, rng, kind)
    gm, s = gpu_system(ctx, mesh, coeff)
    s.assemble(gm)
    rp, col, val = s.get_csr()
    orp, ocol, oval = O.assemble_csr(mesh, QPS[kind], coeff=coeff, nu=0.3)
    assert gm.nnz == len(ocol)
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert np.array_equal(val.view(np.uint64), oval.view(np.uint64))


@pytest.mark.parametrize("kind,n", CASES)
def test_load_and_phibar_bit_exact(ctx, kind, n):
    rng = np.random.default_rng(20 + kind)
    mesh = small_mesh(kind, n, rng, 0.3)
    coeff = coefficients(mesh, rng, kind)
    gm, s = gpu_system(ctx, mesh, coeff)
    f = np.array([0.7, -1.3, 2.1])[: mesh.dof]
    s.assemble_load(gm, f)
    F = s.giveForce()
    assert np.array_equal(F.view(np.uint64), O.assemble_load(mesh, QPS[kind], f).view(np.uint64))
    cf = api.CovarianceForcing(ctx, gm)
    bc = mg.dirichlet_dofs(mesh, "all")
    cf.applyConstraints(bc)
    ph = cf.phibar()
    assert np.array_equal(ph.view(np.uint64), O.unit_load(mesh, QPS[kind], bc).view(np.uint64))


@pytest.mark.parametrize("kind,n", CASES)
def test_constraints_row_zeroing(ctx, kind, n):
    rng = np.random.default_rng(30 + kind)
    mesh = small_mesh(kind, n)
    coeff = coefficients(mesh, rng, kind)
    gm, s = gpu_system(ctx, mesh, coeff)
    s.assemble(gm)
    s.assemble_load(gm, np.ones(mesh.dof))
    bc = mg.dirichlet_dofs(mesh, "x0" if kind == mg.HEX8_ELASTIC else "all")
    vals = rng.standard_normal(len(bc))
    s.applyConstraints((bc, vals), factor=1.5, scalar=2.0)
    rp, col, val, F = O.fem(mesh, QPS[kind], np.ones(mesh.dof), bc, coeff=coeff)
    O.apply_constraints(rp, col, val, F, bc, vals, factor=1.5, scalar=2.0)
    g_rp, g_col, g_val = s.get_csr()
    assert np.array_equal(g_val.view(np.uint64), val.view(np.uint64))
    assert np.array_equal(s.giveForce().view(np.uint64), F.view(np.uint64))


@pytest.mark.parametrize("kind,n", [(mg.TRI3_POISSON, 5), (mg.HEX8_ELASTIC, 2)])
def test_insert_path_matches_triplet_semantics(ctx, kind, n):
    """insertToMatrix per element (MatrixAssembler order) -> GPU sort/merge ==
    the oracle's triplet merge, bit for bit; clearMatrix keeps the pattern."""
    rng = np.random.default_rng(40 + kind)
    mesh = small_mesh(kind, n, rng, 0.3)
    coeff = coefficients(mesh, rng, kind)
    s = api.SystemSolveCuda(ctx, mesh.num_dofs)
    d = mesh.dof
    for e in range(mesh.num_elems):
        Ke = O.element_matrix(kind, QPS[kind], mesh.coords[mesh.conn[e]], coeff[e], 0.3)
        dofs = (mesh.conn[e][:, None].astype(np.int64) * d + np.arange(d)[None, :]).ravel()
        s.insertToMatrix(Ke, dofs, dofs)
        s.insertToRhs(np.full(len(dofs), 0.25), dofs)
    s.finishAssembly()
    rp, col, val = s.get_csr()
    orp, ocol, oval = O.assemble_csr(mesh, QPS[kind], coeff=coeff, nu=0.3)
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert np.array_equal(val.view(np.uint64), oval.view(np.uint64))
    assert s.numNonZeros() == len(ocol)
    F = s.giveForce()
    assert np.allclose(F, 0.25 * np.bincount(np.repeat(mesh.conn.ravel(), 1), minlength=mesh.num_nodes).repeat(d))
    s.clearMatrix()
    assert s.numNonZeros() == len(ocol) and s.normMatrix() == 0.0
