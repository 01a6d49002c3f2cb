"""CPU checks of the two-level preconditioner's algorithm (oracle/coarse_ref.py):
the block Gauss-Jordan inverse with dropped pivots, and PCG with the
preconditioner reaching the direct solution of an elasticity system."""
import numpy as np
import scipy.sparse as sp

from oracle import coarse_ref as C
from oracle import oracle as O
from statfem_b200 import meshgen as mg


def test_gauss_jordan_spd_inverse_and_logdet():
    rng = np.random.default_rng(0)
    n = 100  # several 32-wide panels and a ragged last one
    B = rng.standard_normal((n, n))
    A = B @ B.T + n * np.eye(n)
    Ainv, piv, dropped = C.gauss_jordan_inverse(A, 0.0)
    assert dropped == 0
    assert np.abs(Ainv - np.linalg.inv(A)).max() <= 1e-12 * np.abs(np.linalg.inv(A)).max()
    sign, logdet = np.linalg.slogdet(A)
    assert abs(np.log(piv).sum() - logdet) <= 1e-10 * abs(logdet)


def test_gauss_jordan_drops_dependent_and_empty_pivots():
    rng = np.random.default_rng(1)
    n, rank = 80, 50
    P = rng.standard_normal((n, rank))
    A = P @ P.T
    A[7, :] = 0.0
    A[:, 7] = 0.0  # a mode that vanishes entirely (a fully constrained aggregate)
    Ainv, piv, dropped = C.gauss_jordan_inverse(A, 1e-10)
    assert dropped == n - np.linalg.matrix_rank(A)
    assert np.abs(Ainv - Ainv.T).max() <= 1e-10 * np.abs(Ainv).max()
    assert np.abs(A @ Ainv @ A - A).max() <= 1e-9 * np.abs(A).max()  # a generalised inverse
    assert np.linalg.eigvalsh(0.5 * (Ainv + Ainv.T)).min() >= -1e-9 * np.abs(Ainv).max()


def eliminated_operator(mesh, bc, coeff):
    rp, col, val, F = O.fem(mesh, 8, np.array([0.3, -0.5, 1.0]), bc, coeff=coeff)
    N = mesh.num_dofs
    A = sp.csr_matrix((val, col, rp), shape=(N, N)).tocoo()
    mask = np.zeros(N, bool)
    mask[bc] = True
    keep = ~((mask[A.row] | mask[A.col]) & (A.row != A.col))
    S = sp.csr_matrix((A.data[keep], (A.row[keep], A.col[keep])), shape=(N, N))
    b = F.copy()
    b[mask] = 0.0
    return S, b, mask, (rp, col, val, F)


def test_two_level_pcg_reaches_the_direct_solution():
    rng = np.random.default_rng(3)
    mesh = mg.unit_cube_hex(8, mg.HEX8_ELASTIC)
    coeff = np.exp(0.3 * rng.standard_normal(mesh.num_elems))
    bc = mg.dirichlet_dofs(mesh, "x0")
    S, b, mask, (rp, col, val, F) = eliminated_operator(mesh, bc, coeff)
    M = C.TwoLevel(S, mesh.coords, mask, size=4)
    assert M.coarse_dofs == 6 * 8  # 2 x 2 x 2 boxes of 4-5 nodes per axis
    # M is a fixed symmetric positive definite operator
    u, v = rng.standard_normal((2, mesh.num_dofs))
    assert abs(u @ M(v) - v @ M(u)) <= 1e-10 * abs(u @ M(v))
    assert u @ M(u) > 0
    x, it2 = C.pcg(S, b, M, tol=1e-10)
    Dinv = C.nodal_block_jacobi(S)
    _, it1 = C.pcg(S, b, lambda r: np.einsum('nij,nj->ni', Dinv, r.reshape(-1, 3)).ravel(), tol=1e-10)
    u_ref = O.DirectSolver(rp, col, val).solve(F)
    free = ~mask
    assert np.abs(x[free] - u_ref[free]).max() <= 1e-8 * np.abs(u_ref).max()
    assert it2 < it1


def test_fully_constrained_boxes_are_dropped():
    rng = np.random.default_rng(4)
    mesh = mg.unit_cube_hex(8, mg.HEX8_ELASTIC)
    coeff = np.exp(0.3 * rng.standard_normal(mesh.num_elems))
    slab = np.nonzero(mesh.coords[:, 0] < 0.3)[0]
    bc = np.sort(np.concatenate([3 * slab, 3 * slab + 1, 3 * slab + 2]))
    S, b, mask, (rp, col, val, F) = eliminated_operator(mesh, bc, coeff)
    M = C.TwoLevel(S, mesh.coords, mask, size=2)
    assert M.dropped > 0
    x, _ = C.pcg(S, b, M, tol=1e-10)
    u_ref = O.DirectSolver(rp, col, val).solve(F)
    free = ~mask
    assert np.abs(x[free] - u_ref[free]).max() <= 1e-8 * np.abs(u_ref).max()


def test_scalar_two_level_pcg_reaches_the_direct_solution():
    """Poisson: point Jacobi plus one constant per box aggregate."""
    rng = np.random.default_rng(5)
    mesh = mg.unit_square_tri(24)
    coeff = np.exp(0.5 * rng.standard_normal(mesh.num_elems))
    bc = mg.dirichlet_dofs(mesh, "all")
    rp, col, val, F = O.fem(mesh, 3, np.array([1.0]), bc, coeff=coeff)
    N = mesh.num_dofs
    A = sp.csr_matrix((val, col, rp), shape=(N, N)).tocoo()
    mask = np.zeros(N, bool)
    mask[bc] = True
    keep = ~((mask[A.row] | mask[A.col]) & (A.row != A.col))
    S = sp.csr_matrix((A.data[keep], (A.row[keep], A.col[keep])), shape=(N, N))
    b = F.copy()
    b[mask] = 0.0
    M = C.TwoLevel(S, mesh.coords, mask, size=4, dof=1)
    agg, _ = C.box_aggregates(mesh.coords, 4, max_aggs=2048)
    assert M.Ac.shape[0] == int(agg.max()) + 1
    x, it2 = C.pcg(S, b, M, tol=1e-10)
    dinv = 1.0 / S.diagonal()
    _, it1 = C.pcg(S, b, lambda r: dinv * r, tol=1e-10)
    u_ref = O.DirectSolver(rp, col, val).solve(F)
    free = ~mask
    assert np.abs(x[free] - u_ref[free]).max() <= 1e-8 * np.abs(u_ref).max()
    assert it2 < 0.7 * it1, (it2, it1)


# ---- the library's host-side aggregation (no device needed) ----------------
import pytest  # noqa: E402

from statfem_b200 import api  # noqa: E402


@pytest.mark.parametrize("mesh,size,max_aggs", [
    (mg.unit_cube_hex(12, mg.HEX8_ELASTIC), 4, 512),
    (mg.unit_cube_hex(12, mg.HEX8_POISSON), 3, 2048),
    (mg.unit_square_tri(24), 4, 2048),
    (mg.bar(200), 4, 2048),
])
def test_library_boxes_match_the_oracle(mesh, size, max_aggs):
    agg, nb = api.coarse_boxes(mesh.coords, mesh.conn, size=size, max_aggs=max_aggs)
    ref, _ = C.box_aggregates(mesh.coords, size, max_aggs=max_aggs)
    assert np.array_equal(agg, ref)


def test_boxes_coarsen_until_every_element_spans_one_box():
    """A graded bar whose last element is longer than the boxes: the grid is
    halved until no element reaches past a neighbouring box."""
    x = np.concatenate([np.linspace(0.0, 0.1, 41), [1.0]])
    coords = np.zeros((len(x), 3))
    coords[:, 0] = x
    conn = np.stack([np.arange(len(x) - 1), np.arange(1, len(x))], axis=1).astype(np.uint32)
    agg, nb = api.coarse_boxes(coords, conn, size=2, max_aggs=2048)
    first = int(np.rint(1.0 / (1.0 / min(2048, len(x) / 2.0))))  # the grid before coarsening
    assert nb[0] < first and nb[1] == nb[2] == 1
    box = np.minimum(np.floor(x * nb[0]).astype(int), nb[0] - 1)
    assert np.all(np.abs(box[conn[:, 0]] - box[conn[:, 1]]) <= 1)
    assert agg.max() + 1 == len(np.unique(box))


def test_boxes_reject_a_degenerate_node_set():
    coords = np.zeros((4, 3))
    conn = np.array([[0, 1], [2, 3]], dtype=np.uint32)
    with pytest.raises(api.SfcError):
        api.coarse_boxes(coords, conn)
