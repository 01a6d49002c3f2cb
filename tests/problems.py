"""Seeded test problems shared by the CPU and GPU tests."""
import numpy as np

from statfem_b200 import meshgen as mg

QPS = {mg.LINE2_POISSON: 3, mg.TRI3_POISSON: 3, mg.HEX8_POISSON: 8, mg.HEX8_ELASTIC: 8}


def distort(mesh, rng, amount):
    """Move interior nodes randomly (keeps boundary nodes on the boundary and
    every Jacobian positive for amount < ~0.3 of the cell size)."""
    X = mesh.coords.copy()
    d = mesh.dim
    h = 1.0 / mesh.grid[0]
    inner = np.all((X[:, :d] > 1e-9) & (X[:, :d] < 1 - 1e-9), axis=1)
    X[inner, :d] += amount * h * (rng.random((inner.sum(), d)) - 0.5)
    return mg.Mesh(mesh.kind, X, mesh.conn, grid=mesh.grid)


def small_mesh(kind, n, rng=None, amount=0.0):
    if kind == mg.LINE2_POISSON:
        m = mg.bar(n)
    elif kind == mg.TRI3_POISSON:
        m = mg.unit_square_tri(n)
    else:
        m = mg.unit_cube_hex(n, kind)
    if rng is not None and amount > 0:
        m = distort(m, rng, amount)
    return m


def coefficients(mesh, rng, kind):
    if kind == mg.HEX8_ELASTIC:
        return np.exp(0.3 * rng.standard_normal(mesh.num_elems))
    return np.exp(0.5 * rng.standard_normal(mesh.num_elems))


def statfem_problem(kind, n, ns, seed=0, amount=0.0, faces="all"):
    """Mesh, coefficients, Dirichlet dofs, sensors and projection rows."""
    rng = np.random.default_rng(seed)
    mesh = small_mesh(kind, n, rng, amount)
    coeff = coefficients(mesh, rng, kind)
    bc = mg.dirichlet_dofs(mesh, faces)
    pts = mg.interior_points(rng, ns, mesh.dim, margin=0.05)
    comps = (np.arange(ns) % mesh.dof) if mesh.dof > 1 else None
    P = mg.projection_matrix(mesh, pts if mesh.grid is not None and amount == 0 else pts, comps)
    return dict(mesh=mesh, coeff=coeff, bc=bc, pts=pts, P=P, rng=rng)
