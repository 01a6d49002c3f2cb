"""Seeded synthetic inputs for the statFEM forward-and-conditioning path.

Structured meshes with SMF-compatible numbering (the node/element order a
``corlib::Mesh`` read from an SMF file would have, corlib/Mesh.ipp:63-102),
Dirichlet dof lists in the order ``corlib::ConstraintFunctor`` collects them
(node order, then component), sensor projection rows built from the element
shape functions (the reference reads P from a file, ioHelpers.hpp:85-120; here
the rows are the shape-function weights at the sensor point), and
squared-exponential random fields sampled exactly on tensor grids.

This module is host-side input generation shared by the tests, the oracle and
the benchmark; it computes nothing on the hot path.
"""
from __future__ import annotations

import numpy as np

LINE2_POISSON = 1
TRI3_POISSON = 2
HEX8_POISSON = 3
HEX8_ELASTIC = 4

NODES_PER_ELEM = {LINE2_POISSON: 2, TRI3_POISSON: 3, HEX8_POISSON: 8, HEX8_ELASTIC: 8}
DIM = {LINE2_POISSON: 1, TRI3_POISSON: 2, HEX8_POISSON: 3, HEX8_ELASTIC: 3}
DOFS_PER_NODE = {LINE2_POISSON: 1, TRI3_POISSON: 1, HEX8_POISSON: 1, HEX8_ELASTIC: 3}


class Mesh:
    """Nodes (num_nodes x 3, SMF layout) and connectivity (num_elems x nn)."""

    def __init__(self, kind, coords, conn, grid=None):
        self.kind = kind
        self.coords = np.ascontiguousarray(coords, dtype=np.float64)
        self.conn = np.ascontiguousarray(conn, dtype=np.uint32)
        self.grid = grid  # cells per axis for structured meshes

    @property
    def num_nodes(self):
        return self.coords.shape[0]

    @property
    def num_elems(self):
        return self.conn.shape[0]

    @property
    def dim(self):
        return DIM[self.kind]

    @property
    def dof(self):
        return DOFS_PER_NODE[self.kind]

    @property
    def num_dofs(self):
        return self.num_nodes * self.dof

    def centroids(self):
        return self.coords[self.conn].mean(axis=1)


def bar(num_elems=32, kind=LINE2_POISSON):
    """1-D bar on [0,1] with equally spaced 2-node line elements."""
    n = num_elems
    coords = np.zeros((n + 1, 3))
    coords[:, 0] = np.arange(n + 1) / n
    conn = np.stack([np.arange(n), np.arange(1, n + 1)], axis=1)
    return Mesh(kind, coords, conn, grid=(n,))


def unit_square_tri(nx, ny=None):
    """Unit square, nx x ny cells, each split by the (0,0)-(1,1) diagonal into
    the counter-clockwise triangles (n0,n1,n2) and (n0,n2,n3); nodes numbered
    x fastest."""
    ny = nx if ny is None else ny
    ix, iy = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="xy")
    coords = np.zeros(((nx + 1) * (ny + 1), 3))
    coords[:, 0] = (ix / nx).ravel()
    coords[:, 1] = (iy / ny).ravel()
    cx, cy = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    n0 = (cx + (nx + 1) * cy).ravel()
    n1 = n0 + 1
    n2 = n0 + (nx + 1) + 1
    n3 = n0 + (nx + 1)
    conn = np.empty((2 * nx * ny, 3), dtype=np.int64)
    conn[0::2] = np.stack([n0, n1, n2], axis=1)
    conn[1::2] = np.stack([n0, n2, n3], axis=1)
    return Mesh(TRI3_POISSON, coords, conn, grid=(nx, ny))


def unit_cube_hex(n, kind=HEX8_POISSON):
    """Unit cube, n^3 trilinear hexahedra in Shapefun<HEXAHEDRON,8> node order
    (corlib/Shapefun.ipp:898-937); nodes numbered x fastest, then y, then z."""
    m = n + 1
    iz, iy, ix = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    coords = np.stack([ix.ravel() / n, iy.ravel() / n, iz.ravel() / n], axis=1)
    cz, cy, cx = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    b = (cx + m * (cy + m * cz)).ravel()
    off = [0, 1, 1 + m, m, m * m, m * m + 1, m * m + 1 + m, m * m + m]
    conn = np.stack([b + o for o in off], axis=1)
    return Mesh(kind, coords, conn, grid=(n, n, n))


def fuzzy_equal(a, b, tol=1e-8):
    """corlib/fuzzyEqual.hpp:28-30"""
    return np.abs(a - b) < tol


def dirichlet_dofs(mesh, faces="all", components=None):
    """Constrained dofs in ConstraintFunctor order (node order, then component).

    faces: "all" -> every node with some coordinate (of the first dim) equal to
    0 or 1 (fuzzyEqual); "x" -> x == 0 or x == 1 (laplaceRHSinfer fem.hpp:35-40);
    "x0" -> x == 0 only (the clamped face of the elasticity config)."""
    X = mesh.coords[:, : mesh.dim]
    if faces == "all":
        sel = np.any(fuzzy_equal(X, 0.0) | fuzzy_equal(X, 1.0), axis=1)
    elif faces == "x":
        sel = fuzzy_equal(X[:, 0], 0.0) | fuzzy_equal(X[:, 0], 1.0)
    elif faces == "x0":
        sel = fuzzy_equal(X[:, 0], 0.0)
    else:
        raise ValueError(faces)
    nodes = np.nonzero(sel)[0]
    d = mesh.dof
    comps = range(d) if components is None else components
    dofs = (nodes[:, None] * d + np.array(list(comps))[None, :]).ravel()
    return dofs.astype(np.uint32)


def interior_points(rng, n, dim, margin=0.0):
    return margin + (1.0 - 2 * margin) * rng.random((n, dim))


def projection_matrix(mesh, points, components=None):
    """Sensor projection P (ns x num_dofs) as CSR arrays (indptr, indices, data):
    row a holds the element shape-function values at sensor point a, on the
    dof of component components[a] (0 for scalar problems)."""
    kind, grid = mesh.kind, mesh.grid
    ns = points.shape[0]
    nn = NODES_PER_ELEM[kind]
    d = mesh.dof
    comps = np.zeros(ns, dtype=np.int64) if components is None else np.asarray(components)
    indptr = np.arange(ns + 1, dtype=np.int64) * nn
    indices = np.empty(ns * nn, dtype=np.int32)
    data = np.empty(ns * nn)
    for a in range(ns):
        p = points[a]
        if kind == LINE2_POISSON:
            n = grid[0]
            c = min(int(p[0] * n), n - 1)
            e = c
            xi = p[0] * n - c
            phi = [1 - xi, xi]
        elif kind == TRI3_POISSON:
            nx, ny = grid
            cx = min(int(p[0] * nx), nx - 1)
            cy = min(int(p[1] * ny), ny - 1)
            u, v = p[0] * nx - cx, p[1] * ny - cy
            cell = cx + nx * cy
            e = 2 * cell if v <= u else 2 * cell + 1
            X = mesh.coords[mesh.conn[e], :2]
            G = np.stack([X[1] - X[0], X[2] - X[0]], axis=1)
            xi = np.linalg.solve(G, p[:2] - X[0])
            phi = [1 - xi[0] - xi[1], xi[0], xi[1]]
        else:
            n = grid[0]
            c = [min(int(p[k] * n), n - 1) for k in range(3)]
            e = c[0] + n * (c[1] + n * c[2])
            x, y, z = (p[k] * n - c[k] for k in range(3))
            phi = [(1 - x) * (1 - y) * (1 - z), x * (1 - y) * (1 - z), x * y * (1 - z),
                   (1 - x) * y * (1 - z), (1 - x) * (1 - y) * z, x * (1 - y) * z,
                   x * y * z, (1 - x) * y * z]
        nodes = mesh.conn[e].astype(np.int64)
        indices[a * nn:(a + 1) * nn] = nodes * d + comps[a]
        data[a * nn:(a + 1) * nn] = phi
    return indptr, indices, data


def projection_dense(mesh, indptr, indices, data):
    ns = len(indptr) - 1
    P = np.zeros((ns, mesh.num_dofs))
    for a in range(ns):
        for s in range(indptr[a], indptr[a + 1]):
            P[a, indices[s]] += data[s]
    return P


def _se_sqrt_1d(x, length, jitter=1e-12):
    """Symmetric square root of the 1-D squared-exponential correlation matrix."""
    D = x[:, None] - x[None, :]
    K = np.exp(-D * D / (2.0 * length * length))
    lam, V = np.linalg.eigh(K + jitter * np.eye(len(x)))
    lam = np.clip(lam, 0.0, None)
    return (V * np.sqrt(lam)) @ V.T


def se_field_tensor(rng, axes, sigma, length):
    """Sample g ~ GP(0, sigma^2 exp(-|x-y|^2/(2 l^2))) on the tensor grid
    spanned by the 1-D coordinate arrays ``axes`` (first axis fastest in the
    flattened result).  Exact for the squared-exponential kernel because it
    factorises over coordinates: K = K_z (x) K_y (x) K_x."""
    roots = [_se_sqrt_1d(np.asarray(a, dtype=np.float64), length) for a in axes]
    shape = tuple(len(a) for a in axes[::-1])  # (z, y, x) for C order
    z = rng.standard_normal(shape)
    for k, S in enumerate(roots[::-1]):
        z = np.moveaxis(np.tensordot(S, z, axes=([1], [k])), 0, k)
    return sigma * z.ravel()


def cell_centre_axes(n):
    return (np.arange(n) + 0.5) / n


def matern32_field_cells(rng, n, sigma, length, dim=3, pad=2):
    """Sample a Matérn nu = 3/2 field, c(r) = sigma^2 (1 + sqrt(3) r / l)
    exp(-sqrt(3) r / l), at the n^dim cell centres of the unit square/cube
    (x fastest, the element order of unit_cube_hex / unit_square_tri cells)
    by circulant embedding on a periodic grid of pad*n cells per side
    (Dietrich & Newsam 1997).  Negative eigenvalues of the embedding, which
    appear only when pad*n*h is short against the correlation length, are
    clipped to zero."""
    m = pad * n
    h = 1.0 / n
    d = np.minimum(np.arange(m), m - np.arange(m)) * h  # periodic distance per axis
    grids = np.meshgrid(*([d] * dim), indexing="ij")
    r = np.sqrt(sum(g * g for g in grids))
    a = np.sqrt(3.0) * r / length
    c = sigma * sigma * (1.0 + a) * np.exp(-a)
    lam = np.clip(np.fft.fftn(c).real, 0.0, None)
    w = rng.standard_normal(c.shape) + 1j * rng.standard_normal(c.shape)
    f = np.fft.fftn(np.sqrt(lam / c.size) * w).real
    f = f[tuple(slice(0, n) for _ in range(dim))]
    # C order is (axis0, axis1, axis2); make x (the last index) fastest
    return np.ascontiguousarray(f).ravel()


def disjoint_union(meshes):
    """One mesh holding the given meshes as disjoint blocks (node ids and dofs
    offset block by block).  Returns (mesh, dof_offset)."""
    kind = meshes[0].kind
    coords, conn, off = [], [], [0]
    base = 0
    for m in meshes:
        if m.kind != kind:
            raise ValueError("all meshes must have the same element kind")
        coords.append(m.coords)
        conn.append(m.conn + base)
        base += m.num_nodes
        off.append(off[-1] + m.num_dofs)
    return Mesh(kind, np.concatenate(coords), np.concatenate(conn).astype(np.uint32)), np.array(off, dtype=np.int64)
