"""Dense CPU restatement of the two-level preconditioner of the GPU solver
(statfem_b200/csrc/coarse.cu, dense.cu), for tests.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the
algorithm; the product never imports it.

The reference solves its systems with a direct factorisation
(corlib/SystemSolveEigenSparse.hpp:273-404), so this preconditioner has no
reference counterpart; what the tests pin is that it is a fixed SPD operator
and that PCG with it reaches the direct solution.  Restated here:
* box aggregation: a grid of about `size` nodes per axis over the bounding
  box, nodes assigned by floor of their scaled coordinate;
* the six rigid-body modes of each aggregate (translations, rotations
  e_k x d about the centroid, d in units of the box edge), zero on
  constrained dofs; on scalar meshes the aggregate's constant;
* the Galerkin matrix A_c = P^T S P;
* block Gauss-Jordan elimination without pivoting in 32-wide panels with a
  pivot dropped (row and column zeroed) when it is not above rel x its
  original diagonal;
* M^-1 r = D^-1 r + P A_c^+ P^T r with D the nodal 3 x 3 diagonal blocks
  (the diagonal on scalar meshes).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def box_aggregates(coords, size, max_aggs=512):
    """Aggregate id per node and the box edge (the GPU library additionally
    coarsens the grid until every element spans boxes at most one apart)."""
    X = np.asarray(coords, dtype=np.float64)
    lo, hi = X.min(axis=0), X.max(axis=0)
    ext = hi - lo
    emax = ext.max()
    act = ext > 1e-12 * emax
    dim = int(act.sum())
    vol = float(np.prod(ext[act]))
    target = min(max_aggs, max(1.0, len(X) / float(max(size, 2)) ** dim))
    hb = (vol / target) ** (1.0 / dim)
    nb = np.where(act, np.maximum(1, np.rint(ext / np.where(act, hb, 1.0))), 1).astype(int)
    b = np.zeros_like(X, dtype=int)
    for d in range(3):
        if act[d]:
            b[:, d] = np.clip(np.floor((X[:, d] - lo[d]) / ext[d] * nb[d]).astype(int), 0, nb[d] - 1)
    box = b[:, 0] + nb[0] * (b[:, 1] + nb[1] * b[:, 2])
    ids, agg = np.unique(box, return_inverse=True)
    h = float(np.mean(ext[act] / nb[act]))
    return agg, h


def rigid_modes(coords, agg, h, mask):
    """P (num_dofs x 6 n_agg, sparse): column 6a + k is mode k of aggregate a."""
    X = np.asarray(coords, dtype=np.float64)
    nodes = len(X)
    nagg = int(agg.max()) + 1
    cnt = np.bincount(agg, minlength=nagg)
    cen = np.stack([np.bincount(agg, X[:, d], minlength=nagg) / cnt for d in range(3)], axis=1)
    dx = (X - cen[agg]) / h
    z, o = np.zeros(nodes), np.ones(nodes)
    # modes[node, component, k]; rotation k displaces by e_k x d
    modes = np.stack([np.stack([o, z, z, z, dx[:, 2], -dx[:, 1]], 1),
                      np.stack([z, o, z, -dx[:, 2], z, dx[:, 0]], 1),
                      np.stack([z, z, o, dx[:, 1], -dx[:, 0], z], 1)], 1)
    ii, cc, kk = np.nonzero(modes)
    keep = ~np.asarray(mask, dtype=bool)[3 * ii + cc]
    ii, cc, kk = ii[keep], cc[keep], kk[keep]
    return sp.csr_matrix((modes[ii, cc, kk], (3 * ii + cc, 6 * agg[ii] + kk)), shape=(3 * nodes, 6 * nagg))


def gauss_jordan_inverse(A, rel, panel=32):
    """In-place block Gauss-Jordan inverse as the GPU computes it; returns
    (inverse, Schur pivots, number of dropped pivots)."""
    A = np.array(A, dtype=np.float64)
    n = A.shape[0]
    adiag = np.diag(A).copy()
    piv_out = np.zeros(n)
    dropped = 0
    for k0 in range(0, n, panel):
        kb = min(panel, n - k0)
        D = A[k0:k0 + kb, k0:k0 + kb].copy()
        for p in range(kb):
            piv = D[p, p]
            piv_out[k0 + p] = piv
            if not piv > rel * adiag[k0 + p]:
                D[p, :] = 0.0
                D[:, p] = 0.0
                dropped += 1
                continue
            row, colv = D[p].copy(), D[:, p].copy()
            D = D - np.outer(colv, row) / piv
            D[p, :] = row / piv
            D[:, p] = -colv / piv
            D[p, p] = 1.0 / piv
        colp = A[:, k0:k0 + kb].copy()
        rowp = D @ A[k0:k0 + kb, :]
        rowp[:, k0:k0 + kb] = D
        upd = colp @ rowp
        newA = A - upd
        newA[:, k0:k0 + kb] = -upd[:, k0:k0 + kb]
        newA[k0:k0 + kb, :] = rowp
        A = newA
    return A, piv_out, dropped


def nodal_block_jacobi(S):
    """Inverse 3 x 3 diagonal blocks of S (nodes x 3 x 3)."""
    S = sp.csr_matrix(S).tocoo()
    nodes = S.shape[0] // 3
    D = np.zeros((nodes, 3, 3))
    sel = (S.row // 3) == (S.col // 3)
    np.add.at(D, (S.row[sel] // 3, S.row[sel] % 3, S.col[sel] % 3), S.data[sel])
    return np.linalg.inv(D)


def constant_modes(agg, mask):
    """P (num_nodes x n_agg) for scalar meshes: the indicator of each
    aggregate, zero on constrained dofs."""
    nodes = len(agg)
    free = ~np.asarray(mask, dtype=bool)
    i = np.nonzero(free)[0]
    return sp.csr_matrix((np.ones(len(i)), (i, agg[i])), shape=(nodes, int(agg.max()) + 1))


class TwoLevel:
    """M^-1 = D^-1 + P A_c^+ P^T for the symmetric eliminated operator S:
    nodal 3 x 3 block Jacobi and rigid-body modes (dof = 3), point Jacobi and
    aggregate constants (dof = 1)."""

    def __init__(self, S, coords, mask, size=8, rel=1e-10, dof=3):
        self.S = sp.csr_matrix(S)
        self.dof = dof
        agg, h = box_aggregates(coords, size, max_aggs=512 if dof == 3 else 2048)
        self.P = rigid_modes(coords, agg, h, mask) if dof == 3 else constant_modes(agg, mask)
        Ac = (self.P.T @ self.S @ self.P).toarray()
        self.Ac = Ac
        self.Ainv, self.pivots, self.dropped = gauss_jordan_inverse(Ac, rel)
        if dof == 3:
            self.Dinv = nodal_block_jacobi(self.S)
        else:
            self.dinv = 1.0 / self.S.diagonal()

    @property
    def coarse_dofs(self):
        return self.Ac.shape[0] - self.dropped

    def __call__(self, r):
        if self.dof == 3:
            z = np.einsum('nij,nj->ni', self.Dinv, r.reshape(-1, 3)).ravel()
        else:
            z = self.dinv * r
        return z + self.P @ (self.Ainv @ (self.P.T @ r))


def pcg(S, b, M, tol=1e-10, max_iter=20000):
    """Preconditioned CG on S x = b; returns (x, iterations)."""
    x = np.zeros_like(b)
    r = b.copy()
    z = M(r)
    p = z.copy()
    rz = r @ z
    bb = b @ b
    if bb == 0.0:
        return x, 0
    for it in range(max_iter):
        q = S @ p
        a = rz / (p @ q)
        x += a * p
        r -= a * q
        if r @ r <= tol * tol * bb:
            return x, it + 1
        z = M(r)
        rzn = r @ z
        p = z + (rzn / rz) * p
        rz = rzn
    return x, max_iter
