"""CPU oracle for the statFEM forward-and-conditioning path.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` as the checker.  The product never
imports it.

Finite-element arithmetic (quadrature, element matrices, loads, triplet
assembly, row-zeroing constraints, squared-exponential kernel, dense nodal
forcing covariance) comes from the C restatement in ``sfo.c``; the sparse
direct solves use SuperLU (``scipy.sparse.linalg.splu``), the same LU family
as the reference's ``Eigen::SparseLU`` (corlib/SystemSolveEigenSparse.hpp:
153,299-300,394-397), applied to the same non-symmetric row-zeroed matrix and
its transpose; the small dense statistics are restated in numpy following
statX/infer/{ForwardGaussRHS.hpp,MismatchCovariance.hpp,LikelihoodKOH.ipp}.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libsfo.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def build():
    """Compile sfo.c into _build/libsfo.so (make, no reference sources)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(_HERE, "sfo.c")
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.sfo_quadrature.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.sfo_element_matrix.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_double,
                                         ctypes.c_double, _dp]
        L.sfo_assemble_load.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int64, _u32p,
                                        ctypes.c_int64, _dp, _dp]
        L.sfo_assemble_csr.restype = ctypes.c_int64
        L.sfo_assemble_csr.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int64, _u32p,
                                       ctypes.c_int64, _dp, ctypes.c_double, _i64p, _i32p, _dp]
        L.sfo_apply_constraints.argtypes = [ctypes.c_int64, _i64p, _i32p, _dp, _dp, _u32p, _dp,
                                            ctypes.c_int64, ctypes.c_double, ctypes.c_double]
        L.sfo_se_kernel.restype = ctypes.c_double
        L.sfo_se_kernel.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_double]
        L.sfo_forcing_covariance_dense.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int64, _dp,
                                                   _dp, ctypes.c_double, ctypes.c_double, _dp]
        L.sfo_pcg.argtypes = [ctypes.c_int64, _i64p, _i32p, _dp, _u8p, _dp, _dp, ctypes.c_double,
                              ctypes.c_int, _dp]
        L.sfo_block_pcg.argtypes = [ctypes.c_int64, _i64p, _i32p, _dp, _u8p, ctypes.c_int, _dp, _dp,
                                    ctypes.c_double, ctypes.c_int, ctypes.c_int, _i32p]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


# --------------------------------------------------------------------------
# finite-element part (C restatement)
# --------------------------------------------------------------------------

def quadrature(kind, qps):
    w = np.zeros(125)
    pts = np.zeros(375)
    n = lib().sfo_quadrature(kind, qps, _p(w, _dp), _p(pts, _dp))
    if n <= 0:
        raise ValueError("unsupported quadrature")
    return w[:n].copy(), pts[: 3 * n].reshape(n, 3).copy()


def element_matrix(kind, qps, X, coeff=1.0, nu=0.3):
    X = np.ascontiguousarray(X, dtype=np.float64)
    L = {1: 2, 2: 3, 3: 8, 4: 24}[kind]
    Ke = np.zeros((L, L))
    rc = lib().sfo_element_matrix(kind, qps, _p(X, _dp), coeff, nu, _p(Ke, _dp))
    if rc < 0:
        raise ValueError("element matrix failed (%d)" % rc)
    return Ke


def assemble_csr(mesh, qps, coeff=None, nu=0.3):
    """Row-major sorted-unique triplets (explicit zeros kept) as scipy CSR."""
    L = lib()
    c = None if coeff is None else np.ascontiguousarray(coeff, dtype=np.float64)
    cp = _p(c, _dp) if c is not None else None
    args = (mesh.kind, qps, _p(mesh.coords, _dp), mesh.num_nodes, _p(mesh.conn, _u32p),
            mesh.num_elems, cp, nu)
    nnz = L.sfo_assemble_csr(*args, None, None, None)
    if nnz < 0:
        raise ValueError("assembly failed (%d)" % nnz)
    N = mesh.num_dofs
    rp = np.zeros(N + 1, dtype=np.int64)
    col = np.zeros(nnz, dtype=np.int32)
    val = np.zeros(nnz)
    L.sfo_assemble_csr(*args, _p(rp, _i64p), _p(col, _i32p), _p(val, _dp))
    return rp, col, val


def assemble_load(mesh, qps, f):
    f = np.ascontiguousarray(np.atleast_1d(f), dtype=np.float64)
    F = np.zeros(mesh.num_dofs)
    rc = lib().sfo_assemble_load(mesh.kind, qps, _p(mesh.coords, _dp), mesh.num_nodes,
                                 _p(mesh.conn, _u32p), mesh.num_elems, _p(f, _dp), _p(F, _dp))
    if rc < 0:
        raise ValueError("load failed")
    return F


def apply_constraints(rp, col, val, F, idx, value=None, factor=1.0, scalar=1.0):
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    value = np.zeros(len(idx)) if value is None else np.ascontiguousarray(value, dtype=np.float64)
    rc = lib().sfo_apply_constraints(len(rp) - 1, _p(rp, _i64p), _p(col, _i32p), _p(val, _dp),
                                     _p(F, _dp) if F is not None else None, _p(idx, _u32p),
                                     _p(value, _dp), len(idx), factor, scalar)
    if rc < 0:
        raise ValueError("constraint failed (%d)" % rc)


def se_kernel(dim, x, y, sigma, length):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    return lib().sfo_se_kernel(dim, _p(x, _dp), _p(y, _dp), sigma, length)


def forcing_covariance_dense(dim, dof, coords, phibar, sigma, length):
    """coords: num_nodes x 3 (SMF layout); the first dim columns are used."""
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    if coords.ndim != 2 or coords.shape[1] != 3:
        raise ValueError("coords must be num_nodes x 3")
    phibar = np.ascontiguousarray(phibar, dtype=np.float64)
    n = coords.shape[0]
    Cf = np.zeros((n * dof, n * dof))
    lib().sfo_forcing_covariance_dense(dim, dof, n, _p(coords, _dp), _p(phibar, _dp), sigma,
                                       length, _p(Cf, _dp))
    return Cf


def pcg(rp, col, val, mask, b, tol=1e-8, max_iter=100000):
    N = len(rp) - 1
    x = np.zeros(N)
    work = np.zeros(4 * N)
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    b = np.ascontiguousarray(b, dtype=np.float64)
    it = lib().sfo_pcg(N, _p(rp, _i64p), _p(col, _i32p), _p(val, _dp), _p(m, _u8p), _p(b, _dp),
                       _p(x, _dp), tol, max_iter, _p(work, _dp))
    return x, it


def block_pcg(rp, col, val, mask, B, tol, max_iter=100000, X0=None):
    """FP64 Jacobi-PCG on the symmetric elimination of the row-zeroed matrix
    for every row of B (k x N) at once, OpenMP over matrix rows (sfo.c
    sfo_block_pcg).  Starts from X0 (k x N) when given.  Returns (X, its)."""
    N = len(rp) - 1
    B = np.atleast_2d(np.asarray(B, dtype=np.float64))
    k = B.shape[0]
    Bi = np.ascontiguousarray(B.T)
    Xi = np.zeros((N, k)) if X0 is None else np.ascontiguousarray(np.atleast_2d(X0).T)
    its = np.zeros(k, dtype=np.int32)
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    rc = lib().sfo_block_pcg(N, _p(rp, _i64p), _p(col, _i32p), _p(val, _dp), _p(m, _u8p), k, _p(Bi, _dp),
                             _p(Xi, _dp), tol, max_iter, int(X0 is not None), _p(its, _i32p))
    if rc == -2:
        raise MemoryError("sfo_block_pcg: allocation failed")
    return np.ascontiguousarray(Xi.T), its


# --------------------------------------------------------------------------
# solver: SuperLU on the reference's row-zeroed system
# --------------------------------------------------------------------------

class DirectSolver:
    """SystemSolveEigenSparse restated with SuperLU: solveSystem factorises A,
    solveSystemTranspose factorises A^T (SystemSolveEigenSparse.hpp:273-404)."""

    def __init__(self, rp, col, val):
        N = len(rp) - 1
        self.A = sp.csr_matrix((val, col, rp), shape=(N, N))
        self._lu = None
        self._luT = None

    def solve(self, F):
        if self._lu is None:
            self._lu = spla.splu(self.A.tocsc())
        return self._lu.solve(np.asarray(F, dtype=np.float64))

    def solve_transpose(self, rhs):
        if self._luT is None:
            self._luT = spla.splu(self.A.T.tocsc())
        return self._luT.solve(np.asarray(rhs, dtype=np.float64))


# --------------------------------------------------------------------------
# statistics (numpy restatement of statX/infer)
# --------------------------------------------------------------------------

def se_matrix(X, Y, sigma, length):
    """ExpKernel values for all pairs (statX/infer/ExpKernel.hpp:74-92)."""
    D = X[:, None, :] - Y[None, :, :]
    return sigma * sigma * np.exp(-np.sum(D * D, axis=2) / (2.0 * length * length))


def forward_gauss_rhs(solver, F, P, coords, phibar, dim, dof, sigma_f, length_f, reg):
    """ForwardGaussRHS::updateSolution (statX/infer/ForwardGaussRHS.hpp:95-139):
    R rows solve A^T r_i = P_i; mean = R F; C_s = R C_f R^T + (sigma_f*reg)^2 P P^T
    with C_f from CovarianceForcing::giveProjectedCovar (CovarianceForcing.ipp:38-109)."""
    R = np.stack([solver.solve_transpose(P[i]) for i in range(P.shape[0])])
    mean = R @ F
    Cf = forcing_covariance_dense(dim, dof, coords, phibar, sigma_f, length_f)
    C = R @ Cf @ R.T
    add = sigma_f * reg
    C = C + add * add * (P @ P.T)
    return mean, C, R


def forward_perturbation(mesh, qps, F, rp, col, val, bc_dofs, P, phibar, sigma_f, length_f, sigma_m, length_m,
                         reg):
    """ForwardPerturbation::updateSolution (statX/infer/ForwardPerturbation.hpp:
    109-195), dense: R = P A^-1, u = A^-1 F, M = A^-1 C_f A^-T + u u^T, the
    material covariance C_m over element centroids (CovarianceMaterial.hpp,
    SE kernel under "material."), dA/dkappa_e = the unit-conductivity element
    matrix (ElementPotential.ipp:225-237) scattered with the constrained rows
    zeroed; C = R C_f R^T + sum_e sum_d C_m[e,d] R dA_e M dA_d^T R^T
    + (reg sigma_m)^2 P P^T, mean = P u.  The whole A^-1 is used (the
    reference fills the rows of its A^-1 only up to the number of sensors)."""
    N = mesh.num_dofs
    A = sp.csr_matrix((val, col, rp), shape=(N, N)).toarray()
    Ainv = np.linalg.inv(A)
    u = Ainv @ F
    R = P @ Ainv
    Cf = forcing_covariance_dense(mesh.dim, mesh.dof, mesh.coords, phibar, sigma_f, length_f)
    M = Ainv @ Cf @ Ainv.T + np.outer(u, u)
    cent = mesh.coords[mesh.conn].mean(axis=1)[:, :mesh.dim]
    Cm = se_matrix(cent, cent, sigma_m, length_m)
    free = np.ones(N)
    free[np.asarray(bc_dofs, dtype=np.int64)] = 0.0
    E = mesh.num_elems
    Q = []
    for e in range(E):
        X = mesh.coords[mesh.conn[e]]
        ke = element_matrix(mesh.kind, qps, X, coeff=1.0)
        dofs = mesh.conn[e].astype(np.int64)
        D = np.zeros((N, N))
        D[np.ix_(dofs, dofs)] = ke
        D *= free[:, None]
        Q.append(R @ D)
    Q = np.stack(Q)                      # E x ns x N
    QM = np.einsum("eai,ij->eaj", Q, M)  # R dA_e M
    QS = np.einsum("ed,dbj->ebj", Cm, Q)  # sum_d C_m[e,d] R dA_d
    Cmat = np.einsum("eaj,ebj->ab", QM, QS)
    add = reg * sigma_m
    C = R @ Cf @ R.T + Cmat + add * add * (P @ P.T)
    return P @ u, C


def grid_axes(mesh):
    """The 1-D node coordinates of a structured mesh (x fastest, then y, z),
    checked against every node coordinate."""
    d = mesh.dim
    axes = [np.unique(mesh.coords[:, a]) for a in range(d)]
    grid = np.stack(np.meshgrid(*axes[::-1], indexing="ij")[::-1], axis=-1).reshape(-1, d)
    if grid.shape[0] != mesh.num_nodes or np.abs(grid - mesh.coords[:, :d]).max() > 0:
        raise ValueError("not a tensor-product node grid")
    return axes


def forcing_covariance_apply_grid(mesh, phibar, sigma, length, W):
    """C_f W for the nodal forcing covariance of CovarianceForcing::
    giveProjectedCovar (statX/infer/CovarianceForcing.ipp:38-109) on a
    tensor-product node grid, without forming the N x N matrix: per
    component, C_f = diag(phibar) sigma^2 (K_z (x) K_y (x) K_x) diag(phibar),
    because the squared-exponential kernel factorises over coordinates
    (exp(-|d|^2/2l^2) = prod_a exp(-d_a^2/2l^2); the same matrix as the
    dense restatement up to the rounding of that product).  W: N x m."""
    axes = grid_axes(mesh)
    dof = mesh.dof
    W = np.asarray(W, dtype=np.float64)
    out = np.zeros_like(W)
    Ks = [np.exp(-(x[:, None] - x[None, :]) ** 2 / (2.0 * length * length)) for x in axes]
    shape = tuple(len(x) for x in axes[::-1]) + (W.shape[1],)  # (z, y, x, m)
    for c in range(dof):
        pb = phibar[c::dof]
        T = (pb[:, None] * W[c::dof]).reshape(shape)
        for a, K in enumerate(Ks):
            ax = len(axes) - 1 - a  # x is the last grid axis
            T = np.moveaxis(np.tensordot(K, T, axes=([1], [ax])), 0, ax)
        out[c::dof] = sigma * sigma * pb[:, None] * T.reshape(-1, W.shape[1])
    return out


def forward_gauss_rhs_grid(R, F, Pd, mesh, phibar, sigma_f, length_f, reg):
    """ForwardGaussRHS::updateSolution (statX/infer/ForwardGaussRHS.hpp:95-139)
    from given adjoint rows R: mean = R F, C_s = R C_f R^T + (sigma_f reg)^2 P P^T,
    with C_f applied through its Kronecker factors (tensor-product grids)."""
    mean = R @ F
    C = R @ forcing_covariance_apply_grid(mesh, phibar, sigma_f, length_f, R.T)
    C = 0.5 * (C + C.T)
    add = sigma_f * reg
    return mean, C + add * add * (Pd @ Pd.T)


def statfem_prior_iterative(mesh, qps, f, bc_dofs, Pd, sigma_f, length_f, reg, coeff=None, nu=0.3, tol=1e-13,
                            X0=None):
    """Prior at the sensors for meshes too large for the direct solve: the
    forward solve A u = F and the ns adjoint solves A^T r_i = P_i by FP64
    Jacobi-PCG (block_pcg) to the relative residual tol on the symmetric
    elimination of the row-zeroed system.  With homogeneous Dirichlet data the
    adjoint rows differ from the reference's A^T solve only on constrained
    dofs, where F and phibar vanish, so mean and C_s are those of
    ForwardGaussRHS (SystemSolveEigenSparse.hpp:364-404 with
    ForwardGaussRHS.hpp:95-139).  Returns the dict of statfem_prior plus the
    solution block X (rows: u, r_1..r_ns) and the iteration counts."""
    rp, col, val, F = fem(mesh, qps, f, bc_dofs, coeff=coeff, nu=nu)
    mask = np.zeros(mesh.num_dofs, dtype=np.uint8)
    mask[np.asarray(bc_dofs, dtype=np.int64)] = 1
    B = np.vstack([F[None, :], Pd])
    X, its = block_pcg(rp, col, val, mask, B, tol, X0=X0)
    phibar = unit_load(mesh, qps, bc_dofs)
    R = X[1:]
    mean_s, C_s = forward_gauss_rhs_grid(R, F, Pd, mesh, phibar, sigma_f, length_f, reg)
    return dict(rp=rp, col=col, val=val, F=F, u=X[0], phibar=phibar, mean_s=mean_s, C_s=C_s, R=R, X=X,
                its=its)


def mismatch_covariance(sensor_coords, sigma_d, length_d, eps):
    """MismatchCovariance::giveCovariance (statX/infer/MismatchCovariance.hpp:76-99)."""
    K = se_matrix(sensor_coords, sensor_coords, sigma_d, length_d)
    return K + eps * eps * np.eye(len(sensor_coords))


def koh_log_likelihood(mean_s, C_s, Ks, Y, rho):
    """LikelihoodKOH::giveLogLikelihood (statX/infer/LikelihoodKOH.ipp:75-120):
    C = K_s + rho^2 C_s; n_o * (-ns/2 log 2pi - sum log L_ii) - 1/2 sum_k d_k^T C^-1 d_k."""
    ns, n_o = Y.shape
    C = Ks + rho * rho * C_s
    L = np.linalg.cholesky(C)
    t1 = -0.5 * ns * math.log(2.0 * math.pi)
    t2 = -0.5 * (2.0 * np.sum(np.log(np.diag(L))))
    t3 = 0.0
    for k in range(n_o):
        d = Y[:, k] - rho * mean_s
        z = np.linalg.solve(L, d)
        q = -0.5 * float(z @ z)
        if not q < 0.0:
            raise ValueError("non-negative quadratic term")
        t3 += q
    return n_o * (t1 + t2) + t3


def koh_proj_conditioned(mean_s, C_s, Ks, Y, rho):
    """LikelihoodKOH::giveProjFEconditionedData (LikelihoodKOH.ipp:311-361):
    Sigma = (rho^2 n_o K_s^-1 + C_s^-1)^-1; m = Sigma (rho K_s^-1 sum_k y_k + C_s^-1 mean)."""
    n_o = Y.shape[1]
    Ksi = np.linalg.inv(Ks)
    Cui = np.linalg.inv(C_s)
    S = np.linalg.inv(rho * rho * n_o * Ksi + Cui)
    ysum = Y.sum(axis=1)
    m = S @ (rho * Ksi @ ysum + Cui @ mean_s)
    return m, S


def koh_woodbury(C_s, Ks, Y, rho, P, C_u, u_mean):
    """LikelihoodKOH::giveFEconditionedDataWoodbury (LikelihoodKOH.ipp:442-508):
    S = K_s/(rho^2 n_o) + C_s; D = I - C_u P^T S^-1 P; Sigma = D C_u;
    m = D (rho C_u P^T K_s^-1 sum_k y_k + u_mean).  C_u, u_mean are the
    unprojected (P = I) prior covariance and mean."""
    n_o = Y.shape[1]
    Ksi = np.linalg.inv(Ks)
    Si = np.linalg.inv(Ks / (rho * rho * n_o) + C_s)
    N = C_u.shape[0]
    D = np.eye(N) - C_u @ P.T @ Si @ P
    cov = D @ C_u
    ysum = Y.sum(axis=1)
    vecA = rho * (C_u @ P.T @ Ksi @ ysum)
    mean = D @ (vecA + u_mean)
    return mean, cov


def gp_regression(x_train, y_train, x_pred, sigma, length, eps):
    """statX/infer/GaussianProcess.hpp fit/predictMean/predictVariance/
    giveLogLikelihood (LLT of k(x,x) + eps^2 I)."""
    K = se_matrix(x_train, x_train, sigma, length) + eps * eps * np.eye(len(x_train))
    L = np.linalg.cholesky(K)
    alpha = np.linalg.solve(L.T, np.linalg.solve(L, y_train))
    ks = se_matrix(x_train, x_pred, sigma, length)
    mean = ks.T @ alpha
    v = np.linalg.solve(L, ks)
    var = sigma * sigma - np.sum(v * v, axis=0)
    ll = -0.5 * float(y_train @ alpha) - float(np.sum(np.log(np.diag(L)))) \
        - 0.5 * len(x_train) * math.log(2.0 * math.pi)
    return mean, var, ll


# --------------------------------------------------------------------------
# full problems
# --------------------------------------------------------------------------

def fem(mesh, qps, f, bc_dofs, coeff=None, nu=0.3, bc_values=None):
    """laplaceRHSinfer fem() (del2/apps/reference/laplaceRHSinfer/fem.hpp:49-97):
    assemble K, F, apply row-zeroing constraints; returns (rp, col, val, F)."""
    rp, col, val = assemble_csr(mesh, qps, coeff=coeff, nu=nu)
    F = assemble_load(mesh, qps, f)
    apply_constraints(rp, col, val, F, bc_dofs, bc_values)
    return rp, col, val, F


def unit_load(mesh, qps, bc_dofs):
    """CovarianceForcing::covVec_: phibar = assembled unit load, zero at the
    constrained dofs (inference.hpp:108-124; CovarianceForcing.hpp:101-114)."""
    phibar = assemble_load(mesh, qps, np.ones(mesh.dof))
    phibar[np.asarray(bc_dofs, dtype=np.int64)] = 0.0
    return phibar


def statfem_prior(mesh, qps, f, bc_dofs, P, sigma_f, length_f, reg, coeff=None, nu=0.3):
    rp, col, val, F = fem(mesh, qps, f, bc_dofs, coeff=coeff, nu=nu)
    solver = DirectSolver(rp, col, val)
    u = solver.solve(F)
    phibar = unit_load(mesh, qps, bc_dofs)
    mean_s, C_s, R = forward_gauss_rhs(solver, F, P, mesh.coords, phibar,
                                       mesh.dim, mesh.dof, sigma_f, length_f, reg)
    return dict(rp=rp, col=col, val=val, F=F, u=u, phibar=phibar, mean_s=mean_s, C_s=C_s,
                R=R, solver=solver)
