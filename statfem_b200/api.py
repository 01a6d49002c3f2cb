"""Python mirror of the reference interface for the statFEM hot path, bound to
the C ABI (include/statfem_cuda.h) of libstatfem_cuda.so through ctypes.

Class and method names follow the reference:
  SystemSolveCuda      <- corlib::SystemSolveEigenSparse (corlib/SystemSolveEigenSparse.hpp)
  CovarianceForcing    <- statX::infer::CovarianceForcing (statX/infer/CovarianceForcing.hpp)
  ForwardGaussRHS      <- statX::infer::ForwardGaussRHS (statX/infer/ForwardGaussRHS.hpp)
  LikelihoodKOH        <- statX::infer::LikelihoodKOH + MismatchCovariance
                          (statX/infer/LikelihoodKOH.hpp, MismatchCovariance.hpp)
Hyperparameters are passed as the reference's name -> value maps
("forcing.sigma", "forcing.length", "rho", "mismatch.sigma", "mismatch.length",
"mismatch.sensorEps").  Where the reference aborts (FTL_VERIFY), these raise
SfcError.  There is no CPU fallback: every call goes to the CUDA library, and
importing this module fails if the library has not been built.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import meshgen

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libstatfem_cuda.so")

SFC_SOLVER_PCG_FP64 = 0
SFC_SOLVER_PCG_MIXED = 1
SFC_SOLVER_FCG_MPNN = 2
SFC_PRECOND_JACOBI = 0
SFC_PRECOND_BLOCK_JACOBI = 1
SFC_PRECOND_TWO_LEVEL = 2
# status codes of include/statfem_cuda.h
SFC_ERR_CUDA = -1
SFC_ERR_BAD_ARG = -2
SFC_ERR_NOT_SPD = -3
SFC_ERR_NOT_CONVERGED = -4
SFC_ERR_TIMEOUT = -5
SFC_ERR_NO_MEMORY = -6
SFC_ERR_NEG_JACOBIAN = -7
SFC_ERR_TOO_LARGE = -8

_ERR = {-1: "CUDA error", -2: "bad argument", -3: "not SPD", -4: "not converged", -5: "timeout",
        -6: "out of memory", -7: "negative Jacobian", -8: "too large for the fixed scratch"}


class SfcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (_ERR.get(code, "error"), code, msg))
        self.code = code


class SolverOptions(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int32), ("max_iter", ctypes.c_int32), ("tol", ctypes.c_double),
                ("inner_tol", ctypes.c_double), ("block_width", ctypes.c_int32),
                ("check_every", ctypes.c_int32), ("precond", ctypes.c_int32),
                ("coarse_size", ctypes.c_int32)]


class SolveStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("refinements", ctypes.c_int32),
                ("num_rhs", ctypes.c_int32), ("converged", ctypes.c_int32),
                ("max_rel_residual", ctypes.c_double), ("device_ms", ctypes.c_double),
                ("fallback_columns", ctypes.c_int32), ("coarse_dofs", ctypes.c_int32),
                ("spmm_kernel", ctypes.c_int32), ("reserved", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class HParams(ctypes.Structure):
    _fields_ = [("forcing_sigma", ctypes.c_double), ("forcing_length", ctypes.c_double),
                ("rho", ctypes.c_double), ("mismatch_sigma", ctypes.c_double),
                ("mismatch_length", ctypes.c_double), ("mismatch_sensor_eps", ctypes.c_double)]

    @classmethod
    def from_map(cls, hp):
        g = lambda k: float(hp.get(k, 0.0))  # noqa: E731
        return cls(g("forcing.sigma"), g("forcing.length"), g("rho"), g("mismatch.sigma"),
                   g("mismatch.length"), g("mismatch.sensorEps"))


class MpnnTrainOptions(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int32), ("batch", ctypes.c_int32), ("max_pairs", ctypes.c_int32),
                ("normalize", ctypes.c_int32), ("lr", ctypes.c_double), ("pair_floor", ctypes.c_double),
                ("seed", ctypes.c_uint64)]


_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_d = ctypes.c_double

# name -> (restype, argtypes); the complete exported surface of the header
SIGNATURES = {
    "sfc_version": (_i32, []),
    "sfc_ctx_create": (_i32, [_i32, ctypes.POINTER(_vp)]),
    "sfc_ctx_destroy": (_i32, [_vp]),
    "sfc_last_error": (ctypes.c_char_p, [_vp]),
    "sfc_ctx_synchronize": (_i32, [_vp]),
    "sfc_ctx_kernel_launches": (_i32, [_vp, _i64p]),
    "sfc_ctx_graph_launches": (_i32, [_vp, _i64p]),
    "sfc_ctx_mark": (_i32, [_vp, _i32]),
    "sfc_ctx_marker_ms": (_i32, [_vp, _i32, _i32, _dp]),
    "sfc_ctx_set_profiling": (_i32, [_vp, _i32]),
    "sfc_ctx_profile_report": (_i32, [_vp, ctypes.c_char_p, _i64]),
    "sfc_mesh_create": (_i32, [_vp, _i32, _i32, _dp, _i64, _u32p, _i64, ctypes.POINTER(_vp)]),
    "sfc_mesh_destroy": (_i32, [_vp]),
    "sfc_mesh_set_coefficients": (_i32, [_vp, _dp, _d, _d]),
    "sfc_mesh_num_dofs": (_i64, [_vp]),
    "sfc_mesh_nnz": (_i64, [_vp]),
    "sfc_system_create": (_i32, [_vp, _i64, ctypes.POINTER(_vp)]),
    "sfc_system_destroy": (_i32, [_vp]),
    "sfc_system_set_options": (_i32, [_vp, ctypes.POINTER(SolverOptions)]),
    "sfc_system_get_options": (_i32, [_vp, ctypes.POINTER(SolverOptions)]),
    "sfc_system_last_stats": (_i32, [_vp, ctypes.POINTER(SolveStats)]),
    "sfc_insert_matrix": (_i32, [_vp, _dp, _u32p, ctypes.c_uint32, _u32p, ctypes.c_uint32]),
    "sfc_insert_rhs": (_i32, [_vp, _dp, _u32p, ctypes.c_uint32]),
    "sfc_finish_assembly": (_i32, [_vp]),
    "sfc_assemble_matrix": (_i32, [_vp, _vp]),
    "sfc_assemble_load": (_i32, [_vp, _vp, _dp]),
    "sfc_apply_constraints": (_i32, [_vp, _u32p, _dp, _i64, _d, _d]),
    "sfc_fix_dof": (_i32, [_vp, ctypes.c_uint32, _d]),
    "sfc_solve": (_i32, [_vp, _i32]),
    "sfc_solve_transpose": (_i32, [_vp, _dp, _dp, _i32, _i32]),
    "sfc_solve_multi": (_i32, [_vp, _dp, _dp, _i32]),
    "sfc_solve_multi_device": (_i32, [_vp, _vp, _vp, _i32, _i32]),
    "sfc_give_solution": (_i32, [_vp, _u32p, _i64, _dp]),
    "sfc_give_force": (_i32, [_vp, _u32p, _i64, _dp]),
    "sfc_clear_matrix": (_i32, [_vp]),
    "sfc_clear_rhs": (_i32, [_vp]),
    "sfc_num_nonzeros": (_i64, [_vp]),
    "sfc_norms": (_i32, [_vp, _dp, _dp, _dp, _dp]),
    "sfc_get_csr": (_i32, [_vp, _i64p, _i32p, _dp]),
    "sfc_covar_forcing_create": (_i32, [_vp, _vp, ctypes.POINTER(_vp)]),
    "sfc_covar_forcing_destroy": (_i32, [_vp]),
    "sfc_covar_forcing_apply_constraints": (_i32, [_vp, _u32p, _i64]),
    "sfc_covar_forcing_get_phibar": (_i32, [_vp, _dp]),
    "sfc_covar_forcing_projected": (_i32, [_vp, ctypes.POINTER(HParams), _dp, _i64, _dp]),
    "sfc_forward_gauss_create": (_i32, [_vp, _vp, _d, ctypes.POINTER(_vp)]),
    "sfc_forward_gauss_destroy": (_i32, [_vp]),
    "sfc_forward_gauss_set_projection": (_i32, [_vp, _i64, _i64p, _i32p, _dp]),
    "sfc_forward_gauss_update": (_i32, [_vp, ctypes.POINTER(HParams)]),
    "sfc_forward_gauss_mean": (_i32, [_vp, _dp]),
    "sfc_forward_gauss_covar": (_i32, [_vp, _dp]),
    "sfc_koh_create": (_i32, [_vp, _dp, _i32, ctypes.POINTER(_vp)]),
    "sfc_koh_destroy": (_i32, [_vp]),
    "sfc_koh_set_sensor_values": (_i32, [_vp, _dp, _i32]),
    "sfc_koh_log_likelihood": (_i32, [_vp, ctypes.POINTER(HParams), _dp]),
    "sfc_koh_proj_conditioned": (_i32, [_vp, ctypes.POINTER(HParams), _dp, _dp]),
    "sfc_koh_woodbury": (_i32, [_vp, ctypes.POINTER(HParams), _dp, _dp]),
    "sfc_koh_woodbury_mean": (_i32, [_vp, ctypes.POINTER(HParams), _dp]),
    "sfc_koh_log_likelihood_batch": (_i32, [_vp, ctypes.POINTER(HParams), _i32, _dp]),
    "sfc_perturbation_create": (_i32, [_vp, _d, ctypes.POINTER(_vp)]),
    "sfc_perturbation_destroy": (_i32, [_vp]),
    "sfc_perturbation_update": (_i32, [_vp, ctypes.POINTER(HParams), _d, _d, _d, _i32, _i32p]),
    "sfc_perturbation_mean": (_i32, [_vp, _dp]),
    "sfc_perturbation_covar": (_i32, [_vp, _dp]),
    "sfc_koh_log_likelihood_noalloc": (_i32, [_vp, _vp, _vp, _i32, _vp, _i32, _i32, ctypes.POINTER(HParams), _vp,
                                              _vp, _vp]),
    "sfc_mpnn_num_params": (_i64, []),
    "sfc_mpnn_create": (_i32, [_vp, ctypes.c_uint64, ctypes.POINTER(_vp)]),
    "sfc_mpnn_destroy": (_i32, [_vp]),
    "sfc_mpnn_get_params": (_i32, [_vp, _fp, _i64]),
    "sfc_mpnn_set_params": (_i32, [_vp, _fp, _i64]),
    "sfc_mpnn_save": (_i32, [_vp, ctypes.c_char_p]),
    "sfc_mpnn_load": (_i32, [_vp, ctypes.c_char_p]),
    "sfc_mpnn_loss_grad": (_i32, [_vp, _vp, _dp, _dp, _dp, _fp]),
    "sfc_mpnn_apply": (_i32, [_vp, _vp, _dp, _dp]),
    "sfc_mpnn_default_train_options": (_i32, [ctypes.POINTER(MpnnTrainOptions)]),
    "sfc_mpnn_train": (_i32, [_vp, _vp, ctypes.POINTER(MpnnTrainOptions), _dp]),
    "sfc_system_set_mpnn": (_i32, [_vp, _vp]),
    "sfc_batch_create": (_i32, [_vp, _vp, _i32, _i64p, _i32p, _u32p, _i64, _i32p, _i32p, _dp, _dp, _d, _i32,
                                ctypes.POINTER(_vp)]),
    "sfc_batch_destroy": (_i32, [_vp]),
    "sfc_batch_cluster_size": (_i32, [_vp, _i32p, _i32p]),
    "sfc_batch_set_solver": (_i32, [_vp, _d, _d, _i32]),
    "sfc_batch_set_coefficients": (_i32, [_vp, _dp]),
    "sfc_batch_set_hparams": (_i32, [_vp, ctypes.POINTER(HParams), _d]),
    "sfc_batch_set_readings": (_i32, [_vp, _dp, _i32]),
    "sfc_batch_run": (_i32, [_vp]),
    "sfc_batch_results": (_i32, [_vp, _dp, _dp, _dp, _dp, _dp, _i32p, _i32p]),
    "sfc_batch_autotune": (_i32, [_vp, _i32, _i32p]),
    "sfc_autotune_spmv": (_i32, [_vp, _i32, _i32p]),
    "sfc_autotune_block_solver": (_i32, [_vp, _dp, _i32, _i32, ctypes.POINTER(SolverOptions)]),
    "sfc_autotune_save": (_i32, [ctypes.c_char_p]),
    "sfc_autotune_load": (_i32, [ctypes.c_char_p]),
    "sfc_autotune_clear": (_i32, []),
    "sfc_coarse_boxes": (_i32, [_dp, _i64, _u32p, _i64, _i32, _i32, _i32, _i32p, _i32p, _i32p]),
}

_lib = None


def load():
    """Load the CUDA library; raises when it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libstatfem_cuda.so not built: run `python -m statfem_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _arr(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


class Context:
    def __init__(self, device=0):
        self.lib = load()
        h = _vp()
        rc = self.lib.sfc_ctx_create(device, ctypes.byref(h))
        if rc:
            raise SfcError(rc, "context creation failed")
        self.h = h

    def check(self, rc):
        if rc:
            raise SfcError(rc, self.lib.sfc_last_error(self.h).decode())

    def synchronize(self):
        self.check(self.lib.sfc_ctx_synchronize(self.h))

    def kernel_launches(self):
        c = ctypes.c_int64()
        self.check(self.lib.sfc_ctx_kernel_launches(self.h, ctypes.byref(c)))
        return c.value

    def last_message(self):
        """The context's last message (the last error, or a note such as a
        graph capture that fell back to separate launches)."""
        return self.lib.sfc_last_error(self.h).decode()

    def graph_launches(self):
        v = ctypes.c_int64()
        self.check(self.lib.sfc_ctx_graph_launches(self.h, ctypes.byref(v)))
        return v.value

    def mark(self, slot):
        self.check(self.lib.sfc_ctx_mark(self.h, slot))

    def marker_ms(self, a, b):
        v = ctypes.c_double()
        self.check(self.lib.sfc_ctx_marker_ms(self.h, a, b, ctypes.byref(v)))
        return v.value

    def set_profiling(self, enable=True):
        self.check(self.lib.sfc_ctx_set_profiling(self.h, int(bool(enable))))

    def profile_report(self):
        """{kernel name: (launches, total_ms, algorithmic_bytes)}; clears the records."""
        buf = ctypes.create_string_buffer(1 << 16)
        self.check(self.lib.sfc_ctx_profile_report(self.h, buf, len(buf)))
        out = {}
        for line in buf.value.decode().splitlines():
            name, n, ms, b = line.split()
            out[name] = (int(n), float(ms), float(b))
        return out

    def close(self):
        if getattr(self, "h", None):
            self.lib.sfc_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Mesh:
    """corlib::Mesh + per-element material; builds the CSR pattern on the GPU."""

    def __init__(self, ctx, kind, quad_points, coords, conn):
        self.ctx = ctx
        self.kind = kind
        self.coords = _arr(coords, np.float64)
        self.conn = _arr(conn, np.uint32)
        h = _vp()
        ctx.check(ctx.lib.sfc_mesh_create(ctx.h, kind, quad_points, _p(self.coords, _dp), self.coords.shape[0],
                                          _p(self.conn, _u32p), self.conn.shape[0], ctypes.byref(h)))
        self.h = h
        self.num_dofs = ctx.lib.sfc_mesh_num_dofs(h)
        self.nnz = ctx.lib.sfc_mesh_nnz(h)

    @classmethod
    def from_meshgen(cls, ctx, m, quad_points):
        return cls(ctx, m.kind, quad_points, m.coords, m.conn)

    def set_coefficients(self, values=None, uniform=1.0, poisson_ratio=0.3):
        v = None if values is None else _arr(values, np.float64)
        self.ctx.check(self.ctx.lib.sfc_mesh_set_coefficients(self.h, _p(v, _dp), uniform, poisson_ratio))

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.sfc_mesh_destroy(self.h)
            self.h = None


class SystemSolveCuda:
    """corlib::SystemSolveEigenSparse method set on the GPU."""

    def __init__(self, ctx, num_dofs):
        self.ctx = ctx
        self.N = int(num_dofs)
        h = _vp()
        ctx.check(ctx.lib.sfc_system_create(ctx.h, self.N, ctypes.byref(h)))
        self.h = h

    # -- options / stats (no reference counterpart) --
    def set_options(self, method=SFC_SOLVER_PCG_FP64, tol=1e-8, max_iter=20000, inner_tol=1e-4,
                    block_width=0, check_every=16, precond=SFC_PRECOND_JACOBI, coarse_size=0):
        o = SolverOptions(method, max_iter, tol, inner_tol, block_width, check_every, precond, coarse_size)
        self.ctx.check(self.ctx.lib.sfc_system_set_options(self.h, ctypes.byref(o)))

    def get_options(self):
        o = SolverOptions()
        self.ctx.check(self.ctx.lib.sfc_system_get_options(self.h, ctypes.byref(o)))
        return {k: getattr(o, k) for k, _ in o._fields_}

    def autotune_spmv(self, remeasure=False):
        v = ctypes.c_int32()
        self.ctx.check(self.ctx.lib.sfc_autotune_spmv(self.h, int(bool(remeasure)), ctypes.byref(v)))
        return v.value

    def autotune_block_solver(self, rhs, remeasure=False):
        """Tune block width and preconditioner of the mixed solver on these
        right-hand sides (nrhs x num_dofs); returns the chosen options."""
        R = _arr(rhs, np.float64).reshape(-1, self.N)
        o = SolverOptions()
        self.ctx.check(self.ctx.lib.sfc_autotune_block_solver(self.h, _p(R, _dp), R.shape[0], int(bool(remeasure)),
                                                              ctypes.byref(o)))
        return {k: getattr(o, k) for k, _ in o._fields_}

    def last_stats(self):
        s = SolveStats()
        self.ctx.check(self.ctx.lib.sfc_system_last_stats(self.h, ctypes.byref(s)))
        return s.as_dict()

    # -- insertion (compat path) --
    def insertToMatrix(self, Ke, rows, cols):
        Ke = _arr(Ke, np.float64)
        r = _arr(rows, np.uint32)
        c = _arr(cols, np.uint32)
        self.ctx.check(self.ctx.lib.sfc_insert_matrix(self.h, _p(Ke, _dp), _p(r, _u32p), len(r), _p(c, _u32p),
                                                      len(c)))

    def insertToRhs(self, fe, dofs):
        fe = _arr(fe, np.float64)
        d = _arr(dofs, np.uint32)
        self.ctx.check(self.ctx.lib.sfc_insert_rhs(self.h, _p(fe, _dp), _p(d, _u32p), len(d)))

    def finishAssembly(self):
        self.ctx.check(self.ctx.lib.sfc_finish_assembly(self.h))

    finishMatAssembly = finishAssembly
    finishRhsAssembly = finishAssembly

    # -- GPU assembler --
    def assemble(self, mesh):
        self.ctx.check(self.ctx.lib.sfc_assemble_matrix(self.h, mesh.h))

    def assemble_load(self, mesh, f):
        f = _arr(np.atleast_1d(f), np.float64)
        self.ctx.check(self.ctx.lib.sfc_assemble_load(self.h, mesh.h, _p(f, _dp)))

    # -- constraints --
    def applyConstraints(self, constraints, factor=1.0, scalar=1.0):
        """constraints: iterable of (dof, value) pairs, or (idx_array, value_array)."""
        if isinstance(constraints, tuple) and len(constraints) == 2 and hasattr(constraints[0], "__len__"):
            idx, val = constraints
        else:
            pairs = list(constraints)
            idx = [p[0] for p in pairs]
            val = [p[1] for p in pairs]
        idx = _arr(idx, np.uint32)
        val = _arr(val, np.float64)
        self.ctx.check(self.ctx.lib.sfc_apply_constraints(self.h, _p(idx, _u32p), _p(val, _dp), len(idx), factor,
                                                          scalar))

    def fixDOF(self, index, scalar=1.0):
        self.ctx.check(self.ctx.lib.sfc_fix_dof(self.h, int(index), scalar))

    # -- solves --
    def solveSystem(self, reuse=False):
        self.ctx.check(self.ctx.lib.sfc_solve(self.h, int(bool(reuse))))

    def solveSystemTranspose(self, rhs, reuse=False):
        rhs = _arr(rhs, np.float64)
        single = rhs.ndim == 1
        R = rhs.reshape(1, -1) if single else rhs
        U = np.zeros_like(R)
        self.ctx.check(self.ctx.lib.sfc_solve_transpose(self.h, _p(R, _dp), _p(U, _dp), R.shape[0],
                                                        int(bool(reuse))))
        return U[0] if single else U

    def solveSystemMulti(self, rhs):
        """A U = B for the rows of rhs (nrhs x num_dofs)."""
        R = _arr(rhs, np.float64).reshape(-1, self.N)
        U = np.zeros_like(R)
        self.ctx.check(self.ctx.lib.sfc_solve_multi(self.h, _p(R, _dp), _p(U, _dp), R.shape[0]))
        return U

    def solve_multi_device(self, rhs_ptr, u_ptr, nrhs, ld=None):
        """Device-memory variant: interleaved [num_dofs][ld] arrays given as
        device addresses (integers)."""
        self.ctx.check(self.ctx.lib.sfc_solve_multi_device(self.h, rhs_ptr, u_ptr, int(nrhs),
                                                           int(nrhs if ld is None else ld)))

    def giveSolution(self, dofs=None):
        d = _arr(np.arange(self.N) if dofs is None else dofs, np.uint32)
        out = np.zeros(len(d))
        self.ctx.check(self.ctx.lib.sfc_give_solution(self.h, _p(d, _u32p), len(d), _p(out, _dp)))
        return out

    def giveForce(self, dofs=None):
        d = _arr(np.arange(self.N) if dofs is None else dofs, np.uint32)
        out = np.zeros(len(d))
        self.ctx.check(self.ctx.lib.sfc_give_force(self.h, _p(d, _u32p), len(d), _p(out, _dp)))
        return out

    def clearMatrix(self):
        self.ctx.check(self.ctx.lib.sfc_clear_matrix(self.h))

    def clearRhs(self):
        self.ctx.check(self.ctx.lib.sfc_clear_rhs(self.h))

    def numNonZeros(self):
        return self.ctx.lib.sfc_num_nonzeros(self.h)

    def _norms(self):
        v = [ctypes.c_double() for _ in range(4)]
        self.ctx.check(self.ctx.lib.sfc_norms(self.h, *[ctypes.byref(x) for x in v]))
        return [x.value for x in v]

    def normMatrix(self):
        return self._norms()[0]

    def normRhs(self):
        return self._norms()[1]

    def norm1Rhs(self):
        return self._norms()[2]

    def normSol(self):
        return self._norms()[3]

    def get_csr(self):
        nnz = self.numNonZeros()
        rp = np.zeros(self.N + 1, dtype=np.int64)
        col = np.zeros(nnz, dtype=np.int32)
        val = np.zeros(nnz)
        self.ctx.check(self.ctx.lib.sfc_get_csr(self.h, _p(rp, _i64p), _p(col, _i32p), _p(val, _dp)))
        return rp, col, val

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.sfc_system_destroy(self.h)
            self.h = None


class CovarianceForcing:
    """statX::infer::CovarianceForcing with phibar computed on the GPU."""

    def __init__(self, ctx, mesh):
        self.ctx = ctx
        self.mesh = mesh
        h = _vp()
        ctx.check(ctx.lib.sfc_covar_forcing_create(ctx.h, mesh.h, ctypes.byref(h)))
        self.h = h

    def applyConstraints(self, idx):
        idx = _arr(idx, np.uint32)
        self.ctx.check(self.ctx.lib.sfc_covar_forcing_apply_constraints(self.h, _p(idx, _u32p), len(idx)))

    def phibar(self):
        out = np.zeros(self.mesh.num_dofs)
        self.ctx.check(self.ctx.lib.sfc_covar_forcing_get_phibar(self.h, _p(out, _dp)))
        return out

    def giveProjectedCovar(self, hp, M):
        M = _arr(M, np.float64)
        out = np.zeros((M.shape[0], M.shape[0]))
        h = HParams.from_map(hp)
        self.ctx.check(self.ctx.lib.sfc_covar_forcing_projected(self.h, ctypes.byref(h), _p(M, _dp), M.shape[0],
                                                                _p(out, _dp)))
        return out

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.sfc_covar_forcing_destroy(self.h)
            self.h = None


class ForwardGaussRHS:
    """statX::infer::ForwardGaussRHS on the GPU (block adjoint solve)."""

    def __init__(self, solver, covar_forcing, reg_eps=1e-4):
        self.ctx = solver.ctx
        self.solver = solver
        h = _vp()
        self.ctx.check(self.ctx.lib.sfc_forward_gauss_create(solver.h, covar_forcing.h, reg_eps, ctypes.byref(h)))
        self.h = h
        self.ns = 0

    def setProjectionMatrix(self, P):
        """P: dense (ns x N) array or CSR triple (indptr, indices, data)."""
        if isinstance(P, tuple):
            ip, ix, dv = P
        else:
            P = np.asarray(P, dtype=np.float64)
            ip = [0]
            ix, dv = [], []
            for a in range(P.shape[0]):
                nz = np.nonzero(P[a])[0]
                ix.extend(nz.tolist())
                dv.extend(P[a, nz].tolist())
                ip.append(len(ix))
        ip = _arr(ip, np.int64)
        ix = _arr(ix, np.int32)
        dv = _arr(dv, np.float64)
        self.ns = len(ip) - 1
        self.ctx.check(self.ctx.lib.sfc_forward_gauss_set_projection(self.h, self.ns, _p(ip, _i64p), _p(ix, _i32p),
                                                                     _p(dv, _dp)))

    def updateSolution(self, hp):
        h = HParams.from_map(hp)
        self.ctx.check(self.ctx.lib.sfc_forward_gauss_update(self.h, ctypes.byref(h)))

    def giveProjectedMeanU(self):
        out = np.zeros(self.ns)
        self.ctx.check(self.ctx.lib.sfc_forward_gauss_mean(self.h, _p(out, _dp)))
        return out

    def giveProjectedCovarU(self):
        out = np.zeros((self.ns, self.ns))
        self.ctx.check(self.ctx.lib.sfc_forward_gauss_covar(self.h, _p(out, _dp)))
        return out

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.sfc_forward_gauss_destroy(self.h)
            self.h = None


class LikelihoodKOH:
    """statX::infer::LikelihoodKOH with MismatchCovariance(sensorCoords)."""

    def __init__(self, forward_gauss, sensor_coords):
        self.ctx = forward_gauss.ctx
        self.fg = forward_gauss
        xs = _arr(sensor_coords, np.float64)
        if xs.ndim == 1:
            xs = xs.reshape(-1, 1)
        h = _vp()
        self.ctx.check(self.ctx.lib.sfc_koh_create(forward_gauss.h, _p(xs, _dp), xs.shape[1], ctypes.byref(h)))
        self.h = h
        self.ns = xs.shape[0]

    def setSensorValues(self, Y):
        Y = _arr(Y, np.float64)
        self.ctx.check(self.ctx.lib.sfc_koh_set_sensor_values(self.h, _p(Y, _dp), Y.shape[1]))

    def giveLogLikelihood(self, hp):
        h = HParams.from_map(hp)
        v = ctypes.c_double()
        self.ctx.check(self.ctx.lib.sfc_koh_log_likelihood(self.h, ctypes.byref(h), ctypes.byref(v)))
        return v.value

    def giveProjFEconditionedData(self, hp):
        h = HParams.from_map(hp)
        m = np.zeros(self.ns)
        c = np.zeros((self.ns, self.ns))
        self.ctx.check(self.ctx.lib.sfc_koh_proj_conditioned(self.h, ctypes.byref(h), _p(m, _dp), _p(c, _dp)))
        return m, c

    def giveLogLikelihoodBatch(self, hps):
        """giveLogLikelihood for a list of hyperparameter maps in one launch."""
        arr = (HParams * len(hps))(*[HParams.from_map(h) for h in hps])
        out = np.zeros(len(hps))
        self.ctx.check(self.ctx.lib.sfc_koh_log_likelihood_batch(self.h, arr, len(hps), _p(out, _dp)))
        return out

    def giveFEconditionedMeanWoodbury(self, hp):
        """The posterior mean field of giveFEconditionedDataWoodbury at
        sensor-space cost (any mesh size)."""
        h = HParams.from_map(hp)
        m = np.zeros(self.fg.solver.N)
        self.ctx.check(self.ctx.lib.sfc_koh_woodbury_mean(self.h, ctypes.byref(h), _p(m, _dp)))
        return m

    def giveFEconditionedDataWoodbury(self, hp, with_cov=True):
        h = HParams.from_map(hp)
        N = self.fg.solver.N
        m = np.zeros(N)
        c = np.zeros((N, N)) if with_cov else None
        self.ctx.check(self.ctx.lib.sfc_koh_woodbury(self.h, ctypes.byref(h), _p(m, _dp), _p(c, _dp)))
        return m, c

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.sfc_koh_destroy(self.h)
            self.h = None


class ForwardPerturbation:
    """statX::infer::ForwardPerturbation: prior mean and covariance at the
    sensors with first-order material (conductivity) uncertainty; hp is the
    reference's map including "material.sigma" and "material.length"."""

    def __init__(self, forward_gauss, reg=1e-4):
        self.fg = forward_gauss
        self.ctx = forward_gauss.ctx
        h = _vp()
        self.ctx.check(self.ctx.lib.sfc_perturbation_create(forward_gauss.h, float(reg), ctypes.byref(h)))
        self.h = h
        self.rank = 0

    def updateSolution(self, hp, factor_tol=1e-12, max_rank=4096):
        h = HParams.from_map(hp)
        r = ctypes.c_int32()
        self.ctx.check(self.ctx.lib.sfc_perturbation_update(self.h, ctypes.byref(h), float(hp["material.sigma"]),
                                                            float(hp["material.length"]), float(factor_tol),
                                                            int(max_rank), ctypes.byref(r)))
        self.rank = r.value

    def giveProjectedMeanU(self):
        m = np.zeros(self.fg.ns)
        self.ctx.check(self.ctx.lib.sfc_perturbation_mean(self.h, _p(m, _dp)))
        return m

    def giveProjectedCovarU(self):
        c = np.zeros((self.fg.ns, self.fg.ns))
        self.ctx.check(self.ctx.lib.sfc_perturbation_covar(self.h, _p(c, _dp)))
        return c

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.sfc_perturbation_destroy(self.h)
            self.h = None


class LearnedPreconditioner:
    """Message-passing network M(r) ~ S^-1 r used by flexible CG
    (SFC_SOLVER_FCG_MPNN); no counterpart in the reference, which factorises
    with Eigen::SparseLU."""

    def __init__(self, ctx, seed=0):
        self.ctx = ctx
        h = _vp()
        ctx.check(ctx.lib.sfc_mpnn_create(ctx.h, int(seed), ctypes.byref(h)))
        self.h = h
        self.num_params = int(ctx.lib.sfc_mpnn_num_params())

    def get_params(self):
        out = np.zeros(self.num_params, dtype=np.float32)
        self.ctx.check(self.ctx.lib.sfc_mpnn_get_params(self.h, _p(out, _fp), self.num_params))
        return out

    def set_params(self, params):
        p = _arr(params, np.float32)
        if p.size != self.num_params:
            raise ValueError("expected %d parameters" % self.num_params)
        self.ctx.check(self.ctx.lib.sfc_mpnn_set_params(self.h, _p(p, _fp), self.num_params))

    def save(self, path):
        self.ctx.check(self.ctx.lib.sfc_mpnn_save(self.h, str(path).encode()))

    def load(self, path):
        self.ctx.check(self.ctx.lib.sfc_mpnn_load(self.h, str(path).encode()))

    def loss_grad(self, system, r, e):
        r = _arr(r, np.float64)
        e = _arr(e, np.float64)
        loss = ctypes.c_double()
        g = np.zeros(self.num_params, dtype=np.float32)
        self.ctx.check(self.ctx.lib.sfc_mpnn_loss_grad(self.h, system.h, _p(r, _dp), _p(e, _dp), ctypes.byref(loss),
                                                       _p(g, _fp)))
        return loss.value, g

    def apply(self, system, r):
        r = _arr(r, np.float64)
        z = np.zeros_like(r)
        self.ctx.check(self.ctx.lib.sfc_mpnn_apply(self.h, system.h, _p(r, _dp), _p(z, _dp)))
        return z

    def train(self, system, **opts):
        """Adam on pairs from Jacobi-PCG on `system` (options: steps, batch,
        max_pairs, normalize, lr, pair_floor, seed); returns the loss per step."""
        o = MpnnTrainOptions()
        self.ctx.check(self.ctx.lib.sfc_mpnn_default_train_options(ctypes.byref(o)))
        for k, v in opts.items():
            if not hasattr(o, k):
                raise TypeError("unknown training option %r" % k)
            setattr(o, k, v)
        hist = np.zeros(max(o.steps, 1))
        self.ctx.check(self.ctx.lib.sfc_mpnn_train(self.h, system.h, ctypes.byref(o), _p(hist, _dp)))
        return hist[: o.steps]

    def attach(self, system):
        self.ctx.check(self.ctx.lib.sfc_system_set_mpnn(system.h, self.h))

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.sfc_mpnn_destroy(self.h)
            self.h = None


class BatchStatFEM:
    """Many independent 2-D Poisson statFEM instances (the blocks of one union
    mesh, e.g. MCMC proposals) evaluated by one persistent kernel in a CUDA
    graph: adjoint solves, prior mean / covariance at the sensors,
    LikelihoodKOH log-likelihood and sensor-space posterior per instance.
    sensors: per instance (P, coords) with P the (indptr, indices, data)
    projection rows in the instance's local dofs (<= 3 entries per row, at
    most 32 rows) and coords ns x 2."""

    MAX_SENSORS = 32

    def __init__(self, ctx, mesh, dof_offset, sides, bc_dofs, sensors, forcing_mean=1.0, cluster_size=0):
        self.ctx = ctx
        self.mesh = mesh
        off = _arr(dof_offset, np.int64)
        n = len(off) - 1
        self.n = n
        K = self.MAX_SENSORS
        ns = np.zeros(n, dtype=np.int32)
        sdof = -np.ones((n, K, 3), dtype=np.int32)
        sw = np.zeros((n, K, 3))
        sc = np.zeros((n, K, 2))
        for i, ((ip, ix, dv), xy) in enumerate(sensors):
            m = len(ip) - 1
            if m > K:
                raise ValueError("at most %d sensors per instance" % K)
            ns[i] = m
            for c in range(m):
                cnt = ip[c + 1] - ip[c]
                if cnt > 3:
                    raise ValueError("a projection row has more than 3 entries")
                sdof[i, c, :cnt] = off[i] + np.asarray(ix[ip[c]:ip[c + 1]])
                sw[i, c, :cnt] = dv[ip[c]:ip[c + 1]]
            sc[i, :m] = np.asarray(xy)[:, :2]
        self.ns = ns
        sides = _arr(sides, np.int32)
        bc = _arr(bc_dofs, np.uint32)
        h = _vp()
        ctx.check(ctx.lib.sfc_batch_create(ctx.h, mesh.h, n, _p(off, _i64p), _p(sides, _i32p), _p(bc, _u32p), len(bc),
                                           _p(ns, _i32p), _p(sdof, _i32p), _p(sw, _dp), _p(sc, _dp),
                                           float(forcing_mean), int(cluster_size), ctypes.byref(h)))
        self.h = h

    def autotune(self, remeasure=False):
        c = ctypes.c_int32()
        self.ctx.check(self.ctx.lib.sfc_batch_autotune(self.h, int(bool(remeasure)), ctypes.byref(c)))
        return c.value

    def launch_shape(self):
        c, g = ctypes.c_int32(), ctypes.c_int32()
        self.ctx.check(self.ctx.lib.sfc_batch_cluster_size(self.h, ctypes.byref(c), ctypes.byref(g)))
        return c.value, g.value

    def set_solver(self, tol=1e-8, inner_tol=1e-2, max_iter=50000):
        self.ctx.check(self.ctx.lib.sfc_batch_set_solver(self.h, tol, inner_tol, int(max_iter)))

    def set_coefficients(self, coeff):
        c = _arr(coeff, np.float64)
        self.ctx.check(self.ctx.lib.sfc_batch_set_coefficients(self.h, _p(c, _dp)))

    def set_hparams(self, hps, reg=1e-3):
        """hps: one reference-style hyperparameter map per instance (or one for all)."""
        if isinstance(hps, dict):
            hps = [hps] * self.n
        arr = (HParams * self.n)(*[HParams.from_map(h) for h in hps])
        self.ctx.check(self.ctx.lib.sfc_batch_set_hparams(self.h, arr, float(reg)))

    def set_readings(self, Y):
        """Y: n x ns_i x n_o (a list of per-instance arrays, or an n x 32 x n_o array)."""
        if isinstance(Y, np.ndarray) and Y.ndim == 3 and Y.shape[1] == self.MAX_SENSORS:
            full = _arr(Y, np.float64)
        else:
            n_o = np.asarray(Y[0]).reshape(len(Y[0]), -1).shape[1]
            full = np.zeros((self.n, self.MAX_SENSORS, n_o))
            for i, y in enumerate(Y):
                y = np.asarray(y, dtype=np.float64).reshape(len(y), -1)
                full[i, : y.shape[0]] = y
        self.ctx.check(self.ctx.lib.sfc_batch_set_readings(self.h, _p(full, _dp), full.shape[2]))

    def run(self):
        self.ctx.check(self.ctx.lib.sfc_batch_run(self.h))

    def results(self):
        n, K = self.n, self.MAX_SENSORS
        ll = np.zeros(n)
        ms = np.zeros((n, K))
        cs = np.zeros((n, K, K))
        pm = np.zeros((n, K))
        pc = np.zeros((n, K, K))
        st = np.zeros(n, dtype=np.int32)
        it = np.zeros(n, dtype=np.int32)
        self.ctx.check(self.ctx.lib.sfc_batch_results(self.h, _p(ll, _dp), _p(ms, _dp), _p(cs, _dp), _p(pm, _dp),
                                                      _p(pc, _dp), _p(st, _i32p), _p(it, _i32p)))
        return dict(loglik=ll, mean_s=ms, cov_s=cs, post_mean=pm, post_cov=pc, status=st, iterations=it)

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.sfc_batch_destroy(self.h)
            self.h = None


def autotune_save(path):
    lib = load()
    if lib.sfc_autotune_save(str(path).encode()):
        raise SfcError(-2, "cannot write %s" % path)


def autotune_load(path):
    lib = load()
    if lib.sfc_autotune_load(str(path).encode()):
        raise SfcError(-2, "cannot read %s" % path)


def autotune_clear():
    load().sfc_autotune_clear()


def coarse_boxes(coords, conn, size=8, max_aggs=512):
    """The two-level preconditioner's box aggregation of a mesh (host only):
    (aggregate per node, boxes per axis)."""
    X = _arr(coords, np.float64).reshape(-1, 3)
    C = _arr(conn, np.uint32)
    C2 = C.reshape(C.shape[0], -1) if C.ndim == 2 else C.reshape(-1, 1)
    agg = np.zeros(X.shape[0], dtype=np.int32)
    nagg = ctypes.c_int32()
    nb = np.zeros(3, dtype=np.int32)
    rc = load().sfc_coarse_boxes(_p(X, _dp), X.shape[0], _p(C2, _u32p), C2.shape[0], C2.shape[1], int(size),
                                 int(max_aggs), _p(agg, _i32p), ctypes.byref(nagg), _p(nb, _i32p))
    if rc != 0:
        raise SfcError(rc, "no box grid satisfies the one-box span rule")
    return agg, nb


__all__ = ["Context", "Mesh", "SystemSolveCuda", "CovarianceForcing", "ForwardGaussRHS", "LikelihoodKOH",
           "LearnedPreconditioner", "BatchStatFEM", "ForwardPerturbation", "SfcError", "SIGNATURES", "load", "meshgen", "SFC_SOLVER_PCG_FP64",
           "SFC_SOLVER_PCG_MIXED", "SFC_SOLVER_FCG_MPNN", "autotune_save", "autotune_load", "autotune_clear",
           "coarse_boxes"]
