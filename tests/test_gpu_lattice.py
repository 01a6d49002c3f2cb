"""The lattice SpMMs of the mixed block solver on 3-dof meshes whose nodes
form a structured lattice -- the streamed x-line kernel (the default) and the
TMA-staged brick kernel (SFC_SPMM=lattice) -- against the node-block kernel
(SFC_SPMM=bsr) and against the oracle's LU of A^T, on lattices whose sides
are not multiples of the brick (ragged bricks on every face) and whose x-lines
split across warps, for 32, 64 and 128 columns per block; and the 32-bit size
limit."""
import os

import numpy as np
import pytest

from statfem_b200 import api
from statfem_b200 import meshgen as mg
from tests.test_gpu_solve import setup

pytestmark = pytest.mark.gpu


KERNEL = {"xline": 4, "lattice": 3, "bsr": 2}


def solve(ctx, n, bw, precond, rhs_seed=4, nrhs=130, mode="xline"):
    # the operator (and with it the choice of SpMM) is built at solve time:
    # SFC_SPMM selects the staged bricks ("lattice") or the node blocks ("bsr")
    if mode != "xline":
        os.environ["SFC_SPMM"] = mode
    try:
        mesh, s, ds, F, bc = setup(ctx, mg.HEX8_ELASTIC, n, 17, amount=0.0, faces="x0")
        rng = np.random.default_rng(rhs_seed)
        Rhs = rng.standard_normal((nrhs, mesh.num_dofs))
        s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-10, block_width=bw, precond=precond)
        U = s.solveSystemTranspose(Rhs)
    finally:
        os.environ.pop("SFC_SPMM", None)
    st = s.last_stats()
    return U, st, ds, Rhs


@pytest.mark.parametrize("n,bw,mode", [(6, 128, "lattice"), (6, 64, "lattice"), (9, 128, "lattice"),
                                        (4, 64, "lattice"), (6, 128, "xline"), (6, 64, "xline"),
                                        (9, 128, "xline"), (4, 32, "xline"), (20, 128, "xline")])
@pytest.mark.parametrize("precond", [api.SFC_PRECOND_BLOCK_JACOBI, api.SFC_PRECOND_TWO_LEVEL])
def test_lattice_spmm_matches_lu_and_node_blocks(ctx, n, bw, mode, precond):
    U, st, ds, Rhs = solve(ctx, n, bw, precond, mode=mode)
    assert st["spmm_kernel"] == KERNEL[mode], st
    assert st["converged"] == 1 and st["max_rel_residual"] <= 1e-10
    refs = np.stack([ds.solve_transpose(r) for r in Rhs])
    assert np.abs(U - refs).max() <= 1e-7 * np.abs(refs).max()
    U2, st2, _, _ = solve(ctx, n, bw, precond, mode="bsr")
    assert st2["spmm_kernel"] == 2, st2
    assert np.abs(U2 - refs).max() <= 1e-7 * np.abs(refs).max()
    # the FP32 products differ only in summation order: iteration counts stay close
    assert abs(st["iterations"] - st2["iterations"]) <= max(8, st2["iterations"] // 5)


def test_distorted_mesh_keeps_node_blocks(ctx):
    """A mesh whose nodes are not a lattice uses the node-block kernel."""
    mesh, s, ds, F, bc = setup(ctx, mg.HEX8_ELASTIC, 4, 3, amount=0.3, faces="x0")
    Rhs = np.random.default_rng(1).standard_normal((64, mesh.num_dofs))
    s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-10, block_width=64, precond=api.SFC_PRECOND_BLOCK_JACOBI)
    U = s.solveSystemTranspose(Rhs)
    assert s.last_stats()["spmm_kernel"] == 2
    refs = np.stack([ds.solve_transpose(r) for r in Rhs])
    assert np.abs(U - refs).max() <= 1e-7 * np.abs(refs).max()


def test_system_beyond_32bit_indices_is_rejected(ctx):
    with pytest.raises(api.SfcError) as e:
        api.SystemSolveCuda(ctx, 2 ** 31)
    assert e.value.code == api.SFC_ERR_TOO_LARGE


@pytest.mark.parametrize("mode", ["lattice", "xline"])
@pytest.mark.parametrize("precond", [api.SFC_PRECOND_BLOCK_JACOBI, api.SFC_PRECOND_TWO_LEVEL])
def test_check_interval_graph_matches_eager_launches(ctx, precond, mode):
    """The mixed solver's check intervals replayed from a captured CUDA graph
    give the eager launch sequence's answer (the same kernels in the same
    order), with one graph launch per interval instead of a launch per
    kernel."""
    results = {}
    for mode in ("graph", "eager"):
        if mode == "eager":
            os.environ["SFC_BLOCK_GRAPH"] = "0"
        try:
            g0, k0 = ctx.graph_launches(), ctx.kernel_launches()
            U, st, ds, Rhs = solve(ctx, 5, 128, precond, nrhs=100, mode=mode)
            results[mode] = (U, st, ctx.graph_launches() - g0, ctx.kernel_launches() - k0)
        finally:
            os.environ.pop("SFC_BLOCK_GRAPH", None)
    Ug, stg, gg, kg = results["graph"]
    Ue, ste, ge, ke = results["eager"]
    refs = np.stack([ds.solve_transpose(r) for r in Rhs])
    for U in (Ug, Ue):
        assert np.abs(U - refs).max() <= 1e-7 * np.abs(refs).max()
    assert stg["converged"] == ste["converged"] == 1
    assert abs(stg["iterations"] - ste["iterations"]) <= 32
    # check_every is 16 here: one replay per 16 iterations (the coarse
    # inverse's own graphs are launched in both modes)
    assert gg - ge >= max(1, stg["iterations"] // 16 - 1), ctx.last_message()
    assert kg > 0 and ke > 0
