"""Autotuner on the GPU: the tuned launch shapes are valid, the solves they
select still match the oracle, and a stored choice is reused."""
import numpy as np
import pytest

from statfem_b200 import api
from statfem_b200 import meshgen as mg
from tests.test_gpu_solve import setup

pytestmark = pytest.mark.gpu


def test_spmv_lanes(ctx, tmp_path):
    api.autotune_clear()
    mesh, s, ds, F, bc = setup(ctx, mg.HEX8_ELASTIC, 6, 3, faces="x0")
    lanes = s.autotune_spmv(remeasure=True)
    assert lanes in (4, 8, 16, 32)
    assert s.autotune_spmv() == lanes  # from the table
    s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-12)
    s.solveSystem()
    u_ref = ds.solve(F)
    assert np.abs(s.giveSolution() - u_ref).max() <= 1e-9 * np.abs(u_ref).max()
    api.autotune_save(tmp_path / "t.txt")
    assert "spmv:" in (tmp_path / "t.txt").read_text()


def test_block_solver_choice(ctx):
    api.autotune_clear()
    mesh, s, ds, F, bc = setup(ctx, mg.HEX8_ELASTIC, 5, 4, faces="x0")
    rng = np.random.default_rng(2)
    R = rng.standard_normal((70, mesh.num_dofs))
    s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-10)
    best = s.autotune_block_solver(R, remeasure=True)
    assert best["block_width"] in (32, 64, 128)
    assert best["precond"] in (api.SFC_PRECOND_JACOBI, api.SFC_PRECOND_BLOCK_JACOBI, api.SFC_PRECOND_TWO_LEVEL)
    if best["precond"] == api.SFC_PRECOND_TWO_LEVEL:
        assert best["coarse_size"] in (6, 8, 12)
    assert best["method"] == api.SFC_SOLVER_PCG_MIXED and best["tol"] == 1e-10
    U = s.solveSystemTranspose(R)
    U_ref = np.stack([ds.solve_transpose(r) for r in R])
    assert np.abs(U - U_ref).max() <= 1e-8 * np.abs(U_ref).max()
    assert s.autotune_block_solver(R) == best


def test_batch_cluster(ctx):
    from tests.test_gpu_batch import make_batch, run_gpu, rel
    pb = make_batch([6, 12, 9], [4, 6, 5], 8)
    b, _ = run_gpu(ctx, pb, 1e-3)
    r0 = b.results()
    cs = b.autotune(remeasure=True)
    assert cs in (1, 2, 4, 8, 16) and b.launch_shape()[0] == cs
    b.run()
    r1 = b.results()
    assert (r1["status"] == 0).all()
    assert rel(r1["cov_s"], r0["cov_s"]) < 1e-8
    b.close()
