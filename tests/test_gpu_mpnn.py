"""Learned preconditioner on the GPU: forward/backward kernels against the CPU
oracle (oracle/mpnn_ref.py), flexible CG with the network, checkpoints, and
what training gains over plain Jacobi-PCG."""
import numpy as np
import pytest

from oracle import mpnn_ref as R
from oracle import oracle as O
from statfem_b200 import api
from statfem_b200 import meshgen as mg
from tests.problems import QPS, coefficients, small_mesh

pytestmark = pytest.mark.gpu


def setup(ctx, kind, n, seed, sigma=None):
    rng = np.random.default_rng(seed)
    mesh = small_mesh(kind, n, rng, 0.2)
    coeff = coefficients(mesh, rng, kind) if sigma is None else np.exp(sigma * rng.standard_normal(mesh.num_elems))
    gm = api.Mesh(ctx, kind, QPS[kind], mesh.coords, mesh.conn)
    gm.set_coefficients(coeff)
    s = api.SystemSolveCuda(ctx, mesh.num_dofs)
    s.assemble(gm)
    s.assemble_load(gm, np.array([1.0, -0.5, 0.25])[: mesh.dof])
    bc = mg.dirichlet_dofs(mesh, "all")
    s.applyConstraints((bc, np.zeros(len(bc))))
    rp, col, val, F = O.fem(mesh, QPS[kind], np.array([1.0, -0.5, 0.25])[: mesh.dof], bc, coeff=coeff)
    mask = np.zeros(mesh.num_dofs, dtype=np.uint8)
    mask[bc] = 1
    S = R.symmetric_operator(rp, col, val, mask)
    return mesh, s, S, F, O.DirectSolver(rp, col, val), mask


@pytest.mark.parametrize("kind,n", [(mg.HEX8_POISSON, 6), (mg.TRI3_POISSON, 14), (mg.HEX8_ELASTIC, 3)])
def test_loss_and_gradient_match_oracle(ctx, kind, n):
    """BF16 tensor-core forward and backward kernels vs the float64 oracle
    with the same BF16 rounding points: loss within 1e-4 relative, gradient
    within 1e-2 relative (2-norm, per parameter block) — the slack covers
    FP32 accumulation order and BF16 roundings that flip between FP32 and
    FP64 activations."""
    mesh, s, S, F, _, mask = setup(ctx, kind, n, 11)
    Ahat, sdinv = R.scaled_operator(S)
    net = api.LearnedPreconditioner(ctx, seed=0)
    assert net.num_params == R.NPARAM
    p = R.init_params(5, decoder_scale=0.3)
    net.set_params(p)
    np.testing.assert_array_equal(net.get_params(), p)
    rng = np.random.default_rng(2)
    r = rng.standard_normal(mesh.num_dofs) * 1e3
    e = rng.standard_normal(mesh.num_dofs) * 1e-2
    loss, g = net.loss_grad(s, r, e)
    loss_ref, g_ref = R.loss_grad(p, Ahat, sdinv, mask, r, e, bf16_ops=True)
    assert abs(loss - loss_ref) <= 1e-4 * abs(loss_ref)
    blocks = [(R.OFF_EW, R.OFF_EB), (R.OFF_EB, R.OFF_L)]
    for l in range(R.LAYERS):
        o = R.OFF_L + l * R.LSZ
        blocks += [(o, o + R.H * 2 * R.H), (o + R.H * 2 * R.H, o + R.LSZ)]
    blocks += [(R.OFF_DW, R.OFF_DB), (R.OFF_DB, R.NPARAM)]
    for a, b in blocks:
        err = np.linalg.norm(g[a:b] - g_ref[a:b])
        assert err <= 1e-2 * np.linalg.norm(g_ref[a:b]) + 1e-6 * np.linalg.norm(g_ref), (a, b, err)
    # the application M(r) by the inference kernels (BF16 activations)
    z = net.apply(s, r)
    z_ref = R.apply_inference(p, Ahat, sdinv, mask, r)
    assert np.linalg.norm(z - z_ref) <= 1e-3 * np.linalg.norm(z_ref)
    # and its distance from the FP32-activation forward the training uses
    z_tr = R.apply(p, Ahat, sdinv, mask, r)
    assert np.linalg.norm(z - z_tr) <= 3e-2 * np.linalg.norm(z_tr)
    net.close()


def test_untrained_network_is_jacobi(ctx):
    mesh, s, S, F, _, mask = setup(ctx, mg.HEX8_POISSON, 5, 3)
    net = api.LearnedPreconditioner(ctx, seed=7)
    r = np.random.default_rng(0).standard_normal(mesh.num_dofs)
    z = net.apply(s, r)
    np.testing.assert_allclose(z, r / S.diagonal(), rtol=1e-6)
    net.close()


def test_flexible_cg_solution(ctx):
    """FCG with a (random, non-trivial) network converges to the true FP64
    residual and matches the direct oracle."""
    mesh, s, S, F, ds, _ = setup(ctx, mg.HEX8_POISSON, 8, 4)
    net = api.LearnedPreconditioner(ctx, seed=1)
    net.set_params(R.init_params(9, decoder_scale=0.05))
    net.attach(s)
    s.set_options(method=api.SFC_SOLVER_FCG_MPNN, tol=1e-10)
    s.solveSystem()
    st = s.last_stats()
    assert st["converged"] == 1 and st["max_rel_residual"] <= 1e-10
    u = s.giveSolution()
    u_ref = ds.solve(F)
    assert np.abs(u - u_ref).max() <= 1e-8 * np.abs(u_ref).max()
    net.close()


def test_fcg_without_network_is_an_error(ctx):
    mesh, s, S, F, ds, _ = setup(ctx, mg.HEX8_POISSON, 4, 4)
    s.set_options(method=api.SFC_SOLVER_FCG_MPNN, tol=1e-8)
    with pytest.raises(api.SfcError):
        s.solveSystem()


def test_checkpoint_round_trip(ctx, tmp_path):
    mesh, s, S, F, _, mask = setup(ctx, mg.HEX8_POISSON, 5, 6)
    a = api.LearnedPreconditioner(ctx, seed=3)
    a.train(s, steps=20, lr=1e-3)
    a.save(tmp_path / "net.bin")
    b = api.LearnedPreconditioner(ctx, seed=4)
    b.load(tmp_path / "net.bin")
    np.testing.assert_array_equal(a.get_params(), b.get_params())
    r = np.random.default_rng(1).standard_normal(mesh.num_dofs)
    np.testing.assert_array_equal(a.apply(s, r), b.apply(s, r))
    (tmp_path / "bad.bin").write_bytes(b"not a checkpoint")
    with pytest.raises(api.SfcError):
        b.load(tmp_path / "bad.bin")
    a.close()
    b.close()


def test_training_gain(ctx):
    """Train on residual/error pairs of three heterogeneous 3-D Poisson
    problems (log-conductivity N(0, 1) per element), then solve a held-out
    sample with FCG and with plain FP64 Jacobi-PCG, both to the true relative
    residual 1e-8.  The untrained network is Jacobi, so FCG with it takes the
    PCG iteration count; the trained one must take at most 60% of it."""
    net = api.LearnedPreconditioner(ctx, seed=0)
    hist = []
    for k in range(3):
        _, s_tr, *_ = setup(ctx, mg.HEX8_POISSON, 16, 21 + k, sigma=1.0)
        hist.append(net.train(s_tr, steps=150, seed=k, lr=1e-3))
    hist = np.concatenate(hist)
    # normalised loss: the fraction of Jacobi's error energy left
    assert hist[:30].mean() > 0.4 and hist[-50:].mean() < 0.3
    _, s, S, F, ds, _ = setup(ctx, mg.HEX8_POISSON, 16, 99, sigma=1.0)
    s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-8, check_every=1)
    s.solveSystem()
    it_pcg = s.last_stats()["iterations"]
    base = api.LearnedPreconditioner(ctx, seed=0)
    base.attach(s)
    s.set_options(method=api.SFC_SOLVER_FCG_MPNN, tol=1e-8)
    s.solveSystem()
    it_jac = s.last_stats()["iterations"]
    net.attach(s)
    s.solveSystem()
    st = s.last_stats()
    assert st["converged"] == 1
    u_ref = ds.solve(F)
    assert np.abs(s.giveSolution() - u_ref).max() <= 1e-6 * np.abs(u_ref).max()
    print("training gain: PCG %d, FCG+untrained %d, FCG+trained %d iterations" % (it_pcg, it_jac, st["iterations"]))
    assert abs(it_jac - it_pcg) <= 2
    assert st["iterations"] <= 0.6 * it_pcg
    net.close()
    base.close()


def test_fcg_falls_back_to_jacobi_pcg(ctx):
    """A useless network (huge random decoder) stalls or breaks flexible CG;
    plain FP64 Jacobi-PCG then finishes the solve from the current iterate,
    and the answer still matches the direct oracle."""
    mesh, s, S, F, ds, _ = setup(ctx, mg.HEX8_POISSON, 10, 5)
    net = api.LearnedPreconditioner(ctx, seed=1)
    net.set_params(R.init_params(9, decoder_scale=300.0))
    net.attach(s)
    s.set_options(method=api.SFC_SOLVER_FCG_MPNN, tol=1e-10)
    s.solveSystem()
    st = s.last_stats()
    assert st["converged"] == 1 and st["max_rel_residual"] <= 1e-10
    assert st["fallback_columns"] == 1
    u_ref = ds.solve(F)
    assert np.abs(s.giveSolution() - u_ref).max() <= 1e-8 * np.abs(u_ref).max()
    net.close()
