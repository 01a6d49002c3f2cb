"""The CPU oracle of the learned preconditioner checked against itself:
analytic gradient vs central finite differences (unrounded operands), and the
untrained network (zero decoder) equal to Jacobi."""
import numpy as np

from oracle import mpnn_ref as R
from oracle import oracle as O
from statfem_b200 import meshgen as mg
from tests import problems as pb


def _system(n=5, seed=3):
    pr = pb.statfem_problem(mg.HEX8_POISSON, n, 4, seed=seed)
    mesh = pr["mesh"]
    rp, col, val, F = O.fem(mesh, 8, 1.0, pr["bc"], coeff=pr["coeff"])
    mask = np.zeros(mesh.num_dofs, dtype=np.uint8)
    mask[pr["bc"]] = 1
    S = R.symmetric_operator(rp, col, val, mask)
    return S, mask


def test_oracle_gradient_finite_differences():
    S, mask = _system()
    Ahat, sdinv = R.scaled_operator(S)
    rng = np.random.default_rng(0)
    N = S.shape[0]
    p = R.init_params(1, decoder_scale=0.3).astype(np.float64)
    r = rng.standard_normal(N)
    e = rng.standard_normal(N)
    loss, g = R.loss_grad(p, Ahat, sdinv, mask, r, e, bf16_ops=False)
    assert np.isfinite(loss) and loss > 0
    # parameters from every block: encoder, each layer's W and b, decoder
    idx = [R.OFF_EW + 3, R.OFF_EB + 5, R.OFF_DW + 7, R.OFF_DB]
    for l in range(R.LAYERS):
        o = R.OFF_L + l * R.LSZ
        idx += [o + 17, o + 64 * 2 * 0 + 100, o + R.H * 2 * R.H + 9]
    h = 1e-6
    for k in idx:
        pp = p.copy()
        pm = p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (R.loss_grad(pp, Ahat, sdinv, mask, r, e, bf16_ops=False)[0] -
              R.loss_grad(pm, Ahat, sdinv, mask, r, e, bf16_ops=False)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(g[k])), (k, fd, g[k])


def test_oracle_zero_decoder_is_jacobi():
    S, mask = _system()
    Ahat, sdinv = R.scaled_operator(S)
    r = np.random.default_rng(1).standard_normal(S.shape[0])
    z = R.apply(R.init_params(2, decoder_scale=0.0), Ahat, sdinv, mask, r)
    np.testing.assert_allclose(z, r / S.diagonal(), rtol=2e-6)


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7 + 2 ** -9, -3.140625, 0.0])
    np.testing.assert_array_equal(R.bf16(v), [1.0, 1.0, 1.0 + 2 ** -7, -3.140625, 0.0])
