"""Synthetic-input generators (host side)."""
import numpy as np

from statfem_b200 import meshgen as mg


def test_matern32_statistics():
    """Circulant-embedding Matérn nu=3/2 samples: marginal variance sigma^2
    and the lag-1 correlation (1 + sqrt(3) h/l) exp(-sqrt(3) h/l) along each
    axis, over 200 seeded 16^3 samples."""
    n, length = 16, 0.2
    F = np.stack([mg.matern32_field_cells(np.random.default_rng(s), n, 1.0, length).reshape(n, n, n)
                  for s in range(200)])
    v = F.var()
    assert abs(v - 1.0) < 0.06
    a = np.sqrt(3.0) * (1.0 / n) / length
    expect = (1 + a) * np.exp(-a)
    for ax in range(1, 4):
        lo = [slice(None)] * 4
        hi = [slice(None)] * 4
        lo[ax] = slice(0, -1)
        hi[ax] = slice(1, None)
        c = np.mean(F[tuple(lo)] * F[tuple(hi)]) / v
        assert abs(c - expect) < 0.02, (ax, c, expect)


def test_matern32_cell_order_matches_hex_elements():
    """Element e of unit_cube_hex has its centre at cell (ix, iy, iz) with x
    fastest; the field is laid out the same way (2-D check on a smooth field
    is enough to catch a transposition: shapes differ per axis)."""
    f2 = mg.matern32_field_cells(np.random.default_rng(0), 8, 1.0, 0.3, dim=2)
    assert f2.shape == (64,)
    m = mg.unit_cube_hex(4)
    c = m.centroids()
    assert np.allclose(c[1] - c[0], [0.25, 0, 0]) and np.allclose(c[4] - c[0], [0, 0.25, 0])
