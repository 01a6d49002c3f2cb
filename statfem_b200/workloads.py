"""The seeded synthetic workloads the benchmark and the parity tests share.

c1: 2-D Poisson statFEM on the unit square, 64 x 64 cells each split into two
    P1 triangles (4,225 dofs), kappa = 1, f = 1, u = 0 on the whole boundary,
    forcing GP squared-exponential sigma_f 0.1 length 0.2, 16 seeded interior
    sensors, sensor noise 1e-3.
c2: 3-D linear elasticity statFEM on the unit cube, 48^3 trilinear hex8
    elements (352,947 dofs), Young's modulus lognormal (log-GP squared-
    exponential sigma 0.3, length 0.25, sampled exactly on the element-centre
    grid), nu = 0.3, face x = 0 clamped, body-force mean (0, 0, -1) with a
    squared-exponential GP (sigma_f 0.05, length 0.3), 256 seeded sensors (one
    displacement component each, cycling x/y/z), sensor noise 1e-4.
c3: many independent 2-D Poisson statFEM instances of uneven size (MCMC
    material proposals): sides seeded-uniform in [32, 256] cells, log-
    conductivity squared-exponential (sigma 0.5, length seeded-uniform in
    [0.05, 0.5]) on the cell-centre grid, 32 sensors each.

Everything is drawn from numpy's seeded generator; no dataset is involved.
The reference's apps read the same kinds of inputs from files (SMF meshes,
sensor coordinates, projection rows); here they are generated in memory.
"""
from __future__ import annotations

import numpy as np

from . import meshgen as mg

# hyperparameter names as LikelihoodKOH / ForwardGaussRHS look them up
C2_HP = {"forcing.sigma": 0.05, "forcing.length": 0.3, "rho": 1.0, "mismatch.sigma": 0.0,
         "mismatch.length": 0.25, "mismatch.sensorEps": 1e-4}
C1_HP = dict(C2_HP, **{"forcing.sigma": 0.1, "forcing.length": 0.2, "mismatch.sensorEps": 1e-3})
C3_HP = {"forcing.sigma": 0.1, "forcing.length": 0.2, "rho": 1.0, "mismatch.sigma": 0.0,
         "mismatch.length": 0.2, "mismatch.sensorEps": 1e-3}
# ForwardGaussRHS regularisation (regEps) of the canonical laplaceRHSinfer app
REG = 0.001


def make_workload(config, seed, c2_n=48):
    """c1 or c2 inputs: mesh, element coefficients, Dirichlet dofs, sensor
    points and projection rows, load, hyperparameters; ``rng`` continues the
    seeded stream (the observations are drawn from it)."""
    rng = np.random.default_rng(seed)
    if config == "c2":
        n, ns = c2_n, 256
        mesh = mg.unit_cube_hex(n, mg.HEX8_ELASTIC)
        ax = mg.cell_centre_axes(n)
        g = mg.se_field_tensor(rng, [ax, ax, ax], 0.3, 0.25)
        coeff = np.exp(g)
        bc = mg.dirichlet_dofs(mesh, "x0")
        pts = mg.interior_points(rng, ns, 3, margin=0.02)
        comps = np.arange(ns) % 3
        P = mg.projection_matrix(mesh, pts, comps)
        f = np.array([0.0, 0.0, -1.0])
        hp = dict(C2_HP)
        desc = "3-D elasticity statFEM, %d^3 hex8 (%d dofs), 256 sensors, rel. residual 1e-8" % (n, mesh.num_dofs)
        qps = 8
    elif config == "c1":
        n, ns = 64, 16
        mesh = mg.unit_square_tri(n)
        coeff = np.ones(mesh.num_elems)
        bc = mg.dirichlet_dofs(mesh, "all")
        pts = mg.interior_points(rng, ns, 2, margin=0.02)
        P = mg.projection_matrix(mesh, pts)
        f = np.array([1.0])
        hp = dict(C1_HP)
        desc = "2-D Poisson statFEM, 64^2 cells x 2 P1 triangles (4,225 dofs), 16 sensors, rel. residual 1e-8"
        qps = 3
    else:
        raise ValueError("unknown config " + config)
    return dict(mesh=mesh, coeff=coeff, bc=bc, pts=pts, P=P, f=f, hp=hp, desc=desc, qps=qps, ns=ns, rng=rng)


def make_batch_workload(seed, n_inst=512, smin=32, smax=256, ns=32, sides=None):
    """c3: n_inst 2-D Poisson statFEM instances, side s ~ U{smin..smax} cells
    (or the given ``sides``), P1 triangles, log-conductivity squared-
    exponential (sigma 0.5, length ~ U[0.05, 0.5]) sampled exactly on the
    cell-centre grid (both triangles of a cell share the value), ns sensors at
    seeded interior points, forcing GP sigma_f 0.1 length 0.2, sensor noise
    1e-3."""
    rng = np.random.default_rng(seed)
    sides = rng.integers(smin, smax + 1, n_inst) if sides is None else np.asarray(sides, dtype=np.int64)
    meshes, coeffs, bcs, sensors = [], [], [], []
    for s in sides:
        s = int(s)
        mesh = mg.unit_square_tri(s)
        ax = mg.cell_centre_axes(s)
        g = mg.se_field_tensor(rng, [ax, ax], 0.5, rng.uniform(0.05, 0.5))
        coeffs.append(np.repeat(np.exp(g), 2))
        pts = mg.interior_points(rng, ns, 2, margin=0.02)
        sensors.append((mg.projection_matrix(mesh, pts), pts))
        bcs.append(mg.dirichlet_dofs(mesh, "all"))
        meshes.append(mesh)
    union, off = mg.disjoint_union(meshes)
    bc = np.concatenate([b + off[k] for k, b in enumerate(bcs)])
    return dict(sides=sides, meshes=meshes, coeff=np.concatenate(coeffs), coeffs=coeffs, bcs=bcs,
                sensors=sensors, union=union, off=off, bc=bc, ns=ns, rng=rng,
                desc="%d 2-D Poisson statFEM instances, sides U{%d..%d} (P1 triangles, %d dofs in total), "
                     "%d sensors each, log-likelihood + posterior at the sensors"
                     % (len(sides), int(sides.min()), int(sides.max()), int(off[-1]), ns))


def draw_readings(rng, mean_s, C_s, hp, n_o=1):
    """LikelihoodKOH::giveTypicalReadings (statX/infer/LikelihoodKOH.ipp:43-71):
    y ~ N(rho mean_s, K_s + rho^2 C_s) with the mismatch switched off
    (sigma_d = 0), K_s = eps^2 I; numpy's generator instead of mt19937."""
    ns = len(mean_s)
    C = hp["mismatch.sensorEps"] ** 2 * np.eye(ns) + hp["rho"] ** 2 * C_s
    L = np.linalg.cholesky(C)
    return hp["rho"] * mean_s[:, None] + L @ rng.standard_normal((ns, n_o))


def subset_batch(wl, idx):
    """The batch workload restricted to the instances idx (in that order),
    with its own union mesh and dof offsets (a rank's share of the batch)."""
    idx = [int(k) for k in idx]
    meshes = [wl["meshes"][k] for k in idx]
    union, off = mg.disjoint_union(meshes)
    bcs = [wl["bcs"][k] for k in idx]
    bc = np.concatenate([b + off[i] for i, b in enumerate(bcs)])
    coeffs = [wl["coeffs"][k] for k in idx]
    return dict(wl, sides=np.asarray(wl["sides"])[idx], meshes=meshes, coeffs=coeffs, coeff=np.concatenate(coeffs),
                bcs=bcs, sensors=[wl["sensors"][k] for k in idx], union=union, off=off, bc=bc)


def fingerprint(wl):
    """A few sums over a c1/c2 workload's generated inputs (coefficients,
    projection rows, sensor points, constraints), stored beside oracle
    fixtures so that a fixture is only compared with the inputs it was made
    from."""
    ip, ix, dv = wl["P"]
    return np.array([wl["coeff"].sum(), float(np.dot(wl["coeff"], np.arange(len(wl["coeff"])) % 97)),
                     dv.sum(), float(ix.sum()), wl["pts"].sum(), float(len(wl["bc"]))])


def pivoted_cholesky(K, rel=1e-12):
    """Greedy (largest remaining diagonal) pivoted Cholesky K ~ L L^T, stopped
    when the largest remaining diagonal drops below rel * max(diag K)."""
    n = K.shape[0]
    d = np.diag(K).astype(np.float64).copy()
    L = np.zeros((n, 0))
    stop = rel * d.max()
    while L.shape[1] < n and d.max() > stop:
        j = int(np.argmax(d))
        col = (K[:, j] - L @ L[j]) / np.sqrt(d[j])
        L = np.column_stack([L, col])
        d = np.maximum(d - col * col, 0.0)
        d[j] = 0.0
    return L


def multi_rhs_columns(wl, nrhs, sigma, length, cols=None):
    """The nrhs leading columns of the forcing covariance's factor on the c2
    grid: diag(phibar) (Lz (x) Ly (x) Lx) with L_a the pivoted Cholesky factor
    of exp(-d^2/(2 l^2)) on axis a (numerical rank to 1e-12), the Kronecker
    columns ordered by decreasing norm, one displacement component per column
    (cycling x, y, z), scaled by sigma.  Returns nrhs x num_dofs, or only the
    rows `cols` of it (len(cols) x num_dofs)."""
    mesh = wl["mesh"]
    n = mesh.grid[0] + 1
    x = np.arange(n) / (n - 1)
    L = pivoted_cholesky(np.exp(-(x[:, None] - x[None, :]) ** 2 / (2 * length * length)))
    nrm = np.linalg.norm(L, axis=0)
    r = L.shape[1]
    w = np.einsum("i,j,k->ijk", nrm, nrm, nrm).ravel()
    order = np.argsort(-w, kind="stable")
    phibar = wl["phibar"]
    cols = range(nrhs) if cols is None else [int(c) for c in cols]
    out = np.zeros((len(cols), mesh.num_dofs))
    for row, c in enumerate(cols):
        t = order[c // 3] if c // 3 < len(order) else order[-1]
        kz, ky, kx = t // (r * r), (t // r) % r, t % r
        v = sigma * np.einsum("i,j,k->ijk", L[:, kz], L[:, ky], L[:, kx]).ravel()  # z slowest, x fastest
        out[row, c % 3::3] = v
    return out * phibar[None, :]
