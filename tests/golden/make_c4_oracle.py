"""Generates tests/golden/c4_oracle.npz: FP64 oracle solutions for a sample
of the multi-RHS workload's right-hand sides (the 48^3 elasticity operator of
statfem_b200.workloads.make_workload("c2", seed=1234); columns of the forcing
covariance's pivoted Cholesky factor, statfem_b200.workloads.
multi_rhs_columns, 1024 of them, sigma_f 0.05, length 0.3).

The oracle solves A u = b for 16 evenly spaced columns by FP64 Jacobi-PCG
(oracle.block_pcg, OpenMP) to the relative residual 1e-11 and, restarted from
there, to 1e-13; the change between the two is stored as the oracle's own
error estimate.  A full solution vector is 2.8 MB, so the fixture keeps
functionals of each solution that a comparison can use: its values at the
256 sensor rows (P u), its energy u^T b (= u^T A u) and its squared norm,
plus fingerprints of the inputs.

    python tests/golden/make_c4_oracle.py      # a few minutes on 8 cores
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from statfem_b200 import meshgen as mg  # noqa: E402
from statfem_b200.workloads import fingerprint, make_workload, multi_rhs_columns  # noqa: E402

NRHS = 1024
SAMPLE = 16


def functionals(U, B, Pd):
    return Pd @ U.T, np.einsum("ij,ij->i", U, B), np.einsum("ij,ij->i", U, U)


def main():
    wl = make_workload("c2", seed=1234)
    mesh, hp = wl["mesh"], wl["hp"]
    rp, col, val, F = O.fem(mesh, wl["qps"], wl["f"], wl["bc"], coeff=wl["coeff"], nu=0.3)
    wl["phibar"] = O.unit_load(mesh, wl["qps"], wl["bc"])
    pick = np.linspace(0, NRHS - 1, SAMPLE).astype(np.int64)
    B = multi_rhs_columns(wl, NRHS, hp["forcing.sigma"], hp["forcing.length"], cols=pick)
    mask = np.zeros(mesh.num_dofs, dtype=np.uint8)
    mask[wl["bc"]] = 1
    t0 = time.time()
    U11, its11 = O.block_pcg(rp, col, val, mask, B, 1e-11)
    U13, its13 = O.block_pcg(rp, col, val, mask, B, 1e-13, X0=U11)
    Pd = mg.projection_dense(mesh, *wl["P"])
    pu11, e11, n11 = functionals(U11, B, Pd)
    pu, en, nn = functionals(U13, B, Pd)
    change = max(float(np.abs(pu11 - pu).max() / np.abs(pu).max()), float(np.abs(e11 - en).max() / np.abs(en).max()))
    np.savez_compressed(os.path.join(HERE, "c4_oracle.npz"), fingerprint=fingerprint(wl), pick=pick,
                        b_sums=B.sum(axis=1), b_norms=np.linalg.norm(B, axis=1), Pu=pu, energy=en, norm2=nn,
                        its_1e11=its11, its_1e13_restart=its13, est_rel_change_1e11_to_1e13=np.float64(change))
    print("solves: %.0f s (max %d + %d iterations); relative change 1e-11 -> 1e-13: %.2e"
          % (time.time() - t0, its11.max(), its13.max(), change))


if __name__ == "__main__":
    main()
