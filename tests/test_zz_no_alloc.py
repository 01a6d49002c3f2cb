"""sfc_koh_log_likelihood_noalloc: the log-likelihood for callers that cannot
allocate device memory while they run (an MCMC loop on a stream it owns,
where cudaMalloc / cudaFree would synchronise the device, or an application
with a fixed memory budget).  It takes caller-owned device buffers and keeps
its scratch in a fixed device array; its result must equal the regular entry
point's, on consecutive calls that share that array.

The file name makes pytest collect it last, so a failure here cannot hide the
results of the other tests."""
import ctypes

import numpy as np
import pytest

from statfem_b200 import api
from statfem_b200 import meshgen as mg
from tests.problems import QPS, statfem_problem

pytestmark = pytest.mark.gpu

HP1 = {"forcing.sigma": 0.1, "forcing.length": 0.2, "rho": 1.0, "mismatch.sigma": 0.02, "mismatch.length": 0.3,
       "mismatch.sensorEps": 1e-3}
HP2 = dict(HP1, **{"rho": 0.8, "mismatch.sigma": 0.05, "mismatch.length": 0.15, "mismatch.sensorEps": 2e-3})


def test_noalloc_loglik_matches_regular_entry_point():
    import torch

    ctx = api.Context(0)
    prob = statfem_problem(mg.TRI3_POISSON, 12, 20, seed=5)
    mesh = prob["mesh"]
    gm = api.Mesh(ctx, mesh.kind, QPS[mesh.kind], mesh.coords, mesh.conn)
    gm.set_coefficients(prob["coeff"])
    s = api.SystemSolveCuda(ctx, mesh.num_dofs)
    s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-10)
    s.assemble(gm)
    s.assemble_load(gm, 1.0)
    s.applyConstraints((prob["bc"], np.zeros(len(prob["bc"]))))
    cf = api.CovarianceForcing(ctx, gm)
    cf.applyConstraints(prob["bc"])
    fg = api.ForwardGaussRHS(s, cf, 0.001)
    fg.setProjectionMatrix(prob["P"])
    fg.updateSolution(HP1)
    ns, n_o = 20, 3
    rng = np.random.default_rng(11)
    mean, cov = fg.giveProjectedMeanU(), fg.giveProjectedCovarU()
    Y = mean[:, None] + 1e-3 * rng.standard_normal((ns, n_o))
    koh = api.LikelihoodKOH(fg, prob["pts"])
    koh.setSensorValues(Y)
    refs = [koh.giveLogLikelihood(HP1), koh.giveLogLikelihood(HP2)]

    dev = torch.device("cuda", 0)
    xs = np.zeros((ns, 3))
    xs[:, :2] = prob["pts"]
    t_mean = torch.tensor(mean, dtype=torch.float64, device=dev)
    t_cov = torch.tensor(cov, dtype=torch.float64, device=dev)
    t_xs = torch.tensor(xs, dtype=torch.float64, device=dev)
    t_y = torch.tensor(Y, dtype=torch.float64, device=dev)
    t_out = torch.zeros(1, dtype=torch.float64, device=dev)
    t_info = torch.full((1,), 7, dtype=torch.int32, device=dev)
    lib = api.load()
    for hp, ref in zip((HP1, HP2), refs):  # two calls in a row share the scratch array
        h = api.HParams.from_map(hp)
        rc = lib.sfc_koh_log_likelihood_noalloc(t_mean.data_ptr(), t_cov.data_ptr(), t_xs.data_ptr(), 2,
                                                t_y.data_ptr(), ns, n_o, ctypes.byref(h), t_out.data_ptr(),
                                                t_info.data_ptr(), None)
        assert rc == 0
        torch.cuda.synchronize()
        assert int(t_info.item()) == 0
        assert abs(float(t_out.item()) - ref) <= 1e-10 * max(1.0, abs(ref))

    # sizes beyond the fixed scratch are rejected before any launch
    h = api.HParams.from_map(HP1)
    rc = lib.sfc_koh_log_likelihood_noalloc(t_mean.data_ptr(), t_cov.data_ptr(), t_xs.data_ptr(), 2,
                                            t_y.data_ptr(), 129, n_o, ctypes.byref(h), t_out.data_ptr(),
                                            t_info.data_ptr(), None)
    assert rc == -8
    for obj in (koh, fg, cf, s, gm):
        obj.close()
    ctx.close()
