#!/usr/bin/env python
"""statFEM posterior solves/s on B200.

Default workload (the configuration the headline metric is quoted on that
fits one GPU): 3-D linear elasticity statFEM on the unit cube, 48^3 trilinear
hex8 elements with 2x2x2 Gauss quadrature (352,947 dofs, 27,437,625
nonzeros), Young's modulus lognormal (log-GP squared-exponential sigma 0.3,
length 0.25, sampled exactly on the element-centre grid), nu = 0.3, face x=0
clamped, body force mean (0,0,-1) with a squared-exponential GP
(sigma_f 0.05, length 0.3), 256 seeded sensors (one displacement component
each, cycling x/y/z), sensor noise 1e-4; forward solve to the relative
residual 1e-8, adjoint solves to 1e-10 (which keeps the posterior covariance
within 1e-7 of the FP64 oracle).  Synthetic, seeded inputs; no dataset is
involved.

One step = one posterior solve on the GPU: assemble A and F, apply the
Dirichlet constraints, solve A u = F, the 256 adjoint solves A^T R^T = P^T
(one block solve), C_s = R C_f R^T + (sigma_f reg)^2 P P^T, the KOH
log-likelihood and the posterior mean / covariance at the sensors.

`--impl reference` times the CPU path instead (the oracle's C restatement
of the reference's assembly and a CPU FP64 Jacobi-PCG standing in for the
reference's Eigen SparseLU, which cannot run at this size), on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from statfem_b200 import meshgen as mg  # noqa: E402

from statfem_b200.workloads import C2_HP as HP  # noqa: E402
from statfem_b200.workloads import C3_HP, REG, make_batch_workload, make_workload, multi_rhs_columns  # noqa: E402
from statfem_b200.workloads import subset_batch  # noqa: E402

# the headline metric, verbatim
METRIC = "posterior solves/s at rel. residual 1e-8, learned+batched vs plain PCG, 1xB200"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
            os.unlink(self.path)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# the CUDA kernel behind the solver's "spmm32" step, by last_stats()["spmm_kernel"]
SPMM_KERNELS = {1: "k_spmm32", 2: "k_bspmm32", 3: "k_lspmm32", 4: "k_xspmm32"}


def ncu_traffic(kernel, block_width, impl=None):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, when
    it was captured at this block width on the same CUDA kernel."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            d = json.load(f)
        e = d.get(kernel)
        if e and e.get("block_width") == block_width and (impl is None or e.get("kernel", "").startswith(impl)):
            return float(e["traffic_bytes"])
    except (OSError, ValueError):
        pass
    return None


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def relaunch_if_needed(args):
    """`--gpus N` without a launcher: start N ranks (one process per GPU) with
    torch.distributed.run on this node and return its exit status; with a
    launcher, WORLD_SIZE must equal N."""
    ws = os.environ.get("WORLD_SIZE")
    if ws is None and args.gpus > 1:
        import socket
        with socket.socket() as s:
            s.bind(("127.0.0.1", 0))
            port = s.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(args.gpus),
               "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
        return subprocess.call(cmd)
    if ws is not None and int(ws) != args.gpus:
        raise SystemExit("--gpus %d but WORLD_SIZE=%s" % (args.gpus, ws))
    return None


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cuda_sync(ws):
    try:
        import torch
        if torch.cuda.is_available():
            torch.cuda.synchronize()
    except ImportError:
        pass


# ---------------------------------------------------------------------------
# our GPU arm
# ---------------------------------------------------------------------------
def precond_code(api, name):
    return {"jacobi": api.SFC_PRECOND_JACOBI, "block-jacobi": api.SFC_PRECOND_BLOCK_JACOBI,
            "two-level": api.SFC_PRECOND_TWO_LEVEL}[name]


class GpuStatFEM:
    """One statFEM posterior pipeline on the GPU.  The forward solve runs to
    the relative residual 1e-8; the adjoint (sensor) solves run to
    adjoint_tol (default 1e-10): the posterior covariance at the sensors
    amplifies their error (at c2, 1e-8 leaves it 1.3e-6 from the FP64 oracle;
    see accuracy_vs_oracle)."""

    def __init__(self, wl, device, method, block_width=128, precond=0, coarse_size=0, check_every=16,
                 adjoint_tol=1e-10):
        from statfem_b200 import api
        self.api = api
        self.wl = wl
        self.ctx = api.Context(device)
        m = wl["mesh"]
        self.gm = api.Mesh(self.ctx, m.kind, wl["qps"], m.coords, m.conn)
        self.gm.set_coefficients(wl["coeff"])
        self.s = api.SystemSolveCuda(self.ctx, m.num_dofs)
        self.block_width = block_width
        self.precond = precond
        self.coarse_size = coarse_size
        self.opts = dict(method=method, tol=1e-8, max_iter=30000, inner_tol=1e-4, block_width=block_width,
                         check_every=check_every, precond=precond, coarse_size=coarse_size)
        self.adjoint_tol = adjoint_tol
        self.s.set_options(**self.opts)
        self.cf = api.CovarianceForcing(self.ctx, self.gm)
        self.cf.applyConstraints(wl["bc"])
        self.fg = api.ForwardGaussRHS(self.s, self.cf, REG)
        self.fg.setProjectionMatrix(wl["P"])
        self.bc_vals = np.zeros(len(wl["bc"]))
        self.koh = api.LikelihoodKOH(self.fg, wl["pts"])
        # observations drawn from the prior plus noise (giveTypicalReadings),
        # generated once with this GPU pipeline
        self.prior_step()
        mean, cov = self.fg.giveProjectedMeanU(), self.fg.giveProjectedCovarU()
        hp = wl["hp"]
        ns = wl["ns"]
        C = hp["mismatch.sensorEps"] ** 2 * np.eye(ns) + hp["rho"] ** 2 * cov
        L = np.linalg.cholesky(C)
        self.Y = hp["rho"] * mean[:, None] + L @ wl["rng"].standard_normal((ns, 1))
        self.koh.setSensorValues(self.Y)

    def prior_step(self):
        wl = self.wl
        self.s.assemble(self.gm)
        self.s.clearRhs()
        self.s.assemble_load(self.gm, wl["f"])
        self.s.applyConstraints((wl["bc"], self.bc_vals))
        self.s.solveSystem()
        if self.adjoint_tol != self.opts["tol"]:
            self.s.set_options(**dict(self.opts, tol=self.adjoint_tol))
            self.fg.updateSolution(wl["hp"])
            self.s.set_options(**self.opts)
        else:
            self.fg.updateSolution(wl["hp"])

    def step(self, e2e=False):
        """One posterior solve.  e2e: the step's inputs come from host memory
        (coefficient field, sensor values) and the results go back to it."""
        if e2e:
            self.gm.set_coefficients(self.wl["coeff"])
            self.koh.setSensorValues(self.Y)
        self.prior_step()
        ll = self.koh.giveLogLikelihood(self.wl["hp"])
        pm, pc = self.koh.giveProjFEconditionedData(self.wl["hp"])
        return ll, pm, pc


def run_ours(args, ws, rank, local):
    from statfem_b200 import api
    method = api.SFC_SOLVER_PCG_MIXED if args.method == "mixed" else api.SFC_SOLVER_PCG_FP64
    wl = make_workload(args.config, seed=1234 + rank, c2_n=args.c2_n)
    g = GpuStatFEM(wl, local, method, args.block_width, precond_code(api, args.precond), args.coarse_size,
                   args.check_every, adjoint_tol=args.adjoint_tol)
    ctx = g.ctx
    for _ in range(args.warmup):
        g.step()
    g.s.solveSystem()
    stats_fwd = g.s.last_stats()
    g.fwd_iters = stats_fwd["iterations"]
    # ---- device-resident timed region ----
    barrier(ws)
    cuda_sync(ws)
    ctx.synchronize()
    l0, gl0 = ctx.kernel_launches(), ctx.graph_launches()
    with ClockSampler(local) as clk:
        ctx.mark(0)
        for _ in range(args.steps):
            ll, pm, pc = g.step()
        ctx.mark(1)
        ctx.synchronize()
    cuda_sync(ws)
    barrier(ws)
    ms = ctx.marker_ms(0, 1)
    launches = ctx.kernel_launches() - l0
    graph_launches = ctx.graph_launches() - gl0
    block_stats = g.s.last_stats()
    ms_max = max_over_ranks(ws, ms)
    # kernel timing: the same steps again with an event pair around every hot
    # kernel (kept out of the timed region above, whose value they would lower)
    ctx.set_profiling(True)
    ctx.mark(4)
    for _ in range(args.prof_steps):
        g.step()
    ctx.mark(5)
    ctx.synchronize()
    ctx.set_profiling(False)
    prof_ms = ctx.marker_ms(4, 5)
    prof_all = ctx.profile_report()
    phases = {k.split(":", 1)[1]: round(v[1] / max(args.prof_steps, 1), 3) for k, v in prof_all.items()
              if k.startswith("phase:")}
    prof = {k: v for k, v in prof_all.items() if not k.startswith("phase:")}
    value = ws * args.steps / (ms_max / 1e3)
    # ---- end-to-end through the public API with host buffers ----
    barrier(ws)
    cuda_sync(ws)
    ctx.synchronize()
    t0 = time.perf_counter()
    ctx.mark(2)
    e2e_steps = 0 if args.no_e2e else max(1, args.steps)
    for _ in range(e2e_steps):
        g.step(e2e=True)
    ctx.mark(3)
    ctx.synchronize()
    e2e_wall = time.perf_counter() - t0
    e2e_ms = max_over_ranks(ws, ctx.marker_ms(2, 3))
    ns = wl["ns"]
    h2d = wl["coeff"].nbytes + g.Y.nbytes + wl["bc"].nbytes + g.bc_vals.nbytes
    d2h = 8 * (1 + ns + ns * ns)
    # ---- roofline of the dominant kernel ----
    peak, peak_kind = peaks()
    top = max(prof.items(), key=lambda kv: kv[1][1]) if prof else None
    roof = None
    if top:
        name, (cnt, tms, tbytes) = top
        per_launch_bytes = tbytes / cnt
        per_launch_s = tms / 1e3 / cnt
        achieved = per_launch_bytes / per_launch_s / 1e9
        impl = SPMM_KERNELS.get(block_stats.get("spmm_kernel")) if name == "spmm32" else None
        roof = {"kernel": name, "cuda_kernel": impl, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4),
                "traffic": ncu_traffic(name, args.block_width, impl),
                "traffic_source": "profiles/ncu_traffic.json (ncu DRAM bytes of the same kernel on the same workload)",
                "peak_source": peak_kind,
                "bytes_per_launch": per_launch_bytes, "avg_launch_us": round(per_launch_s * 1e6, 2),
                "launches": cnt, "share_of_step": round(tms / max(prof_ms, 1e-9), 4),
                "timed_over": "%d profiled steps after the timed region" % args.prof_steps}
    out = {
        "metric": METRIC,
        "value": round(value, 4), "unit": "posterior solves/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 (FP32 inner PCG iterations, FP64 residuals)",
        "data": "synthetic (seeded)",
        "config": {"workload": wl["desc"], "block_width": args.block_width, "precond": args.precond,
                   "method": "mixed block PCG (%s preconditioner)" % args.precond if args.method == "mixed"
                   else "plain FP64 Jacobi-PCG", "parallelism": "replicas" if ws > 1 else "single GPU",
                   "learned_part": "not in this step: the learned preconditioner (FCG + message-passing "
                                   "network, --config c5) gains iterations over Jacobi but loses wall time "
                                   "to this step's two-level preconditioner",
                   "l2": "inputs larger than L2 (matrix 220+ MB)"},
        "e2e": ({"value": round(ws * e2e_steps / (e2e_ms / 1e3), 4), "unit": "posterior solves/s",
                 "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                 "wall_s": round(e2e_wall, 3)} if e2e_steps else None),
        "gpu_launches": int(launches),
        "graph_launches": int(graph_launches),
        "roofline": roof,
        "kernels": {k: {"launches": v[0], "ms": round(v[1], 3), "GBps": round(v[2] / max(v[1], 1e-9) / 1e6, 1)}
                    for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])},
        "phases_ms_per_step": phases,
        "solver": {"forward": stats_fwd, "adjoint_block": block_stats},
        "clocks": clk.summary(),
        "loglik": ll,
    }
    if rank == 0 and args.config == "c2" and args.c2_n == 48:
        out["accuracy_vs_fp64_oracle"] = accuracy_vs_oracle(g, wl)
    if not args.no_plain and args.plain_sample > 0 and args.method == "mixed":
        out["plain_fp64"] = plain_fp64_measured(g, wl)
        out["speedup_vs_plain_fp64"] = round(out["value"] / ws / out["plain_fp64"]["value"], 2)
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args, wl, g, sample_iters=args.cpu_iters)
    if rank == 0:
        print(json.dumps(out))


def run_learned(args, ws, rank, local):
    """Learned-preconditioner workload: 3-D Poisson, 128^3 hex8 elements
    (2,146,689 dofs), log-conductivity Matérn nu=3/2 (sigma 1, length 0.1).
    The network is trained on the GPU on --c5-train samples of a
    --c5-train-n^3 grid (the network is local, so it transfers across grid
    sizes), then every held-out 128^3 sample is solved to the true relative
    residual 1e-8 by flexible CG with the network and by plain FP64
    Jacobi-PCG, and (for reference) by FP64 PCG with the two-level
    preconditioner; value = held-out solves/s of the learned method."""
    from statfem_b200 import api
    from statfem_b200 import learned as L
    ctx = api.Context(local)
    if args.mpnn_apply:
        # profiling aid: only the network's application M(r) on one held-out
        # system (random parameters, no training), --mpnn-apply times
        te = L.PoissonSamples(ctx, args.c5_n, seed0=900_000)
        s = te.assemble(0, te.coefficients(0))
        net = api.LearnedPreconditioner(ctx, seed=0)
        r = np.random.default_rng(0).standard_normal(te.mesh.num_dofs)
        for _ in range(args.warmup):
            net.apply(s, r)
        ctx.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.mpnn_apply):
            z = net.apply(s, r)
        ctx.synchronize()
        ms = (time.perf_counter() - t0) * 1e3 / args.mpnn_apply
        # the device time of the same applications, kernel by kernel
        ctx.set_profiling(True)
        for _ in range(args.mpnn_apply):
            net.apply(s, r)
        ctx.synchronize()
        ctx.set_profiling(False)
        prof = ctx.profile_report()
        if rank == 0:
            print(json.dumps({"metric": "network applications (host wall, with the host copies of r and z)",
                              "ms_per_application": round(ms, 3), "n": args.c5_n, "applications": args.mpnn_apply,
                              "device_ms_per_application": {k: round(v[1] / args.mpnn_apply, 3)
                                                            for k, v in prof.items()},
                              "checksum": float(np.abs(z).sum())}))
        return
    # the network is local: train on smaller grids whose fields have the same
    # correlation length in cells as the 128^3 target (length 0.1 x 128 / n)
    tr = L.PoissonSamples(ctx, args.c5_train_n, length=0.1 * 128 / args.c5_train_n, seed0=10_000 + 1000 * rank)
    net = api.LearnedPreconditioner(ctx, seed=0)
    info = L.train(net, tr, list(range(args.c5_train)), epochs=1, steps_per_sample=args.c5_steps,
                   checkpoint=None, lr=1e-3, batch=4)
    te = L.PoissonSamples(ctx, args.c5_n, seed0=900_000 + 1000 * rank)
    coeffs = [te.coefficients(k) for k in range(args.warmup + args.steps)]
    net.attach(te.system)
    rows = []
    for k, c in enumerate(coeffs):
        s = te.assemble(k, c)
        s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-8, max_iter=50000, check_every=32)
        s.solveSystem()
        sp = s.last_stats()
        u_pcg = s.giveSolution()
        # the classical reference arm: the same FP64 PCG with the two-level
        # preconditioner (point Jacobi + one constant per box aggregate)
        s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-8, max_iter=50000, check_every=32,
                      precond=api.SFC_PRECOND_TWO_LEVEL)
        s.solveSystem()
        st2 = s.last_stats()
        d2 = float(np.abs(s.giveSolution() - u_pcg).max() / np.abs(u_pcg).max())
        s.set_options(method=api.SFC_SOLVER_FCG_MPNN, tol=1e-8, max_iter=50000, check_every=8)
        s.solveSystem()
        sf = s.last_stats()
        u = s.giveSolution()
        if k >= args.warmup:
            rows.append((sp, sf, float(np.abs(u - u_pcg).max() / np.abs(u_pcg).max()), st2, d2))
    pcg_ms = max_over_ranks(ws, sum(r[0]["device_ms"] for r in rows))
    fcg_ms = max_over_ranks(ws, sum(r[1]["device_ms"] for r in rows))
    n = len(rows)
    out = {
        "metric": "held-out solves/s at rel. residual 1e-8 (FCG + learned preconditioner), 128^3 Poisson",
        "value": round(ws * n / (fcg_ms / 1e3), 4), "unit": "solves/s", "n_gpus": ws, "steps": n,
        "warmup": args.warmup, "ms_per_step": round(fcg_ms / n, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 (network BF16 x BF16 -> FP32)",
        "data": "synthetic (seeded Matérn 3/2 log-conductivity, circulant embedding)",
        "config": {"workload": "3-D Poisson, %d^3 hex8 (%d dofs), log-conductivity Matérn nu=3/2 "
                               % (args.c5_n, (args.c5_n + 1) ** 3) + 
                               "sigma 1 length 0.1, u=0 on the boundary, f=1, rel. residual 1e-8",
                   "train": "%d samples of %d^3 (Matern length %.2f: the same length in cells), %d Adam steps "
                            "each (batch 4 pairs), 1 epoch"
                            % (args.c5_train, args.c5_train_n, 0.1 * 128 / args.c5_train_n, args.c5_steps),
                   "held_out": n, "parallelism": "replicas" if ws > 1 else "single GPU"},
        "plain_pcg": {"value": round(ws * n / (pcg_ms / 1e3), 4), "unit": "solves/s",
                      "ms_per_step": round(pcg_ms / n, 2),
                      "iterations_mean": float(np.mean([r[0]["iterations"] for r in rows]))},
        "two_level_pcg": {"value": round(ws * n / (max_over_ranks(ws, sum(r[3]["device_ms"] for r in rows)) / 1e3), 4),
                          "unit": "solves/s",
                          "iterations_mean": float(np.mean([r[3]["iterations"] for r in rows])),
                          "coarse_dofs": int(rows[0][3]["coarse_dofs"]) if rows else 0,
                          "max_rel_diff_vs_pcg": max(r[4] for r in rows) if rows else None},
        "learned": {"iterations_mean": float(np.mean([r[1]["iterations"] for r in rows])),
                    "max_rel_residual": max(r[1]["max_rel_residual"] for r in rows),
                    "max_rel_diff_vs_pcg": max(r[2] for r in rows)},
        "iteration_ratio": round(float(np.mean([r[0]["iterations"] for r in rows])) /
                                 float(np.mean([r[1]["iterations"] for r in rows])), 3),
        "time_ratio": round(pcg_ms / fcg_ms, 3),
        "training": {"seconds": round(info["seconds"], 2), "steps": int(len(info["loss"])),
                     "loss_first": round(float(info["loss"][:20].mean()), 4) if len(info["loss"]) else None,
                     "loss_last": round(float(info["loss"][-20:].mean()), 4) if len(info["loss"]) else None},
    }
    if rank == 0:
        print(json.dumps(out))


# algorithmic bytes of one FP32 block-PCG inner iteration per dof, 32 columns:
# CSR row (7 nnz x 8 B + 4 B), p gather and own row 2 x 128, q write 128,
# update (x, r, p, q read, x, r write, dinv) 6 x 128 + 4, p update (p, r read,
# p write, dinv) 3 x 128 + 4
C3_BYTES_PER_DOF_ITER = 60 + 256 + 128 + 772 + 388


def run_batch(args, ws, rank, local):
    """Config 3 on our GPU path: every step assembles all instances and runs
    the persistent batch kernel (CUDA graph)."""
    from statfem_b200 import api
    from statfem_b200 import shard
    full_wl = make_batch_workload(4321, n_inst=args.c3_instances, smin=args.c3_sides[0], smax=args.c3_sides[1])
    n_total = len(full_wl["sides"])
    # one batch split over the ranks: each takes a cost-balanced share of the
    # instances; the per-instance results are all-gathered every step
    parts = shard.partition(shard.instance_costs(full_wl["sides"]), ws)
    wl = subset_batch(full_wl, parts[rank]) if ws > 1 else full_wl
    n = len(wl["sides"])
    ctx = api.Context(local)
    t0 = time.perf_counter()
    gm = api.Mesh(ctx, mg.TRI3_POISSON, 3, wl["union"].coords, wl["union"].conn)
    b = api.BatchStatFEM(ctx, gm, wl["off"], wl["sides"], wl["bc"], wl["sensors"], 1.0, args.cluster)
    b.set_solver(tol=args.c3_tol, inner_tol=args.inner_tol)
    b.set_coefficients(wl["coeff"])
    b.set_hparams(C3_HP, REG)
    # observations drawn from each instance's prior plus noise
    b.set_readings(np.zeros((n, 32, 1)))
    b.run()
    r = b.results()
    Y = np.zeros((n, 32, 1))
    m = wl["ns"]
    for k in range(n):
        pts = wl["sensors"][k][1]
        D = pts[:, None, :] - pts[None, :, :]
        Ks = C3_HP["mismatch.sigma"] ** 2 * np.exp(-np.sum(D * D, axis=2) / (2 * C3_HP["mismatch.length"] ** 2)) \
            + C3_HP["mismatch.sensorEps"] ** 2 * np.eye(m)
        C = Ks + C3_HP["rho"] ** 2 * r["cov_s"][k, :m, :m]
        Y[k, :m, 0] = C3_HP["rho"] * r["mean_s"][k, :m] + np.linalg.cholesky(C) @ wl["rng"].standard_normal(m)
    b.set_readings(Y)
    setup_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        b.run()
    ctx.synchronize()
    barrier(ws)
    cuda_sync(ws)
    l0 = ctx.kernel_launches()

    def gathered():
        r = b.results()
        if ws == 1:
            return r
        return shard.gather({k: r[k] for k in ("loglik", "post_mean", "post_cov", "status")}, parts, n_total)

    with ClockSampler(local) as clk:
        ctx.mark(0)
        for _ in range(args.steps):
            b.run()
            if ws > 1:
                gathered()
        ctx.mark(1)
        ctx.synchronize()
    cuda_sync(ws)
    barrier(ws)
    ms = max_over_ranks(ws, ctx.marker_ms(0, 1))
    launches = ctx.kernel_launches() - l0
    res = b.results()
    status_all = gathered()["status"]
    # phase split and the persistent kernel's own time (one profiled step)
    ctx.set_profiling(True)
    b.run()
    ctx.synchronize()
    ctx.set_profiling(False)
    prof = ctx.profile_report()
    kern_ms = prof.get("phase:batch_solve_likelihood", (1, float("nan"), 0))[1]
    asm_ms = prof.get("phase:batch_assembly", (1, float("nan"), 0))[1]
    dofs = np.diff(wl["off"])
    alg_bytes = float(np.sum(res["iterations"].astype(np.float64) * dofs) * C3_BYTES_PER_DOF_ITER)
    peak, peak_kind = peaks()
    achieved = alg_bytes / (kern_ms / 1e3) / 1e9
    # end to end: coefficients and readings from host memory, results back
    ctx.synchronize()
    ctx.mark(2)
    for _ in range(args.steps):
        b.set_coefficients(wl["coeff"])
        b.set_readings(Y)
        b.run()
        b.results()
    ctx.mark(3)
    ctx.synchronize()
    e2e_ms = max_over_ranks(ws, ctx.marker_ms(2, 3))
    h2d = wl["coeff"].nbytes + Y.nbytes
    d2h = 8 * n * (1 + 32 + 32 * 32 + 32 + 32 * 32) + 8 * n
    value = n_total * args.steps / (ms / 1e3)
    cs, grid = b.launch_shape()
    out = {
        "metric": "posterior solves/s at rel. residual 1e-8 (batched instances, 1xB200)",
        "value": round(value, 3), "unit": "posterior solves/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 2), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": "f64 (FP32 inner PCG iterations, FP64 residuals, covariance and Cholesky)",
        "data": "synthetic (seeded)",
        "config": {"workload": full_wl["desc"], "rel_residual": args.c3_tol, "cluster_size": cs, "grid_ctas": grid,
                   "parallelism": ("instances split over %d ranks (cost-balanced), results all-gathered every step"
                                   % ws) if ws > 1 else "single GPU",
                   "l2": "inputs larger than L2 (solver vectors 17 GB)"},
        "e2e": {"value": round(n_total * args.steps / (e2e_ms / 1e3), 3), "unit": "posterior solves/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "roofline": {"kernel": "k_batch (persistent)", "bound": "hbm", "achieved": round(achieved, 1),
                     "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None,
                     "peak_source": peak_kind, "bytes_per_launch": alg_bytes,
                     "avg_launch_us": round(kern_ms * 1e3, 1),
                     "algorithmic_bytes": "%d B per dof per inner iteration x sum(iterations x dofs)"
                                          % C3_BYTES_PER_DOF_ITER},
        "phases_ms_per_step": {"assembly": round(asm_ms, 2), "solve_likelihood_kernel": round(kern_ms, 2)},
        "iterations": {"mean": float(res["iterations"].mean()), "max": int(res["iterations"].max())},
        "status_ok": int((status_all == 0).sum()),
        "setup_s": round(setup_s, 1),
        "clocks": clk.summary(),
    }
    if args.plain_sample > 0:
        out["plain_fp64"] = batch_plain_estimate(ctx, wl, args.plain_sample)
        out["speedup_vs_plain_fp64"] = round(out["value"] / ws / out["plain_fp64"]["value"], 2)
    if rank == 0:
        print(json.dumps(out))
    b.close()


def batch_plain_estimate(ctx, wl, sample):
    """Posterior solves/s of the plain method on the same GPU for config 3:
    each instance through the single-system path (SystemSolveCuda with FP64
    Jacobi-PCG, one right-hand side at a time; ForwardGaussRHS;
    LikelihoodKOH), timed on `sample` instances spread over the sizes and
    interpolated in the side length to all instances."""
    from statfem_b200 import api
    sides = wl["sides"]
    order = np.argsort(sides)
    pick = order[np.linspace(0, len(order) - 1, sample).astype(int)]
    times = []
    for k in pick:
        mesh = wl["meshes"][k]
        gm = api.Mesh(ctx, mg.TRI3_POISSON, 3, mesh.coords, mesh.conn)
        gm.set_coefficients(wl["coeffs"][k])
        s = api.SystemSolveCuda(ctx, mesh.num_dofs)
        s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-8, max_iter=100000, check_every=32)
        cf = api.CovarianceForcing(ctx, gm)
        cf.applyConstraints(wl["bcs"][k])
        fg = api.ForwardGaussRHS(s, cf, REG)
        fg.setProjectionMatrix(wl["sensors"][k][0])
        koh = api.LikelihoodKOH(fg, wl["sensors"][k][1])
        koh.setSensorValues(np.zeros((wl["ns"], 1)))
        zero = np.zeros(len(wl["bcs"][k]))

        def one():
            s.assemble(gm)
            s.clearRhs()
            s.assemble_load(gm, np.array([1.0]))
            s.applyConstraints((wl["bcs"][k], zero))
            fg.updateSolution(C3_HP)
            koh.giveLogLikelihood(C3_HP)
            koh.giveProjFEconditionedData(C3_HP)

        one()
        ctx.synchronize()
        ctx.mark(6)
        one()
        ctx.mark(7)
        ctx.synchronize()
        times.append(ctx.marker_ms(6, 7))
        for o in (koh, fg, cf, s, gm):
            o.close()
    xs = sides[pick].astype(float)
    est = float(np.sum(np.interp(sides.astype(float), xs, np.array(times))))
    return {"value": round(len(sides) / (est / 1e3), 4), "unit": "posterior solves/s",
            "ms_per_step": round(est, 1),
            "sample": "%d instances (sides %s) through the single-system path with FP64 Jacobi-PCG, one RHS at a "
                      "time: %s ms; interpolated in the side length over all %d instances"
                      % (sample, ",".join(str(int(v)) for v in xs), ",".join("%.1f" % t for t in times),
                         len(sides))}


def c4_accuracy(wl, B, U):
    """Per-column errors of the multi-RHS solutions against the committed
    FP64 oracle fixture (tests/golden/c4_oracle.npz: 16 columns solved by the
    oracle's Jacobi-PCG to 1e-13; made by tests/golden/make_c4_oracle.py),
    through the functionals the fixture keeps: the values at the 256 sensor
    rows and the energy u^T b.  Only the fixture's arrays are read here."""
    from statfem_b200.workloads import fingerprint
    path = os.path.join(ROOT, "tests", "golden", "c4_oracle.npz")
    if not os.path.exists(path):
        return None
    f = np.load(path)
    pick = f["pick"]
    if (not np.allclose(f["fingerprint"], fingerprint(wl), rtol=1e-12, atol=0)
            or not np.allclose(f["b_sums"], B[pick].sum(axis=1), rtol=1e-12, atol=1e-300)):
        return None
    Pd = mg.projection_dense(wl["mesh"], *wl["P"])
    pu = Pd @ U[pick].T
    en = np.einsum("ij,ij->i", U[pick], B[pick])
    sens = np.abs(pu - f["Pu"]).max(axis=0) / np.abs(f["Pu"]).max(axis=0)
    ener = np.abs(en - f["energy"]) / np.abs(f["energy"])
    return {"columns": int(len(pick)), "sensor_values_max_rel": float(sens.max()),
            "energy_max_rel": float(ener.max()),
            "oracle": "FP64 Jacobi-PCG to rel. residual 1e-13 on 16 evenly spaced columns; oracle's own change "
                      "from 1e-11 to 1e-13: %.1e" % float(f["est_rel_change_1e11_to_1e13"])}


def run_multi(args, ws, rank, local):
    """Config 4: 1024 right-hand sides (forcing-covariance factor columns) on
    the c2 elasticity mesh, mixed block PCG to the true relative residual
    1e-10, inputs resident on the device."""
    import torch
    from statfem_b200 import api
    wl = make_workload("c2", seed=1234 + rank)
    nrhs = args.c4_rhs
    g = GpuStatFEM(wl, local, api.SFC_SOLVER_PCG_MIXED, args.block_width,
                   precond_code(api, args.precond), args.coarse_size)
    ctx, s = g.ctx, g.s
    wl["phibar"] = g.cf.phibar()
    B = multi_rhs_columns(wl, nrhs, HP["forcing.sigma"], HP["forcing.length"])
    N = B.shape[1]
    s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-10, max_iter=30000, inner_tol=1e-4,
                  block_width=args.block_width, check_every=32, precond=g.precond, coarse_size=g.coarse_size)
    dev = torch.device("cuda", local)
    Bd = torch.from_numpy(np.ascontiguousarray(B.T)).to(dev)  # interleaved [N][nrhs]
    Ud = torch.empty_like(Bd)
    torch.cuda.synchronize(dev)
    for _ in range(args.warmup):
        s.solve_multi_device(Bd.data_ptr(), Ud.data_ptr(), nrhs)
    ctx.synchronize()
    barrier(ws)
    l0 = ctx.kernel_launches()
    with ClockSampler(local) as clk:
        ctx.mark(0)
        for _ in range(args.steps):
            s.solve_multi_device(Bd.data_ptr(), Ud.data_ptr(), nrhs)
        ctx.mark(1)
        ctx.synchronize()
    barrier(ws)
    ms = max_over_ranks(ws, ctx.marker_ms(0, 1))
    launches = ctx.kernel_launches() - l0
    st = s.last_stats()
    U = Ud.cpu().numpy().T
    accuracy = c4_accuracy(wl, B, U) if rank == 0 and nrhs == 1024 else None
    pick = np.linspace(0, nrhs - 1, args.c4_check).astype(int)
    # plain FP64 PCG at 1e-10, one column at a time, on a sample of columns
    s.set_options(method=api.SFC_SOLVER_PCG_FP64, tol=1e-10, max_iter=200000, check_every=32)
    s.solveSystemMulti(B[pick])
    plain = s.last_stats()
    # end to end through the host API
    s.set_options(method=api.SFC_SOLVER_PCG_MIXED, tol=1e-10, max_iter=30000, inner_tol=1e-4,
                  block_width=args.block_width, check_every=32, precond=g.precond, coarse_size=g.coarse_size)
    ctx.synchronize()
    ctx.mark(2)
    s.solveSystemMulti(B)
    ctx.mark(3)
    ctx.synchronize()
    e2e_ms = ctx.marker_ms(2, 3)
    value = ws * nrhs * args.steps / (ms / 1e3)
    out = {
        "metric": "right-hand-side solves/s at rel. residual 1e-10 (multi-RHS prior covariance, 1xB200)",
        "value": round(value, 2), "unit": "RHS solves/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (FP32 inner PCG iterations, FP64 residuals)", "data": "synthetic (seeded)",
        "config": {"workload": "c2 mesh (48^3 hex8 elasticity, 352,947 dofs), %d right-hand sides = leading "
                               "columns of the forcing covariance's pivoted Cholesky factor, rel. residual 1e-10"
                               % nrhs,
                   "block_width": args.block_width, "precond": args.precond,
                   "parallelism": "replicas" if ws > 1 else "single GPU"},
        "e2e": {"value": round(nrhs / (e2e_ms / 1e3), 2), "unit": "RHS solves/s",
                "h2d_bytes_per_step": int(B.nbytes), "d2h_bytes_per_step": int(B.nbytes)},
        "gpu_launches": int(launches),
        "solver": st,
        "accuracy_vs_fp64_oracle": accuracy,
        "plain_fp64": {"value": round(len(pick) / (plain["device_ms"] / 1e3), 3), "unit": "RHS solves/s",
                       "sample": "%d columns, FP64 Jacobi-PCG one at a time to 1e-10, max %d iterations"
                                 % (len(pick), plain["iterations"])},
        "clocks": clk.summary(),
    }
    out["speedup_vs_plain_fp64"] = round(out["value"] / ws / out["plain_fp64"]["value"], 2)
    if rank == 0:
        print(json.dumps(out))


def accuracy_vs_oracle(g, wl):
    """Relative errors of one posterior step against the committed FP64
    oracle fixture of the 48^3 elasticity workload (tests/golden/
    c2_oracle.npz: the oracle's Jacobi-PCG to 1e-13 with its own readings;
    made by tests/golden/make_c2_oracle.py).  Only the fixture's arrays are
    read here; the oracle itself does not run.  None when the fixture is
    absent or was made from other inputs."""
    from statfem_b200.workloads import fingerprint
    path = os.path.join(ROOT, "tests", "golden", "c2_oracle.npz")
    if not os.path.exists(path):
        return None
    f = np.load(path)
    if not np.allclose(f["fingerprint"], fingerprint(wl), rtol=1e-12, atol=0):
        return None
    ns = wl["ns"]
    iu = np.triu_indices(ns)

    def sym(u):
        M = np.zeros((ns, ns))
        M[iu] = u
        return M + np.triu(M, 1).T

    def rel(a, b):
        return float(np.abs(a - b).max() / np.abs(b).max())

    g.koh.setSensorValues(f["Y"])
    ll, pm, pc = g.step()
    out = {"prior_mean": rel(g.fg.giveProjectedMeanU(), f["mean_s"]),
           "prior_cov": rel(g.fg.giveProjectedCovarU(), sym(f["C_s_upper"])),
           "posterior_mean": rel(pm, f["post_mean"]), "posterior_cov": rel(pc, sym(f["post_cov_upper"])),
           "loglik": abs(ll - float(f["loglik"])) / abs(float(f["loglik"])),
           "oracle": "FP64 Jacobi-PCG to rel. residual 1e-13 (forward + 256 adjoint solves), Kronecker C_f, "
                     "numpy LikelihoodKOH; oracle's own change from 1e-11 to 1e-13: %.1e"
                     % float(f["est_rel_change_1e11_to_1e13"].max())}
    out["max"] = max(out[k] for k in ("prior_mean", "prior_cov", "posterior_mean", "posterior_cov"))
    g.koh.setSensorValues(g.Y)
    return out


def plain_fp64_measured(g, wl):
    """Posterior solves/s of the plain method on the same GPU, measured on one
    whole step: FP64 Jacobi-PCG for the forward solve and for each of the ns
    adjoint solves (one right-hand side at a time), then the same covariance,
    likelihood and posterior as the timed step."""
    from statfem_b200 import api
    keep = g.opts
    g.opts = dict(method=api.SFC_SOLVER_PCG_FP64, tol=1e-8, max_iter=30000, check_every=32,
                  precond=api.SFC_PRECOND_JACOBI)
    g.s.set_options(**g.opts)
    g.ctx.synchronize()
    g.ctx.mark(6)
    g.step()
    g.ctx.mark(7)
    g.ctx.synchronize()
    ms = g.ctx.marker_ms(6, 7)
    st = g.s.last_stats()
    g.opts = keep
    g.s.set_options(**keep)
    return {"value": round(1e3 / ms, 5), "unit": "posterior solves/s", "ms_per_step": round(ms, 1),
            "sample": "measured: one whole posterior step with FP64 Jacobi-PCG (forward solve to 1e-8 and %d "
                      "adjoint solves to %.0e, one right-hand side at a time, max %d iterations per solve)"
                      % (wl["ns"], g.adjoint_tol, st["iterations"])}


# ---------------------------------------------------------------------------
# CPU arms (oracle port)
# ---------------------------------------------------------------------------
CPU_BLOCK = 32  # right-hand sides per CPU block-PCG pass


def cpu_setup(wl, rp, col, val, F, adjoint_tol=1e-8):
    """One-off CPU measurements for the posterior-solve model of the CPU path
    (oracle C restatement, FP64 Jacobi-PCG on all host cores):
    * assembly: the oracle's element loop + triplet merge on the mesh with
      half the elements per side, scaled by the element count;
    * forward solve: A u = F solved in full to the relative residual 1e-8;
    * covariance: C_s = R C_f R^T through the forcing covariance's Kronecker
      factors (numpy), in full, on ns unit-norm rows standing in for R."""
    from oracle import oracle as O
    mesh = wl["mesh"]
    N = mesh.num_dofs
    mask = np.zeros(N, dtype=np.uint8)
    mask[wl["bc"]] = 1
    n = mesh.grid[0]
    half = max(2, n // 2)
    sub = (mg.unit_cube_hex(half, mesh.kind) if mesh.dim == 3 else mg.unit_square_tri(half))
    sub_coeff = np.ones(sub.num_elems)
    t0 = time.perf_counter()
    O.fem(sub, wl["qps"], wl["f"], mg.dirichlet_dofs(sub, "x0" if mesh.dof == 3 else "all"), coeff=sub_coeff, nu=0.3)
    t_asm = (time.perf_counter() - t0) * mesh.num_elems / sub.num_elems
    t0 = time.perf_counter()
    x, its = O.pcg(rp, col, val, mask, F, tol=1e-8, max_iter=60000)
    t_fwd = time.perf_counter() - t0
    # iterations the adjoint solves need at their tolerance (the same
    # operator; measured on the forward right-hand side)
    adj_its = its if adjoint_tol >= 1e-8 else O.pcg(rp, col, val, mask, F, tol=adjoint_tol, max_iter=60000)[1]
    phibar = O.unit_load(mesh, wl["qps"], wl["bc"])
    Pd = mg.projection_dense(mesh, *wl["P"])
    hp = wl["hp"]
    t0 = time.perf_counter()
    O.forward_gauss_rhs_grid(Pd, F, Pd, mesh, phibar, hp["forcing.sigma"], hp["forcing.length"], REG)
    t_cov = time.perf_counter() - t0
    return dict(mask=mask, Pd=Pd, t_asm=t_asm, t_fwd=t_fwd, fwd_its=int(its), adj_its=int(adj_its),
                adj_tol=adjoint_tol, t_cov=t_cov, half=half)


def cpu_adjoint_sample(rp, col, val, setup, sample_iters):
    """Seconds per block-PCG iteration over CPU_BLOCK adjoint right-hand sides
    (the first CPU_BLOCK sensor rows), timed over sample_iters iterations."""
    from oracle import oracle as O
    B = setup["Pd"][:CPU_BLOCK]
    t0 = time.perf_counter()
    O.block_pcg(rp, col, val, setup["mask"], B, 1e-300, max_iter=sample_iters)
    return (time.perf_counter() - t0) / sample_iters


def cpu_posterior_seconds(wl, setup, per_block_iter):
    """assembly + forward solve + ceil(ns / CPU_BLOCK) adjoint blocks of the
    iteration count at the adjoint tolerance + covariance."""
    blocks = -(-wl["ns"] // CPU_BLOCK)
    return setup["t_asm"] + setup["t_fwd"] + blocks * setup["adj_its"] * per_block_iter + setup["t_cov"]


def cpu_sample_text(wl, setup, per_block_iter, sample_iters, threads):
    return ("oracle C restatement, FP64 Jacobi-PCG, OpenMP on %d host threads: forward solve to 1e-8 measured "
            "in full (%d iterations, %.1f s); adjoint solves to %.0e as %d blocks of %d right-hand sides at "
            "%.1f ms per block iteration (%d iterations timed) x %d iterations; C_s through the Kronecker factors "
            "measured in full (%.1f s); assembly measured on the %d^%d mesh and scaled by elements (%.1f s)"
            % (threads, setup["fwd_its"], setup["t_fwd"], setup["adj_tol"], -(-wl["ns"] // CPU_BLOCK), CPU_BLOCK,
               per_block_iter * 1e3, sample_iters, setup["adj_its"], setup["t_cov"], setup["half"],
               wl["mesh"].dim, setup["t_asm"]))


def host_threads():
    try:
        return int(os.environ.get("OMP_NUM_THREADS") or len(os.sched_getaffinity(0)))
    except (AttributeError, ValueError):
        return os.cpu_count() or 1


def cpu_baseline(args, wl, g, sample_iters):
    rp, col, val = g.s.get_csr()
    rp = rp.astype(np.int64)
    F = g.s.giveForce()
    setup = cpu_setup(wl, rp, col, val, F, g.adjoint_tol)
    per = cpu_adjoint_sample(rp, col, val, setup, sample_iters)
    sec = cpu_posterior_seconds(wl, setup, per)
    threads = host_threads()
    return {"value": round(1.0 / sec, 6), "unit": "posterior solves/s", "cores": threads, "kind": "port",
            "sample": cpu_sample_text(wl, setup, per, sample_iters, threads)}


def run_reference_c5(args):
    """CPU arm of the learned-preconditioner workload: the oracle's C
    assembly and FP64 Jacobi-PCG (1 core) on one held-out 128^3 sample,
    solved in full to the relative residual 1e-8."""
    from oracle import oracle as O
    mesh = mg.unit_cube_hex(128, mg.HEX8_POISSON)
    rng = np.random.default_rng(900_000)
    coeff = np.exp(mg.matern32_field_cells(rng, 128, 1.0, 0.1))
    bc = mg.dirichlet_dofs(mesh, "all")
    rp, col, val, F = O.fem(mesh, 8, np.array([1.0]), bc, coeff=coeff)
    mask = np.zeros(mesh.num_dofs, dtype=np.uint8)
    mask[bc] = 1
    t0 = time.perf_counter()
    x, its = O.pcg(rp, col, val, mask, F, tol=1e-8, max_iter=100000)
    dt = time.perf_counter() - t0
    value = 1.0 / dt
    out = {"impl": "reference", "metric": "held-out solves/s at rel. residual 1e-8 (FCG + learned "
           "preconditioner), 128^3 Poisson", "value": round(value, 6), "unit": "solves/s", "n_gpus": 0,
           "steps": 1, "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic (seeded Matérn 3/2 log-conductivity)",
           "config": {"workload": "3-D Poisson, 128^3 hex8 (2,146,689 dofs), rel. residual 1e-8",
                      "method": "CPU FP64 Jacobi-PCG (oracle port)"},
           "cpu_baseline": {"value": round(value, 6), "unit": "solves/s", "cores": 1, "kind": "port",
                            "sample": "one held-out sample solved in full: %d iterations, %.1f s" % (its, dt)},
           "e2e": {"value": round(value, 6), "unit": "solves/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def run_reference(args, ws, rank):
    """The CPU path on the host cores (rank 0 only): the oracle's C
    restatement of the reference's assembly and FP64 Jacobi-PCG standing in
    for the reference's Eigen SparseLU (which cannot factor this system in
    any reasonable time), OpenMP on every host thread.  One-off: assembly of
    the full matrix (not timed: it only provides the operator), a full
    forward solve, the covariance and a scaled assembly sample; each step
    then times cpu_iters block-PCG iterations over 32 adjoint right-hand
    sides, and the step's rate is the posterior-solve model built from them."""
    if rank != 0:
        return
    if args.config == "c5":
        return run_reference_c5(args)
    from oracle import oracle as O
    wl = make_workload(args.config, seed=1234)
    mesh = wl["mesh"]
    rp, col, val, F = O.fem(mesh, wl["qps"], wl["f"], wl["bc"], coeff=wl["coeff"], nu=0.3)
    setup = cpu_setup(wl, rp, col, val, F, args.adjoint_tol)
    rates, pers = [], []
    for k in range(args.warmup + args.steps):
        per = cpu_adjoint_sample(rp, col, val, setup, args.cpu_iters)
        if k >= args.warmup:
            pers.append(per)
            rates.append(1.0 / cpu_posterior_seconds(wl, setup, per))
    value = float(np.mean(rates))
    threads = host_threads()
    out = {"impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "posterior solves/s",
           "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
           "config": {"workload": wl["desc"], "method": "CPU FP64 Jacobi-PCG (oracle port, OpenMP)"},
           "cpu_baseline": {"value": round(value, 6), "unit": "posterior solves/s", "cores": threads,
                            "kind": "port",
                            "sample": "per step: " + cpu_sample_text(wl, setup, float(np.mean(pers)), args.cpu_iters,
                                                                     threads)},
           "e2e": {"value": round(value, 6), "unit": "posterior solves/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--c2-n", type=int, default=48,
                    help="c2: elements per side (48 is the benchmark; smaller for profiler captures)")
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=["c2", "c1", "c3", "c4", "c5"])
    ap.add_argument("--c4-rhs", type=int, default=1024, help="c4: right-hand sides")
    ap.add_argument("--c4-check", type=int, default=8, help="c4: columns checked against FP64 PCG at 1e-13")
    ap.add_argument("--c3-instances", type=int, default=512, help="c3: number of instances")
    ap.add_argument("--c3-sides", type=int, nargs=2, default=[32, 256], help="c3: range of the grid sides")
    ap.add_argument("--inner-tol", type=float, default=1e-2, help="c3: FP32 reduction between FP64 residuals")
    ap.add_argument("--c3-tol", type=float, default=1e-9,
                    help="c3: relative residual of every instance's solves (1e-9 keeps the prior mean and the "
                         "log-likelihood within 1e-7 of the oracle; at 1e-8 the worst instance is at 1.1e-7)")
    ap.add_argument("--cluster", type=int, default=0, help="c3: CTAs per instance (0: default)")
    ap.add_argument("--c5-train", type=int, default=48, help="c5: training samples")
    ap.add_argument("--c5-train-n", type=int, default=32, help="c5: training grid (elements per side)")
    ap.add_argument("--c5-steps", type=int, default=40, help="c5: Adam steps per training sample")
    ap.add_argument("--c5-n", type=int, default=128, help="c5: held-out grid (elements per side)")
    ap.add_argument("--mpnn-apply", type=int, default=0,
                    help="c5 profiling aid: time this many network applications on one held-out system and exit")
    ap.add_argument("--method", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--cpu-iters", type=int, default=20,
                    help="CPU arms: block-PCG iterations timed per sample")
    ap.add_argument("--no-plain", action="store_true",
                    help="c2/c1: skip the whole-step plain FP64 Jacobi-PCG measurement")
    ap.add_argument("--plain-sample", type=int, default=8, help="c3: instances timed through the plain path (0: no plain-method measurement, any config)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--prof-steps", type=int, default=1)
    ap.add_argument("--block-width", type=int, default=128, choices=[32, 64, 128])
    ap.add_argument("--precond", default="two-level", choices=["jacobi", "block-jacobi", "two-level"])
    ap.add_argument("--check-every", type=int, default=16,
                    help="iterations between the solver's convergence checks (c1/c2)")
    ap.add_argument("--coarse-size", type=int, default=0,
                    help="two-level: nodes per aggregate along each axis (0: library default)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--adjoint-tol", type=float, default=1e-10,
                    help="c1/c2: relative residual of the adjoint (sensor) solves; the forward solve stays at 1e-8 "
                         "(1e-10 keeps the posterior covariance within 1e-7 of the FP64 oracle)")
    args = ap.parse_args()
    rc = relaunch_if_needed(args)
    if rc is not None:
        sys.exit(rc)
    ws, rank, local = dist_setup() if args.impl == "ours" else (int(os.environ.get("WORLD_SIZE", "1")),
                                                                int(os.environ.get("RANK", "0")), 0)
    if args.impl == "reference":
        run_reference(args, ws, rank)
    elif args.config == "c5":
        run_learned(args, ws, rank, local)
    elif args.config == "c3":
        run_batch(args, ws, rank, local)
    elif args.config == "c4":
        run_multi(args, ws, rank, local)
    else:
        run_ours(args, ws, rank, local)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
