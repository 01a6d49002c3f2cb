"""The laplaceRHSinfer front end run on input files in the reference's formats
(written here from the committed fixture): the Woodbury posterior mean with
the watchdog's hyperparameters matches the golden vector, and the sampling
path writes its outputs."""
import os

import numpy as np
import pytest

from statfem_b200 import io as sio
from statfem_b200 import meshgen as mg
from statfem_b200.apps import laplace_rhs_infer as app

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def write_inputs(d, num_samples=20000):
    k = np.load(os.path.join(ROOT, "tests", "golden", "kat1_laplaceRHSinfer.npz"))
    sio.write_smf(os.path.join(d, "bar.smf"), mg.Mesh(mg.LINE2_POISSON, k["coords"], k["conn"]))
    with open(os.path.join(d, "input.dat"), "w") as f:
        f.write("meshFile          bar.smf\nallParamFile      allParam.dat\ninfInputFile      inferenceInput.dat\n")
    with open(os.path.join(d, "allParam.dat"), "w") as f:
        f.write("# parameters\nforcing.sigma %.17g\nforcing.length %.17g\nrho 1.\nmismatch.sigma 0.01\n"
                "mismatch.length 0.1\nmismatch.sensorEps %.17g\nconductivity %.17g\n"
                "priorMean.rho 0.8\npriorMean.mismatch.sigma 0.01\npriorMean.mismatch.length 0.1\n"
                "priorCov.rho 0.05\npriorCov.mismatch.sigma 0.05\npriorCov.mismatch.length 0.1\n"
                "init.rho 0.8\ninit.mismatch.sigma 0.03\ninit.mismatch.length 0.1\n"
                "propStDev.rho 0.01\npropStDev.mismatch.sigma 0.01\npropStDev.mismatch.length 0.005\n"
                % (float(k["forcing_sigma"]), float(k["forcing_length"]), float(k["sensor_eps"]),
                   float(k["conductivity"])))
    with open(os.path.join(d, "inferenceInput.dat"), "w") as f:
        f.write("numReadings 10\nphiMatFile ./phiMat.dat\nsensorPosFile ./sensorCoordinates.dat\n"
                "sensorValFile ./sensorValues.dat\nnumSamples %d\nenrichWithPrior 0\n"
                "hpsMeanFile ./inferredHyperParam.dat\nsampleMCMCFile ./logMLsamples.dat\n"
                "feCondDataFile ./inferredFEcondData.dat\n" % num_samples)
    P = k["P"]
    with open(os.path.join(d, "phiMat.dat"), "w") as f:
        for i, j in zip(*np.nonzero(P)):
            f.write("%d %d %.17g\n" % (i, j, P[i, j]))
    Y = k["Y"]
    with open(os.path.join(d, "sensorValues.dat"), "w") as f:
        f.write("%d %d\n" % Y.shape)
        for row in Y:
            f.write(" ".join("%.17g" % v for v in row) + " \n")
    with open(os.path.join(d, "sensorCoordinates.dat"), "w") as f:
        for x in k["sensor_coords"][:, 0]:
            f.write("%.17g\n" % x)
    return k


def test_fixed_hyperparameters_reproduce_watchdog(tmp_path):
    k = write_inputs(str(tmp_path))
    fixed = {"rho": float(k["rho"]), "mismatch.sigma": float(k["mismatch_sigma"]),
             "mismatch.length": float(k["mismatch_length"])}
    out = app.run(str(tmp_path), fixed_hp=fixed, log=lambda *a: None)
    assert np.abs(out["mean"] - k["expected_mean"]).max() < 1e-6
    written = sio.read_vector(tmp_path / "inferredFEcondData.dat")
    assert np.abs(written - k["expected_mean"]).max() < 1e-6


def test_sampling_path_writes_outputs(tmp_path):
    write_inputs(str(tmp_path), num_samples=64 * 200)
    out = app.run(str(tmp_path), chains=64, seed=1, log=lambda *a: None)
    hp = {l.split()[0]: float(l.split()[1]) for l in (tmp_path / "inferredHyperParam.dat").read_text().splitlines()}
    assert set(hp) == {"rho", "mismatch.sigma", "mismatch.length"}
    assert all(v > 0 and np.isfinite(v) for v in hp.values())
    assert abs(hp["rho"] - out["hp"]["rho"]) <= 1e-5 * hp["rho"]
    assert (tmp_path / "logMLsamples.dat").stat().st_size > 0
    assert np.all(np.isfinite(sio.read_vector(tmp_path / "inferredFEcondData.dat")))
