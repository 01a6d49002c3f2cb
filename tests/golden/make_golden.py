"""Regenerates the golden fixtures in this directory from the reference's own
watchdog test data (run in a checkout that has the reference tree; the
fixtures are committed so that the tests never need the reference at run
time).

  kat1_laplaceRHSinfer.npz  del2/apps/reference/laplaceRHSinfer: 1-D bar mesh
      (bar.smf), sensor readings (sensorValues.dat, 33 x 10), projection
      (phiMat.dat, identity), fixed parameters (allParam.dat), the
      hyperparameter means checked by watchDog.0.mk:19-22 and the expected
      Woodbury posterior mean watchDog.0.mk.inferredFEcondData.dat.
  kat2_gaussianProcess.npz  statX/apps/reference/gaussianProcess: training
      coordinates / hyperparameters (gpCoordinates.dat, gpHps.dat), prediction
      points, expected predictive mean/variance and log-likelihood
      (watchDog.0.mk).

Usage: python tests/golden/make_golden.py /path/to/statFEM
"""
import os
import re
import sys

import numpy as np


def _floats(path):
    with open(path) as f:
        return np.array([float(t) for t in f.read().split()])


def _params(path):
    out = {}
    with open(path) as f:
        for line in f:
            line = line.strip()
            if not line or line.startswith("#"):
                continue
            parts = line.split()
            if len(parts) >= 2:
                try:
                    out[parts[0]] = float(parts[1])
                except ValueError:
                    pass
    return out


def kat1(root, outdir):
    d = os.path.join(root, "del2/apps/reference/laplaceRHSinfer")
    with open(os.path.join(d, "bar.smf")) as f:
        lines = [l for l in f if not l.startswith("!") and not l.startswith("#")]
    nn, ne = (int(t) for t in lines[0].split())
    coords = np.array([[float(t) for t in l.split()] for l in lines[1:1 + nn]])
    conn = np.array([[int(t) for t in l.split()] for l in lines[1 + nn:1 + nn + ne]])
    sv = _floats(os.path.join(d, "sensorValues.dat"))
    ns, no = int(sv[0]), int(sv[1])
    Y = sv[2:].reshape(ns, no)
    phi = _floats(os.path.join(d, "phiMat.dat")).reshape(-1, 3)
    P = np.zeros((ns, nn))
    for r, c, v in phi:
        P[int(r), int(c)] = v
    sc = _floats(os.path.join(d, "sensorCoordinates.dat")).reshape(ns, 1)
    prm = _params(os.path.join(d, "allParam.dat"))
    with open(os.path.join(d, "watchDog.0.mk")) as f:
        wd = f.read()
    hp = {k: float(re.search(r"^%s\s*=\s*(\S+)" % k, wd, re.M).group(1))
          for k in ("RHO", "SIGMAD", "ELLD")}
    expected = _floats(os.path.join(d, "watchDog.0.mk.inferredFEcondData.dat"))
    np.savez(os.path.join(outdir, "kat1_laplaceRHSinfer.npz"), coords=coords, conn=conn, Y=Y,
             P=P, sensor_coords=sc, expected_mean=expected,
             forcing_sigma=prm["forcing.sigma"], forcing_length=prm["forcing.length"],
             sensor_eps=prm["mismatch.sensorEps"], conductivity=prm["conductivity"],
             rho=hp["RHO"], mismatch_sigma=hp["SIGMAD"], mismatch_length=hp["ELLD"],
             reg=0.001, force=np.pi * np.pi / 5.0)


def kat2(root, outdir):
    d = os.path.join(root, "statX/apps/reference/gaussianProcess")
    hps = {}
    with open(os.path.join(d, "gpHps.dat")) as f:
        toks = f.read().split()
    for k, v in zip(toks[0::2], toks[1::2]):
        hps[k] = float(v)
    xc = _floats(os.path.join(d, "gpCoordinates.dat"))
    nr, ncl = int(xc[0]), int(xc[1])
    x_train = xc[2:].reshape(ncl, nr).T  # Eigen::Map is column-major
    x_pred = _floats(os.path.join(d, "predictionCoord.dat"))
    with open(os.path.join(d, "watchDog.0.mk")) as f:
        wd = f.read()
    ll = float(re.search(r"^LIKELIHOOD\s*=\s*(\S+)", wd, re.M).group(1))
    n = x_train.shape[0]
    y = np.array([hps["gaussianProcess.w%d" % i] for i in range(n)])
    np.savez(os.path.join(outdir, "kat2_gaussianProcess.npz"), x_train=x_train, y_train=y,
             x_pred=x_pred, sigma=hps["gaussianProcess.sigma"],
             length=hps["gaussianProcess.length"], eps=hps["gaussianProcess.eps"],
             expected_mean=_floats(os.path.join(d, "watchDog.0.mk.predictionMean.dat")),
             expected_var=_floats(os.path.join(d, "watchDog.0.mk.predictionVar.dat")),
             expected_loglik=ll)


if __name__ == "__main__":
    root = sys.argv[1]
    out = os.path.dirname(os.path.abspath(__file__))
    kat1(root, out)
    kat2(root, out)
