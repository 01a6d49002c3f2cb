"""The C++ drop-in classes (corlib::SystemSolveCuda, corlib::GpuMatrixAssembler)
in the laplaceRHSinfer flow reproduce the reference's golden posterior mean."""
import os
import subprocess

import numpy as np
import pytest

from statfem_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def compile_driver(tmp_path):
    from statfem_b200 import api
    lib = api.LIB_PATH if os.path.exists(api.LIB_PATH) else build.build()
    exe = str(tmp_path / "laplace_rhs_infer")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "laplace_rhs_infer.cpp"), "-o", exe,
                    "-L", os.path.dirname(lib), "-lstatfem_cuda", "-Wl,-rpath," + os.path.dirname(lib)],
                   check=True)
    return exe


def test_cpp_driver_compiles(tmp_path):
    assert os.path.exists(compile_driver(tmp_path))


@pytest.mark.gpu
def test_cpp_driver_kat1(tmp_path):
    exe = compile_driver(tmp_path)
    k = np.load(os.path.join(GOLDEN, "kat1_laplaceRHSinfer.npz"))
    coords, conn, Y = k["coords"], k["conn"], k["Y"]
    ns, no = Y.shape
    vals = [len(coords), len(conn), ns, no, float(k["force"]), float(k["forcing_sigma"]),
            float(k["forcing_length"]), float(k["rho"]), float(k["mismatch_sigma"]),
            float(k["mismatch_length"]), float(k["sensor_eps"]), float(k["reg"]), float(k["conductivity"])]
    path = tmp_path / "problem.txt"
    with open(path, "w") as f:
        f.write(" ".join(repr(v) for v in vals) + "\n")
        f.write(" ".join(repr(float(x)) for x in coords[:, 0]) + "\n")
        for a, b in conn:
            f.write("%d %d\n" % (a, b))
        f.write(" ".join(repr(float(v)) for v in Y.ravel()) + "\n")
        f.write(" ".join(repr(float(v)) for v in k["sensor_coords"].ravel()) + "\n")
    out = subprocess.run([exe, str(path)], check=True, capture_output=True, text=True).stdout
    mean = np.array([float(t) for t in out.split()])
    assert np.abs(mean - k["expected_mean"]).max() < 1e-6
