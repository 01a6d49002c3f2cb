"""Reference file formats (no GPU): SMF meshes, property files, parameter
maps and the app's data files; when STATFEM_REFERENCE names a checkout of the
reference tree, its laplaceRHSinfer inputs parse to the committed fixture."""
import os

import numpy as np
import pytest

from statfem_b200 import io as sio
from statfem_b200 import meshgen as mg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# a checkout of the reference tree, when one is available (skipped otherwise)
REF_TREE = os.environ.get("STATFEM_REFERENCE", "")
REF_APP = os.path.join(REF_TREE, "del2", "apps", "reference", "laplaceRHSinfer") if REF_TREE else ""


@pytest.mark.parametrize("mesh", [mg.bar(7), mg.unit_square_tri(3), mg.unit_cube_hex(2)])
def test_smf_round_trip(tmp_path, mesh):
    p = tmp_path / "m.smf"
    sio.write_smf(p, mesh)
    m = sio.read_smf(p)
    assert m.kind == mesh.kind
    np.testing.assert_array_equal(m.coords, mesh.coords)
    np.testing.assert_array_equal(m.conn, mesh.conn)


def test_smf_header_and_comments(tmp_path):
    p = tmp_path / "c.smf"
    p.write_text("# a mesh\n# of two lines\n! elementShape line\n! elementNumPoints 2\n# nodes\n3 2\n"
                 "0 0 0\n0.5 0 0\n1 0 0\n0 1\n1 2\n")
    m = sio.read_smf(p)
    assert m.num_nodes == 3 and m.num_elems == 2 and m.coords[2, 0] == 1.0
    (tmp_path / "bad.smf").write_text("3 2\n0 0 0\n")
    with pytest.raises(ValueError):
        sio.read_smf(tmp_path / "bad.smf")


def test_properties_and_param_map(tmp_path):
    p = tmp_path / "input.dat"
    p.write_text("meshFile   bar.smf\n  \n# comment\nnumReadings  10\n")
    assert sio.read_properties(p) == {"meshFile": "bar.smf", "numReadings": "10"}
    q = tmp_path / "allParam.dat"
    q.write_text("# header\nforcing.sigma   0.3\nrho 1.\n\nmismatch.length 0.1\n")
    assert sio.read_param_map(q) == {"forcing.sigma": 0.3, "rho": 1.0, "mismatch.length": 0.1}


def test_data_files(tmp_path):
    (tmp_path / "phi.dat").write_text("0 0 1.\n1 2 0.5\n1 3 0.5\n")
    P = sio.read_matrix_phi(tmp_path / "phi.dat", 5)
    np.testing.assert_array_equal(P, [[1, 0, 0, 0, 0], [0, 0, 0.5, 0.5, 0]])
    (tmp_path / "y.dat").write_text("2 3\n1 2 3 \n4 5 6\n")
    np.testing.assert_array_equal(sio.read_matrix_data(tmp_path / "y.dat"), [[1, 2, 3], [4, 5, 6]])
    (tmp_path / "x.dat").write_text("0.\n0.25\n")
    np.testing.assert_array_equal(sio.read_coord_data(tmp_path / "x.dat", 1), [[0.0], [0.25]])
    v = np.array([-3.13145e-05, 0.029965, 0.0579921, 1.0])
    sio.write_vector(tmp_path / "v.dat", v)
    lines = (tmp_path / "v.dat").read_text().split("\n")
    assert len({len(l) for l in lines}) == 1  # right-aligned to one width
    np.testing.assert_allclose(sio.read_vector(tmp_path / "v.dat"), v, rtol=1e-6)


@pytest.mark.skipif(not REF_APP or not os.path.isdir(REF_APP), reason="STATFEM_REFERENCE not set")
def test_reference_app_inputs_parse_to_fixture():
    k = np.load(os.path.join(ROOT, "tests", "golden", "kat1_laplaceRHSinfer.npz"))
    top = sio.read_properties(os.path.join(REF_APP, "input.dat"))
    mesh = sio.read_smf(os.path.join(REF_APP, top["meshFile"]))
    np.testing.assert_array_equal(mesh.coords, k["coords"])
    np.testing.assert_array_equal(mesh.conn, k["conn"])
    hp = sio.read_param_map(os.path.join(REF_APP, top["allParamFile"]))
    assert hp["forcing.sigma"] == float(k["forcing_sigma"]) and hp["conductivity"] == float(k["conductivity"])
    inf = sio.read_properties(os.path.join(REF_APP, top["infInputFile"]))
    P = sio.read_matrix_phi(os.path.join(REF_APP, inf["phiMatFile"]), mesh.num_dofs)
    np.testing.assert_array_equal(P, k["P"])
    np.testing.assert_array_equal(sio.read_matrix_data(os.path.join(REF_APP, inf["sensorValFile"])), k["Y"])
    np.testing.assert_array_equal(sio.read_coord_data(os.path.join(REF_APP, inf["sensorPosFile"]), 1),
                                  k["sensor_coords"])
