"""Readers and writers for the reference's file formats, so that statFEM
inputs run unchanged.

* SMF meshes: corlib::Mesh::read (corlib/Mesh.ipp:63-102) with the header of
  corlib::SmfHead (corlib/SmfHead.hpp): '#' comment lines, '!' header lines
  ("! elementShape line|triangle|quadrilateral|tetrahedron|hexahedron",
  "! elementNumPoints n"), then "numNodes numElements", one node per line
  (three coordinates) and one element per line (0-based node ids).
* Property files (input.dat, inferenceInput.dat): "name value" lines with
  '#' comments (corlib::PropertiesParser, corlib/PropertiesParser.hpp).
* Parameter maps (allParam.dat): apps::readParamToMap (laplaceRHSinfer/
  ioHelpers.hpp): "key value" pairs, lines starting with '#' skipped.
* Matrices: readMatrixPhi (triplets "row col value", size from the largest
  row index), readMatrixData ("rows cols" then the values row by row),
  readCoordData (one point per line), readVecData (whitespace-separated).
"""
from __future__ import annotations

import numpy as np

from . import meshgen as mg

_SHAPE_KIND = {("line", 2): mg.LINE2_POISSON, ("triangle", 3): mg.TRI3_POISSON,
               ("hexahedron", 8): mg.HEX8_POISSON}


def _tokens_without_comments(lines):
    for line in lines:
        s = line.strip()
        if not s or s.startswith("#"):
            continue
        yield s


def read_smf(path, kind=None):
    """Mesh (coords num_nodes x 3, conn num_elems x npe, 0-based) from an SMF
    file.  kind: the element kind to build (default: Poisson of the header's
    shape; pass mg.HEX8_ELASTIC for elasticity on a hexahedral mesh)."""
    with open(path) as f:
        lines = f.read().splitlines()
    shape, npe = None, None
    body = []
    for line in lines:
        s = line.strip()
        if s.startswith("!"):
            parts = s[1:].split()
            if len(parts) >= 2 and parts[0] == "elementShape":
                shape = parts[1]
            elif len(parts) >= 2 and parts[0] == "elementNumPoints":
                npe = int(parts[1])
            continue
        if not s or s.startswith("#"):
            continue
        body.append(s)
    if shape is None or npe is None:
        raise ValueError("%s: SMF header lacks elementShape / elementNumPoints" % path)
    if kind is None:
        if (shape, npe) not in _SHAPE_KIND:
            raise ValueError("%s: unsupported element %s with %d points" % (path, shape, npe))
        kind = _SHAPE_KIND[(shape, npe)]
    nn, ne = (int(v) for v in body[0].split()[:2])
    coords = np.zeros((nn, 3))
    for i in range(nn):
        v = body[1 + i].split()
        coords[i, :len(v[:3])] = [float(t) for t in v[:3]]
    conn = np.array([[int(t) for t in body[1 + nn + e].split()[:npe]] for e in range(ne)], dtype=np.uint32)
    if conn.size and int(conn.max()) >= nn:
        raise ValueError("%s: element refers to node %d of %d" % (path, int(conn.max()), nn))
    return mg.Mesh(kind, coords, conn)


_KIND_SHAPE = {mg.LINE2_POISSON: ("line", 2), mg.TRI3_POISSON: ("triangle", 3), mg.HEX8_POISSON: ("hexahedron", 8),
               mg.HEX8_ELASTIC: ("hexahedron", 8)}


def write_smf(path, mesh):
    shape, npe = _KIND_SHAPE[mesh.kind]
    with open(path, "w") as f:
        f.write("! elementShape %s\n! elementNumPoints %d\n" % (shape, npe))
        f.write("%d %d\n" % (mesh.num_nodes, mesh.num_elems))
        for x in mesh.coords:
            f.write("%.17g %.17g %.17g\n" % tuple(x))
        for e in mesh.conn:
            f.write(" ".join(str(int(v)) for v in e) + "\n")


def read_properties(path):
    """name -> value string (corlib::PropertiesParser input)."""
    out = {}
    with open(path) as f:
        for s in _tokens_without_comments(f):
            parts = s.split(None, 1)
            if len(parts) == 2:
                out[parts[0]] = parts[1].split("#", 1)[0].strip()
    return out


def read_param_map(path):
    """apps::readParamToMap: key -> float."""
    out = {}
    with open(path) as f:
        for line in f:
            if not line.strip() or line.startswith("#"):
                continue
            t = line.split()
            for k in range(0, len(t) - 1, 2):
                try:
                    out[t[k]] = float(t[k + 1])
                except ValueError:
                    break
    return out


def read_matrix_phi(path, num_dofs):
    """apps::readMatrixPhi: dense P (rows from the largest row index + 1)."""
    data = np.loadtxt(path, ndmin=2)
    rows = data[:, 0].astype(np.int64)
    cols = data[:, 1].astype(np.int64)
    P = np.zeros((int(rows.max()) + 1, num_dofs))
    np.add.at(P, (rows, cols), data[:, 2])
    return P


def read_matrix_data(path):
    """apps::readMatrixData: 'rows cols' then the values row by row."""
    with open(path) as f:
        vals = f.read().split()
    r, c = int(vals[0]), int(vals[1])
    arr = np.array([float(v) for v in vals[2:]])
    if arr.size != r * c:
        raise ValueError("%s: expected %d values, found %d" % (path, r * c, arr.size))
    return arr.reshape(r, c)


def read_coord_data(path, dim):
    """apps::readCoordData: one point per line, dim coordinates each."""
    pts = []
    with open(path) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            if len(t) != dim:
                raise ValueError("%s: a point with %d coordinates, expected %d" % (path, len(t), dim))
            pts.append([float(v) for v in t])
    return np.array(pts)


def write_vector(path, v):
    """A vector the way Eigen streams one (six significant digits, right-aligned
    to a common width, one entry per line)."""
    s = ["%g" % x for x in np.asarray(v, dtype=np.float64)]
    w = max(len(t) for t in s) if s else 0
    with open(path, "w") as f:
        f.write("\n".join(t.rjust(w) for t in s))


def read_vector(path):
    with open(path) as f:
        return np.array([float(v) for v in f.read().split()])
