"""The .vtu / .pvd writer on CPU: structure, VTK node order, values read back."""
import xml.etree.ElementTree as ET

import numpy as np

from neon_b200 import mesh as M
from neon_b200 import vtk


def _arrays(path):
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    out = {}
    for da in root.iter("DataArray"):
        vals = np.array(da.text.split(), dtype=float)
        k = int(da.get("NumberOfComponents", "1"))
        out[da.get("Name")] = vals.reshape(-1, k) if k > 1 else vals
    return piece, out


def test_write_vtu_tet4_round_trip(tmp_path):
    m = M.structured_tet4(2, 1, 1)
    rng = np.random.Generator(np.random.PCG64(1))
    stress = rng.standard_normal((m.num_nodes, 9))
    vm = rng.standard_normal(m.num_nodes)
    p = tmp_path / "t.vtu"
    vtk.write_vtu(str(p), m.X, m.conn, {"cauchy_stress": stress, "von_mises_stress": vm})
    piece, a = _arrays(p)
    assert int(piece.get("NumberOfPoints")) == m.num_nodes
    assert int(piece.get("NumberOfCells")) == m.num_elements
    np.testing.assert_array_equal(a["Points"], m.X)
    np.testing.assert_array_equal(a["cauchy_stress"], stress)
    np.testing.assert_array_equal(a["von_mises_stress"], vm)
    conn = a["connectivity"].astype(int).reshape(-1, 4)
    np.testing.assert_array_equal(conn, m.conn[:, [1, 0, 2, 3]])  # convert_to_vtk for tet4
    assert set(a["types"].astype(int)) == {vtk.VTK_TETRA}
    np.testing.assert_array_equal(a["offsets"], 4 * np.arange(1, m.num_elements + 1))


def test_write_vtu_hex8_keeps_corner_order(tmp_path):
    m = M.structured_hex8(2, 1, 1)
    p = tmp_path / "h.vtu"
    vtk.write_vtu(str(p), m.X, m.conn, {})
    _, a = _arrays(p)
    np.testing.assert_array_equal(a["connectivity"].astype(int).reshape(-1, 8), m.conn)
    assert set(a["types"].astype(int)) == {vtk.VTK_HEXAHEDRON}


class _FakeMesh:
    def __init__(self, n):
        self.n = n

    def displacement(self):
        return np.arange(3 * self.n, dtype=float)

    def nodal_averaged(self, name):
        return np.full(self.n, 7.0)


def test_output_series_and_pvd(tmp_path):
    m = M.structured_hex8(1, 1, 1)
    out = vtk.VtkOutput("cube", ["displacement", "von_mises_stress"], write_every=2,
                        root=str(tmp_path))
    for step, t in enumerate([0.5, 1.0, 1.5]):
        out.write(step, t, _FakeMesh(m.num_nodes), m.X, m.conn)
    files = sorted(p.name for p in (tmp_path / "visualisation").iterdir())
    assert files == ["cube_0.vtu", "cube_2.vtu"]
    pvd = ET.parse(tmp_path / "cube.pvd").getroot()
    sets = [(float(d.get("timestep")), d.get("file")) for d in pvd.iter("DataSet")]
    assert sets == [(0.5, "visualisation/cube_0.vtu"), (1.5, "visualisation/cube_2.vtu")]
    _, a = _arrays(tmp_path / "visualisation" / "cube_2.vtu")
    np.testing.assert_array_equal(a["displacement"], np.arange(24.0).reshape(-1, 3))
