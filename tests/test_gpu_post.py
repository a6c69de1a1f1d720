"""Quadrature variables averaged to the nodes on the device (neon's output fields) against the
oracle's restatement of submesh::nodal_averaged_variable + average_internal_variable, and a
.vtu written from a device solve."""
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from conftest import random_displacement, rel_err
from neon_b200 import mesh as M
from neon_b200 import problem as P
from test_gpu_parity import MATERIALS, SCALE

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from neon_b200 import api, build
    build.build()
    return api


@pytest.mark.parametrize("topo,model,fields", [
    ("hex8", "j2", ["cauchy_stress", "DetF", "plastic_strain", "accumulated_plastic_strain",
                    "von_mises_stress"]),
    ("hex8", "linear_elastic", ["cauchy_stress", "von_mises_stress", "DetF"]),
    ("tet4", "neohooke", ["cauchy_stress", "DetF"]),
])
def test_nodal_average_parity(api, oracle, topo, model, fields):
    m = M.structured_hex8(4, 3, 3, jitter=0.1, seed=3) if topo == "hex8" else \
        M.structured_tet4(3, 2, 2)
    mat = MATERIALS[model]
    u = random_displacement(m, SCALE[model], 11)
    g = api.SolidMesh(m.X, m.conn, mat)
    g.update_internal_variables(u)
    om = oracle.OracleMesh(m.X, m.conn, mat)
    st, _ = om.update(u)
    assert st == 0
    for f in fields:
        a, b = g.nodal_averaged(f), om.nodal_average(f)
        assert a.shape == b.shape, f
        assert rel_err(a, b) < 1e-12, f
    g.close()


def test_vtu_from_a_device_solve(api, tmp_path):
    from neon_b200 import vtk
    pr = P.config_c1(4)
    sm = api.StaticMatrix(pr)
    u = sm.solve()
    out = vtk.VtkOutput("c1", ["displacement", "cauchy_stress", "von_mises_stress"],
                        root=str(tmp_path))
    path = out.write(0, 1.0, sm.mesh, pr.mesh.X, pr.mesh.conn, displacement=u)
    root = ET.parse(path).getroot()
    arrays = {d.get("Name"): np.array(d.text.split(), float) for d in root.iter("DataArray")}
    np.testing.assert_allclose(arrays["displacement"], u, rtol=1e-15)
    assert arrays["cauchy_stress"].size == 9 * pr.mesh.num_nodes
    assert np.all(np.isfinite(arrays["von_mises_stress"]))
