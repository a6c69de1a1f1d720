"""Non-follower loads on the device against the oracle (nonfollower_load.cpp:12-121): the nodal
vectors per unit load of a traction, a pressure and a body force, and static solves driven by
them.

Reference: neumann.hpp:69-192 (surface and volume loads), pressure.cpp:9-37 (pressure),
interpolation_factory.cpp:99-117 (surface rules).
"""
import numpy as np
import pytest

from conftest import rel_err
from neon_b200 import mesh as M
from neon_b200 import problem as P

pytestmark = pytest.mark.gpu

TOL = 1e-14


@pytest.fixture(scope="module")
def api():
    from neon_b200 import api, build
    build.build()
    api.lib()
    return api


def _warped_hex8():
    """A 4x3x5 box whose boundary is warped (non-planar faces)."""
    m = M.structured_hex8(4, 3, 5)
    X = m.X + 0.03 * np.sin(np.pi * m.X[:, [1, 2, 0]]) * np.sin(np.pi * m.X[:, [2, 0, 1]])
    return M.Mesh(X=X, conn=m.conn, faces=m.faces)


def _tri3(quads):
    """Each quad4 face as two tri3 faces (same orientation)."""
    return np.concatenate([quads[:, [0, 1, 2]], quads[:, [0, 2, 3]]]).astype(np.int32)


LE = P.make_material({"elastic_modulus": 1.0, "poissons_ratio": 0.3},
                     {"name": "isotropic_linear_elasticity"})


@pytest.mark.parametrize("topo", ["hex8", "tet4"])
def test_unit_load_vectors_match_oracle(api, oracle, topo):
    if topo == "hex8":
        m = _warped_hex8()
        faces = {k: v for k, v in m.faces.items()}
    else:
        m = M.structured_tet4(3, 2, 3)
        m = M.Mesh(X=m.X + 0.02 * np.sin(3.0 * m.X[:, [2, 0, 1]]), conn=m.conn, faces=m.faces)
        faces = {k: _tri3(v) for k, v in m.faces.items()}
    g = api.SolidMesh(m.X, m.conn, LE)
    om = oracle.OracleMesh(m.X, m.conn, LE)
    cases = [(P.PRESSURE, 0, faces["top"], False), (P.PRESSURE, 0, faces["x1"], False),
             (P.TRACTION, 2, faces["top"], False), (P.TRACTION, 0, faces["y0"], False),
             (P.BODY_FORCE, 2, None, False), (P.BODY_FORCE, 1, None, False)]
    if topo == "hex8":
        cases += [(P.TRACTION, 1, faces["x0"], True), (P.PRESSURE, 0, faces["bottom"], True)]
    for kind, comp, fc, red in cases:
        f = g.nonfollower_load(kind, comp, fc, red)
        fo = om.nonfollower_load(kind, comp, fc, red)
        assert np.count_nonzero(fo) > 0
        assert rel_err(f, fo) < TOL, (kind, comp, red)
    # the device vector is the same on every call (fixed-order node sums)
    f1 = g.nonfollower_load(P.PRESSURE, 0, faces["top"])
    f2 = g.nonfollower_load(P.PRESSURE, 0, faces["top"])
    assert np.array_equal(f1, f2)


def test_nonfollower_load_rejects_bad_input(api):
    m = M.structured_hex8(2)
    g = api.SolidMesh(m.X, m.conn, LE)
    bad = m.faces["top"].copy()
    bad[0, 0] = m.num_nodes  # out of range: refused on the host before any launch
    with pytest.raises(ValueError):
        g.nonfollower_load(P.PRESSURE, 0, bad)
    with pytest.raises(ValueError):
        g.nonfollower_load(P.TRACTION, 3, m.faces["top"])
    with pytest.raises(ValueError):
        g.nonfollower_load(7, 0, m.faces["top"])


def _loaded_block(material, pressure, gravity, increments, warped=True):
    m = _warped_hex8() if warped else M.structured_hex8(4, 3, 5)
    bcs = [{"name": "bottom", "type": "displacement", "time": [0.0, 1.0], "x": [0.0, 0.0],
            "y": [0.0, 0.0], "z": [0.0, 0.0]},
           {"name": "top", "type": "pressure", "time": [0.0, 1.0], "value": [0.0, pressure]},
           {"name": "x1", "type": "traction", "time": [0.0, 1.0], "y": [0.0, 0.5 * pressure]},
           {"name": "cube", "type": "body_force", "time": [0.0, 1.0], "z": [0.0, gravity]}]
    dt = 1.0 / increments
    opts = P.Options(residual_tolerance=1e-9, displacement_tolerance=1e-9, linear_iterations=15,
                     period=1.0, initial=dt, minimum=dt, maximum=dt, adaptive=False,
                     cg_tolerance=1e-12, cg_maximum_iterations=100000)
    return P.Problem("loaded_block", m, material, P.dirichlet_boundaries(m, bcs), opts,
                     loads=P.nonfollower_loads(m, bcs))


@pytest.mark.parametrize("model", ["linear_elastic", "neohooke"])
def test_static_solve_with_pressure_traction_and_body_force(api, oracle, model):
    if model == "linear_elastic":
        mat = P.make_material({"elastic_modulus": 200e3, "poissons_ratio": 0.3},
                              {"name": "isotropic_linear_elasticity"})
        pr = _loaded_block(mat, pressure=50.0, gravity=-20.0, increments=1)
    else:
        mat = P.make_material({"shear_modulus": 1.0, "bulk_modulus": 10.0}, {"name": "neohooke"})
        pr = _loaded_block(mat, pressure=0.2, gravity=-0.3, increments=3)
    assert [s.kind for s in pr.loads] == [P.PRESSURE, P.TRACTION, P.BODY_FORCE]
    rep_o, u_o, _, log_o, _ = oracle.static_solve(pr)
    assert rep_o["status"] == 0, rep_o["message"]
    sm = api.StaticMatrix(pr)
    u = sm.solve()
    assert sm.report["newton_iterations"] == rep_o["newton_iterations"]
    assert np.array_equal(sm.log[:, :2], log_o[:, :2])
    assert np.abs(u_o).max() > 0
    assert rel_err(u, u_o) < 1e-10
    # the loaded top moves down under compression and gravity
    top = np.unique(pr.mesh.faces["top"])
    assert u[3 * top + 2].mean() < 0
