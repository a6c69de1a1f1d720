"""The .mesh reader (neon_b200.mesh.read_neon_mesh) on the reference's own mesh data: its mesh
test fixture and its neo-Hookean cube example, written out in neon's .mesh JSON format in the
test and read back, plus the gmsh -> neon tet4 reordering and the boundary DOF sets.

Reference: mesh/basic_mesh.cpp:8-19 and basic_submesh.cpp:12-53 (groups), nodal_coordinates.cpp:
13-33 (coordinates), node_ordering_adapter.cpp:46-68 (tet4: neon = gmsh (1, 2, 3, 0)),
dof_allocator.hpp:19-47 (sorted unique boundary nodes x 3 + component), test/mesh.cpp "Basic
mesh test" (the known answers), test/fixtures/cube_mesh.cpp (the fixture mesh).
"""
import json
import os

import numpy as np

from conftest import GOLDEN
from neon_b200 import mesh as M
from neon_b200 import problem as P


def _write(tmp_path, name, data):
    path = os.path.join(str(tmp_path), name)
    with open(path, "w") as fh:
        json.dump(data, fh)
    return path


def test_reference_cube_fixture(tmp_path, kats, oracle):
    k = kats["cube_fixture_mesh"]
    with open(os.path.join(GOLDEN, "cube_fixture.json")) as fh:
        fixture = json.load(fh)
    m = M.read_neon_mesh(_write(tmp_path, "cube.mesh", fixture), "cube")
    assert m.num_nodes == k["nodes"] == kats["cube_fixture"]["nodes"]
    np.testing.assert_array_equal(m.X[:4], np.array(k["corners"]))
    assert m.conn.shape == (k["elements"]["cube"], 8)
    for name in ("bottom", "sides", "top"):
        assert m.faces[name].shape == (k["elements"][name], 4)
    for name, nodes in k["unique_nodes"].items():
        assert np.array_equal(m.boundary_nodes(name), np.array(nodes, np.int32))
    # the volume group uses every node (test/mesh.cpp: unique nodes of "cube" = 0..63)
    assert np.array_equal(np.unique(m.conn), np.arange(64))
    # boundary DOF sets: sorted unique nodes x 3 + component, per listed component, in x, y, z
    # order (mesh.cpp:116-143 with dof_allocator.hpp:19-37)
    bcs = [{"name": "bottom", "time": [0.0, 1.0], "x": [0.0, 0.0], "z": [0.0, 0.0]},
           {"name": "top", "time": [0.0, 1.0], "y": [0.0, 1.0]}]
    tables = P.dirichlet_boundaries(m, bcs)
    bottom = np.array(k["unique_nodes"]["bottom"])
    top = np.array(k["unique_nodes"]["top"])
    assert [t.name for t in tables] == ["bottom", "bottom", "top"]
    assert np.array_equal(tables[0].dofs, 3 * bottom + 0)
    assert np.array_equal(tables[1].dofs, 3 * bottom + 2)
    assert np.array_equal(tables[2].dofs, 3 * top + 1)
    # 192 active DOFs on the oracle (test/mesh.cpp: number_of_active_dofs)
    mat = P.make_material({"elastic_modulus": 1.0, "poissons_ratio": 0.3},
                          {"name": "isotropic_linear_elasticity"})
    om = oracle.OracleMesh(m.X, m.conn, mat)
    assert om.ndofs == kats["cube_fixture"]["active_dofs"] == 192


def test_neohooke_cube_example_round_trip(tmp_path):
    """The example mesh of examples/solid_mechanics/hyperelastic/neohooke/cube, rewritten as a
    .mesh file and read back: the same nodes, hex8 connectivity and boundary groups."""
    data = np.load(os.path.join(GOLDEN, "neohooke_cube.npz"))
    groups = [k[6:] for k in data.files if k.startswith("group_")]
    mesh_json = {"Nodes": [{"Coordinates": data["X"].tolist()}],
                 "Elements": [{"Name": g, "Type": int(data["type_" + g]),
                               "NodalConnectivity": data["group_" + g].tolist()} for g in groups]}
    m = M.read_neon_mesh(_write(tmp_path, "cube.mesh", mesh_json), "cube")
    np.testing.assert_array_equal(m.X, data["X"])
    np.testing.assert_array_equal(m.conn, data["group_cube"])
    assert sorted(m.faces) == sorted(g for g in groups if g != "cube")
    for g in m.faces:
        np.testing.assert_array_equal(m.faces[g], data["group_" + g])
    assert m.num_nodes == 216 and m.num_elements == 125


def test_tet4_gmsh_ordering(tmp_path):
    """A tet4 mesh stored in gmsh order (type 4, tri3 boundary faces of type 2) reads back in
    neon's local order (1, 2, 3, 0), in which every element's Jacobian (columns x0-x3, x1-x3,
    x2-x3, tetrahedron.cpp:6-45) is positive."""
    ref = M.structured_tet4(2, 3, 2)
    gmsh = ref.conn[:, [3, 0, 1, 2]]  # the inverse of neon = gmsh (1, 2, 3, 0)
    tri = np.concatenate([ref.faces["top"][:, [0, 1, 2]], ref.faces["top"][:, [0, 2, 3]]])
    mesh_json = {"Nodes": [{"Coordinates": ref.X.tolist()}],
                 "Elements": [{"Name": "block", "Type": 4, "NodalConnectivity": gmsh.tolist()},
                              {"Name": "top", "Type": 2, "NodalConnectivity": tri.tolist()}]}
    m = M.read_neon_mesh(_write(tmp_path, "block.mesh", mesh_json), "block")
    assert np.array_equal(m.conn, ref.conn)
    X = m.X
    a = X[m.conn[:, 0]] - X[m.conn[:, 3]]
    b = X[m.conn[:, 1]] - X[m.conn[:, 3]]
    c = X[m.conn[:, 2]] - X[m.conn[:, 3]]
    assert (np.einsum("ij,ij->i", a, np.cross(b, c)) > 0).all()
    assert np.array_equal(m.boundary_nodes("top"), np.unique(ref.faces["top"]))
    # a misspelt volume group is an error, not an empty mesh
    try:
        M.read_neon_mesh(_write(tmp_path, "block2.mesh", mesh_json), "blok")
    except ValueError:
        pass
    else:
        raise AssertionError("a missing part must raise")
