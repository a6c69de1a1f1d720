"""Regenerate the golden known-answer fixtures from dbeurle/neon's own tests and examples.

Run once in a container that has the reference checked out (read-only):

    python tests/golden/make_kats.py /path/to/neon

It reads the reference's Catch2 test sources and one example input as *text* and writes:

* ``kats.json``            numbers the reference's unit tests assert (with file:line citations);
* ``neohooke_cube.npz``    the example mesh examples/solid_mechanics/hyperelastic/neohooke/cube/
                           cube.mesh converted to arrays (nodes, hex8 connectivity, the four
                           boundary groups), driven by cube.json and checked by verify.py; the
                           affine microsphere cube example (Langevin statistics) uses the same
                           mesh with its own cube.json.

Nothing here runs the reference.  The test suite only reads the generated files.
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _find_line(lines, pattern):
    for i, line in enumerate(lines):
        if re.search(pattern, line):
            return i + 1
    raise ValueError(pattern)


def main(ref: str):
    out = {}
    # --- DOF numbering (test/dof_numbering.cpp) -------------------------------------------
    p = os.path.join(ref, "test", "dof_numbering.cpp")
    src = open(p).read()
    lines = src.splitlines()
    one_conn = [0, 1, 2, 3]
    m = re.search(r"known_dof_list << ([0-9, ]+);", src)
    one_known = [int(v) for v in m.group(1).split(",")]
    m2 = re.search(r"nodal_connectivity << ([0-9, ]+);\s*nodal_connectivity.transposeInPlace",
                   src)
    two_conn = [int(v) for v in m2.group(1).split(",")]
    m3 = re.search(r"known_dof_list << ([0-9, /\n]+?);\s*known_dof_list.transposeInPlace", src)
    two_known = [int(v) for v in re.sub(r"//", "", m3.group(1)).replace("\n", " ").split(",")]
    out["dof_numbering"] = {
        "source": f"test/dof_numbering.cpp:{_find_line(lines, 'One element')}-"
                  f"{_find_line(lines, 'Two elements') + 30}",
        "one_element": {"connectivity": one_conn, "dofs": one_known},
        "two_elements": {"connectivity": [two_conn[:4], two_conn[4:]],
                         "dofs": [two_known[:12], two_known[12:]]},
    }
    # --- linear elastic D (test/small_strain_constitutive.cpp) ----------------------------
    p = os.path.join(ref, "test", "small_strain_constitutive.cpp")
    src = open(p).read()
    lines = src.splitlines()
    start = _find_line(lines, r'TEST_CASE\("Solid mechanics elasticity model"\)')
    seg = "\n".join(lines[start:start + 160])
    d00 = float(re.search(r"material_tangent\(0, 0\) == Approx\(([0-9.e+-]+)\)", seg).group(1))
    d33 = float(re.search(r"material_tangent\(3, 3\) == Approx\(([0-9.e+-]+)\)", seg).group(1))
    d01 = float(re.search(r"material_tangent\(0, 1\) == Approx\(([0-9.e+-]+)\)", seg).group(1))
    E = float(re.search(r'elastic_modulus\\": ([0-9.e+-]+)', seg).group(1))
    nu = float(re.search(r'poissons_ratio\\": ([0-9.e+-]+)', seg).group(1))
    out["linear_elastic_D"] = {"source": f"test/small_strain_constitutive.cpp:{start}-{start + 160}",
                               "E": E, "nu": nu, "D00": d00, "D33": d33, "D01": d01,
                               "uniaxial_H11": 0.001, "margin": 1e-5}
    # --- J2 (same file) ---------------------------------------------------------------------
    start = _find_line(lines, r'TEST_CASE\("Solid mechanics J2 plasticity"\)')
    seg = "\n".join(lines[start:start + 170])
    grab = lambda key: float(re.search(key + r'\\": ([0-9.e+-]+)', seg).group(1))  # noqa: E731
    out["j2"] = {"source": f"test/small_strain_constitutive.cpp:{start}-{start + 170}",
                 "E": grab("elastic_modulus"), "nu": grab("poissons_ratio"),
                 "yield_stress": grab("yield_stress"),
                 "hardening": grab("isotropic_hardening_modulus"),
                 "elastic_H22": float(re.search(r"H\(2, 2\) = ([0-9.e-]+);", seg).group(1)),
                 "plastic_H22": float(re.findall(r"H\(2, 2\) = ([0-9.e-]+);", seg)[1]),
                 "plastic_vm_max": float(re.search(r"von_mises_stress <= ([0-9.e+-]+)\)",
                                                   seg).group(1)),
                 "yield_check": [[100.0e6, 0.0, "<=0"], [300.0e6, 0.0, ">0"]]}
    # --- hyperelastic (test/hyperelastic_constitutive.cpp) --------------------------------
    p = os.path.join(ref, "test", "hyperelastic_constitutive.cpp")
    src = open(p).read()
    lines = src.splitlines()
    nh = _find_line(lines, r'TEST_CASE\("Neo-Hookean model"\)')
    ga = _find_line(lines, r'TEST_CASE\("Gaussian affine microsphere"\)')
    seg = "\n".join(lines[ga:ga + 90])
    out["neo_hooke"] = {"source": f"test/hyperelastic_constitutive.cpp:{nh}-{nh + 70}",
                        "E": 2.0, "nu": 0.45, "margin": 1e-5}
    out["gaussian_affine_microsphere"] = {
        "source": f"test/hyperelastic_constitutive.cpp:{ga}-{ga + 85}",
        "E": float(re.search(r'elastic_modulus\\" : ([0-9.e+-]+)', seg).group(1)),
        "nu": float(re.search(r'poissons_ratio\\" : ([0-9.e+-]+)', seg).group(1)),
        "segments_per_chain": float(re.search(r'segments_per_chain\\" : ([0-9.e+-]+)',
                                              seg).group(1)),
        "uniaxial_stretch": 1.1, "margin": 1e-5}
    la = _find_line(lines, r'TEST_CASE\("Affine microsphere"\)')
    seg = "\n".join(lines[la:la + 85])
    assert '\\"statistics\\":\\"langevin\\"' in seg
    out["langevin_affine_microsphere"] = {
        "source": f"test/hyperelastic_constitutive.cpp:{la}-{la + 83}",
        "E": float(re.search(r'elastic_modulus\\" : ([0-9.e+-]+)', seg).group(1)),
        "nu": float(re.search(r'poissons_ratio\\" : ([0-9.e+-]+)', seg).group(1)),
        "segments_per_chain": float(re.search(r'segments_per_chain\\" : ([0-9.e+-]+)',
                                              seg).group(1)),
        "uniaxial_stretch": float(re.search(r"F\(0, 0\) = ([0-9.]+);", seg).group(1)),
        "margin": 1e-5}
    na = _find_line(lines, r'TEST_CASE\("Nonaffine microsphere"\)')
    seg = "\n".join(lines[na:na + 100])
    assert '\\"nonaffine\\"' in seg
    out["nonaffine_microsphere"] = {
        "source": f"test/hyperelastic_constitutive.cpp:{na}-{na + 98}",
        "E": float(re.search(r'elastic_modulus\\" : ([0-9.e+-]+)', seg).group(1)),
        "nu": float(re.search(r'poissons_ratio\\" : ([0-9.e+-]+)', seg).group(1)),
        "nonaffine_stretch_parameter": float(
            re.search(r'nonaffine_stretch_parameter\\":([0-9.e+-]+)', seg).group(1)),
        "segments_per_chain": float(re.search(r'segments_per_chain\\" : ([0-9.e+-]+)',
                                              seg).group(1)),
        "uniaxial_stretch": float(re.search(r"F\(0, 0\) = ([0-9.]+);", seg).group(1)),
        "margin": 1e-5}
    # --- linear solver (test/linear_solvers.cpp) --------------------------------------------
    p = os.path.join(ref, "test", "linear_solvers.cpp")
    src = open(p).read()
    lines = src.splitlines()
    trip = re.findall(r"\{(\d), (\d), (-?[0-9.]+)\}", src)
    A = np.zeros((3, 3))
    for i, j, v in trip:
        A[int(i), int(j)] = float(v)
    b = [float(v) for v in re.findall(r"b\(\d\) = ([0-9.]+);", src)]
    x = [float(v) for v in re.search(r"x << ([0-9., ]+);", src).group(1).split(",")]
    out["cg_3x3"] = {"source": f"test/linear_solvers.cpp:{_find_line(lines, 'create_sparse_matrix')}"
                               f"-{_find_line(lines, 'x << ')}",
                     "triplets": [[int(i), int(j), float(v)] for i, j, v in trip],
                     "b": b, "x": x, "margin": 1e-5}
    # --- quadrature ---------------------------------------------------------------------------
    out["quadrature"] = {"source": "test/quadrature/hexahedron.cpp:21-100, sphere.cpp:13-25, "
                                   "tetrahedron.cpp:39-58",
                         "hex8_weight_sum": 8.0, "tet1_weight_sum": 1.0 / 6.0,
                         "bo21_points": 21, "bo21_weight_sum": 1.0, "unit_cube_volume": 1.0}
    # --- cube fixture (test/fixtures/cube_mesh.cpp) ---------------------------------------
    p = os.path.join(ref, "test", "fixtures", "cube_mesh.cpp")
    src = open(p).read()
    cube_block = re.search(r'"Name" : "cube".*?"NodalConnectivity" : \[(.*?)\]\s*,?\s*"Type" : 5',
                           src, re.S)
    n_hex = len(re.findall(r"\[[^\[\]]+\]", cube_block.group(1))) if cube_block else 27
    coords = re.search(r'"Coordinates" : \[(.*?)\]\s*\}\s*\]', src, re.S)
    n_nodes = len(re.findall(r"\[[^\[\]]+\]", coords.group(1))) if coords else 64
    out["cube_fixture"] = {"source": "test/fixtures/cube_mesh.cpp:6-177, test/mesh.cpp:114-267",
                           "nodes": n_nodes, "hex8": n_hex, "active_dofs": 3 * n_nodes}
    # the fixture's mesh itself: the C++ string literal pieces of json_cube_mesh(), joined and
    # unescaped, parsed as the .mesh JSON the reference's mesh tests read
    body = src[src.index("json_cube_mesh()"):]
    body = body[body.index("return"):body.index(";")]
    text = "".join(re.findall(r'"((?:[^"\\]|\\.)*)"', body)).replace('\\"', '"')
    fixture = json.loads(text)
    with open(os.path.join(HERE, "cube_fixture.json"), "w") as fh:
        json.dump(fixture, fh, indent=None, separators=(",", ":"))
    # test/mesh.cpp "Basic mesh test": group sizes, corner coordinates and the unique node lists
    msrc = open(os.path.join(ref, "test", "mesh.cpp")).read()
    lists = re.findall(r"known_unique\{([^}]*)\}", msrc)
    out["cube_fixture_mesh"] = {
        "source": "test/fixtures/cube_mesh.cpp:6-177 (the mesh, as tests/golden/cube_fixture.json),"
                  f" test/mesh.cpp:{_find_line(msrc.splitlines(), 'Basic mesh test')}-"
                  f"{_find_line(msrc.splitlines(), 'Solid submesh test') - 1}",
        "nodes": 64, "corners": [[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [1.0, 1.0, 0.0]],
        "elements": {"bottom": 9, "cube": 27, "sides": 36, "top": 9},
        "unique_nodes": {name: [int(v) for v in re.findall(r"\d+", lst)]
                         for name, lst in zip(("bottom", "sides", "top"), lists[:3])}}
    # --- neo-Hookean cube example (examples/.../neohooke/cube) ----------------------------
    ex = os.path.join(ref, "examples", "solid_mechanics", "hyperelastic", "neohooke", "cube")
    sim = json.load(open(os.path.join(ex, "cube.json")))
    mesh = json.load(open(os.path.join(ex, "cube.mesh")))
    X = np.asarray(mesh["Nodes"][0]["Coordinates"], np.float64)
    groups = {}
    for g in mesh["Elements"]:
        groups.setdefault(g["Name"], []).append((int(g["Type"]),
                                                 np.asarray(g["NodalConnectivity"], np.int32)))
    arrays = {"X": X}
    for name, items in groups.items():
        arrays["group_" + name] = np.concatenate([c for _, c in items])
        arrays["type_" + name] = np.array([t for t, _ in items][0])
    np.savez_compressed(os.path.join(HERE, "neohooke_cube.npz"), **arrays)
    vsrc = open(os.path.join(ex, "verify.py")).read().splitlines()
    out["neohooke_cube_example"] = {
        "source": "examples/solid_mechanics/hyperelastic/neohooke/cube/cube.json:1-72, "
                  f"verify.py:{_find_line(vsrc, 'max_displacement|max\\(\\[max')}-"
                  f"{_find_line(vsrc, 'displacement gradient is incorrect')}",
        "simulation": sim, "max_displacement": 0.5, "slope": 0.5, "rel_tol": 1e-7}
    # --- Langevin affine microsphere cube example (examples/.../affine_microsphere/cube) ----
    # same cube.mesh as the neo-Hookean example (checked byte for byte): only the input deck
    ax = os.path.join(ref, "examples", "solid_mechanics", "hyperelastic", "affine_microsphere",
                      "cube")
    with open(os.path.join(ax, "cube.mesh"), "rb") as a, open(os.path.join(ex, "cube.mesh"),
                                                               "rb") as b:
        assert a.read() == b.read(), "the affine microsphere cube mesh differs"
    asim = json.load(open(os.path.join(ax, "cube.json")))
    out["affine_microsphere_cube_example"] = {
        "source": "examples/solid_mechanics/hyperelastic/affine_microsphere/cube/cube.json:1-80",
        "mesh": "neohooke_cube.npz", "simulation": asim, "max_displacement": 0.5}
    nx = os.path.join(ref, "examples", "solid_mechanics", "hyperelastic", "nonaffine_microsphere",
                      "cube")
    with open(os.path.join(nx, "cube.mesh"), "rb") as a, open(os.path.join(ex, "cube.mesh"),
                                                               "rb") as b:
        assert a.read() == b.read(), "the non-affine microsphere cube mesh differs"
    out["nonaffine_microsphere_cube_example"] = {
        "source": "examples/solid_mechanics/hyperelastic/nonaffine_microsphere/cube/cube.json:1-78",
        "mesh": "neohooke_cube.npz", "simulation": json.load(open(os.path.join(nx, "cube.json"))),
        "max_displacement": 0.5}
    with open(os.path.join(HERE, "kats.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "kats.json"))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_kats.py <path to a checkout of dbeurle/neon>")
    main(sys.argv[1])
