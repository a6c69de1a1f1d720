"""neon input decks and .mesh files: the Python reader (neon_b200/deck.py) and the C++ one
(include/neon_b200_json.hpp, through the adapter driver's --parse-only mode) against each other,
against hand-built problems, and against neon's error behaviour (simulation_parser.cpp,
static_matrix.hpp:109-143, adaptive_time_step.cpp:108-160, linear_solver_factory.cpp:20-120,
boundary.cpp:87-176, constitutive_model_factory.cpp:26-161, mesh.cpp:75-104, 229-248).
No GPU: parsing never touches the device."""
import copy
import math

import numpy as np
import pytest

from conftest import (cube_example_deck, cube_example_problem, cube_mesh_file, loaded_block_deck,
                      run_adapter_driver)
from neon_b200 import deck as D
from neon_b200 import mesh as M
from neon_b200 import problem as P

EXAMPLES = ("neohooke_cube_example", "affine_microsphere_cube_example",
            "nonaffine_microsphere_cube_example")


def _material_row(m: P.Material):
    return [m.model, m.K, m.G, m.yield_stress, m.hardening, m.segments_per_chain,
            m.nonaffine_stretch_parameter]


def _options_row(o: P.Options):
    return [o.residual_tolerance, o.displacement_tolerance, o.linear_iterations,
            int(o.absolute_tolerance), o.period, o.initial, o.minimum, o.maximum, int(o.adaptive),
            o.cg_tolerance, o.cg_maximum_iterations]


def _same_tables(py, cpp):
    assert len(py) == len(cpp)
    for a, b in zip(py, cpp):
        assert np.array_equal(a.dofs, b["dofs"])
        assert np.array_equal(a.times, b["times"])   # bitwise: the same arithmetic both sides
        assert np.array_equal(a.values, b["values"])


def _check_same_parse(tmp_path, deck, mesh_file, **kw):
    pr = D.problem_from_deck(deck, mesh_file, **kw)
    args = ["--parse-only"]
    if "direct_solver" in kw:
        args += ["--direct", repr(kw["direct_solver"][0]), str(kw["direct_solver"][1])]
    out = run_adapter_driver(tmp_path, deck, mesh_file, *args)
    if out is None:
        pytest.skip("the adapter driver was built without nlohmann/json.hpp")
    assert "error" not in out, out
    assert out["nodes"] == pr.mesh.num_nodes
    assert out["nodes_per_element"] == pr.mesh.nodes_per_element
    assert np.array_equal(np.asarray(out["connectivity"]).reshape(pr.mesh.conn.shape),
                          pr.mesh.conn)
    assert out["material"][:7] == _material_row(pr.material)
    if pr.material.model in (P.GAUSS_AFFINE_MICROSPHERE, P.LANGEVIN_AFFINE_MICROSPHERE,
                             P.NONAFFINE_MICROSPHERE):
        assert out["material"][7] == pr.material.unit_sphere_points
    assert out["options"] == _options_row(pr.options)
    _same_tables(pr.dirichlet, out["dirichlet"])
    _same_tables(pr.nodal_forces, out["nodal_forces"])
    assert len(out["loads"]) == len(pr.loads)
    for spec, c in zip(pr.loads, out["loads"]):
        assert (c["kind"], c["component"], bool(c["reduced"]), c["name"]) == \
            (spec.kind, spec.component, spec.reduced, spec.name)
        assert np.array_equal(spec.times, c["times"]) and np.array_equal(spec.values, c["values"])
        if spec.faces is None:
            assert c["faces"] == []
        else:
            assert np.array_equal(np.asarray(c["faces"]).reshape(spec.faces.shape), spec.faces)
    return pr, out


@pytest.mark.parametrize("example", EXAMPLES)
def test_cube_example_decks(tmp_path, example):
    """neon's three cube example decks on the example mesh: the Python and C++ readers agree
    field by field, and the deck gives the example's material, Newton options and the four
    symmetry / load boundaries (names sorted as static_matrix iterates them)."""
    pr, _ = _check_same_parse(tmp_path, cube_example_deck(example), cube_mesh_file(),
                              direct_solver=(1e-10, 20000))
    assert [t.name for t in pr.dirichlet] == ["Xsym", "Ysym", "ZLoad", "Zsym"]
    zload = pr.dirichlet[2]
    assert np.array_equal(zload.values, [0.0, 0.5]) and len(zload.dofs) == 36
    assert np.all(zload.dofs % 3 == 2)
    assert pr.mesh.num_nodes == 216 and pr.mesh.num_elements == 125


@pytest.mark.parametrize("element", ["hex8", "tet4"])
@pytest.mark.parametrize("model", ["neohooke", "j2"])
def test_loaded_block_deck(tmp_path, element, model):
    """Every boundary kind on the path (displacement with a two-block sinusoid, pressure,
    traction, body force, nodal force) on hexahedra and gmsh-ordered tetrahedra: both readers
    agree, the tetrahedra come back in neon's local order, and the tables follow neon's rules."""
    deck, mesh_file = loaded_block_deck(element, model)
    pr, _ = _check_same_parse(tmp_path, deck, mesh_file)
    ref = M.structured_hex8(4, 3, 3) if element == "hex8" else M.structured_tet4(4, 3, 3)
    assert np.array_equal(pr.mesh.conn, ref.conn)
    # Dirichlet: bottom x, y, z then x0 y (names sorted), DOFs = unique face nodes * 3 + k
    assert [t.name for t in pr.dirichlet] == ["bottom"] * 3 + ["x0"]
    bottom = np.unique(ref.faces["bottom"])
    for k in range(3):
        assert np.array_equal(pr.dirichlet[k].dofs, 3 * bottom + k)
    # the two sinusoid blocks (boundary.cpp:87-147): 2 samples each at dt 0.25, the second block
    # starting where the first ended
    t, v = pr.dirichlet[3].times, pr.dirichlet[3].values
    assert np.allclose(t, [0.0, 0.25, 0.5, 0.75, 1.0], rtol=0, atol=1e-15)
    w = 2.0 * math.pi
    expect = [0.0, 2e-3 * math.sin(w * 0.25), 2e-3 * math.sin(w * 0.5),
              1e-3 * math.sin(w * 0.75 + math.pi), 1e-3 * math.sin(w * 1.0 + math.pi)]
    assert np.allclose(v, expect, rtol=0, atol=1e-18)
    kinds = [(s.kind, s.component, s.name) for s in pr.loads]
    assert kinds == [(P.PRESSURE, 0, "top"), (P.TRACTION, 0, "x1"), (P.TRACTION, 2, "x1"),
                     (P.BODY_FORCE, 2, "block")]
    assert len(pr.nodal_forces) == 1
    assert np.array_equal(pr.nodal_forces[0].dofs, 3 * np.unique(ref.faces["y1"]) + 1)
    if model == "j2":
        assert pr.material.model == P.J2_SMALL_STRAIN
        assert pr.material.yield_stress == 200.0 and pr.material.hardening == 1e3


def test_deck_matches_hand_built_problem():
    """The deck route gives exactly the problem that the hand-built cube example used to:
    the same mesh, material, Dirichlet tables and options."""
    pr = cube_example_problem("neohooke_cube_example")
    deck = cube_example_deck("neohooke_cube_example")
    step = deck["steps"][0]
    mat = P.make_material(deck["materials"][0], step["meshes"][0]["constitutive"])
    assert pr.material == mat
    assert pr.options.cg_tolerance == step["linear_solver"]["tolerance"]
    assert pr.options.cg_maximum_iterations == step["linear_solver"]["maximum_iterations"]
    assert pr.options.adaptive and pr.options.minimum == 0.001


def _errors(tmp_path, deck, mesh_file, **kw):
    """The Python error message and the C++ one (None when the driver has no JSON support)."""
    with pytest.raises((ValueError, NotImplementedError)) as info:
        D.problem_from_deck(deck, mesh_file, **kw)
    out = run_adapter_driver(tmp_path, deck, mesh_file, "--parse-only")
    cpp = None
    if out is not None:
        assert out.get("error") == "domain_error", out
        cpp = out["what"].strip()
    return str(info.value).strip(), cpp


def _step(deck):
    return deck["steps"][0]


def _part(deck):
    return deck["steps"][0]["meshes"][0]


ERROR_CASES = {
    "missing residual tolerance": (
        lambda d: _step(d)["nonlinear_options"].pop("residual_tolerance"),
        "residual_tolerance not specified in nonlinear_options"),
    "missing period": (lambda d: _step(d)["time"].pop("period"),
                       'Time data requires a "period" value'),
    "missing minimum increment": (lambda d: _step(d)["time"]["increments"].pop("minimum"),
                                  "increment minimum value not provided!"),
    "unknown linear solver": (lambda d: _step(d)["linear_solver"].update(type="spectral"),
                              'Linear solver spectral is not recognised.  Please use "PaStiX", '
                              '"MUMPS", "direct" or "iterative"'),
    "direct solver": (lambda d: _step(d)["linear_solver"].update(type="direct"),
                      'linear solver "direct": the path solves with the Jacobi PCG ("type": '
                      '"iterative")'),
    "poissons ratio": (lambda d: d["materials"][0].update(poissons_ratio=0.5),
                       '"poissons_ratio" must be less than or equal to 0.5'),
    "unknown model": (lambda d: _part(d)["constitutive"].update(name="hypoelastic"),
                      "The model name hypoelastic is not recognised"),
    "missing finite_strain": (lambda d: _part(d)["constitutive"].pop("finite_strain"),
                              '"small_strain_J2_plasticity" must have a boolean value for '
                              '"finite_strain"'),
    "missing yield stress": (lambda d: d["materials"][0].pop("yield_stress"),
                             '"yield_stress" was not specified in material properties'),
    "reduced hexahedra": (lambda d: _part(d)["element_options"].update(quadrature="reduced"),
                          "reduced (one-point) hexahedron8 quadrature is not on this path; the "
                          "element kernels integrate hexahedron8 with eight points"),
    "no element options": (lambda d: _part(d).pop("element_options"),
                           'Missing "part": {"element_options" : {}}'),
    "no time on a boundary": (lambda d: _part(d)["boundaries"][0].pop("time"),
                              'Neither "time" nor "generate_type" was specified in "boundary".'),
    "unsorted times": (lambda d: _part(d)["boundaries"][2].update(time=[0.0, 1.0, 0.5]),
                       "Load times must be monotonically increasing."),
    "short table": (lambda d: _part(d)["boundaries"][1].update(time=[0.0], value=[0.0]),
                    '"time" is not a vector of at least two elements'),
    "pressure without value": (lambda d: _part(d)["boundaries"][1].pop("value"),
                               'Pressure boundary condition must specify a "value" array'),
    "unknown boundary": (lambda d: _part(d)["boundaries"][1].update(type="spring"),
                         'boundary "spring" is not recognised'),
    "sinusoid sizes": (lambda d: _part(d)["boundaries"][5].update(phase=[0.0]),
                       "The amplitude, period, number_of_cycles, time_step and phase vectors "
                       "must be of the same size."),
    "missing boundary group": (lambda d: _part(d)["boundaries"][0].update(name="floor"),
                               'The mesh name "floor" does not exist in the mesh file'),
}


@pytest.mark.parametrize("case", sorted(ERROR_CASES))
def test_deck_errors(tmp_path, case):
    """Each malformed deck is refused by both readers with neon's message (or, for what the path
    does not cover, the same message of ours)."""
    deck, mesh_file = loaded_block_deck("hex8", "j2")
    deck = copy.deepcopy(deck)
    edit, message = ERROR_CASES[case]
    edit(deck)
    py, cpp = _errors(tmp_path, deck, mesh_file)
    assert py == message
    if cpp is not None:
        assert cpp == message


def test_mesh_file_errors(tmp_path):
    deck, mesh_file = loaded_block_deck("hex8", "neohooke")
    bad = copy.deepcopy(mesh_file)
    bad["Elements"][0]["NodalConnectivity"][0][0] = 10**6
    py, cpp = _errors(tmp_path, deck, bad)
    assert py == 'group "block" refers to a node that does not exist'
    assert cpp in (None, py)
    bad = copy.deepcopy(mesh_file)
    bad["Elements"][0]["Type"] = 17  # hexahedron20
    with pytest.raises(NotImplementedError):
        D.problem_from_deck(deck, bad)
    out = run_adapter_driver(tmp_path, deck, bad, "--parse-only")
    if out is not None:
        assert out["error"] == "domain_error" and "gmsh element type 17" in out["what"]


def test_body_force_on_another_group_is_refused(tmp_path):
    deck, mesh_file = loaded_block_deck("hex8", "neohooke")
    _part(deck)["boundaries"][3]["name"] = "top"
    with pytest.raises(NotImplementedError, match="body force acts on the part"):
        D.problem_from_deck(deck, mesh_file)
    out = run_adapter_driver(tmp_path, deck, mesh_file, "--parse-only")
    if out is not None:
        assert out["error"] == "domain_error" and "body force acts on the part" in out["what"]


def test_non_adaptive_and_absolute_tolerance():
    """adaptive false pins the minimum and maximum increments to the initial one
    (adaptive_time_step.cpp:112-118); the mere presence of "absolute_tolerance" switches the
    Newton test to absolute norms (static_matrix.hpp:127-130); the iterative solver's defaults
    are 1e-5 and 2000 (linear_solver.hpp:49-50)."""
    deck, mesh_file = loaded_block_deck("hex8", "neohooke")
    step = _step(deck)
    step["time"]["increments"]["adaptive"] = False
    step["nonlinear_options"]["absolute_tolerance"] = False
    step["linear_solver"] = {"type": "iterative"}
    pr = D.problem_from_deck(deck, mesh_file)
    o = pr.options
    assert (o.initial, o.minimum, o.maximum, o.adaptive) == (0.25, 0.25, 0.25, False)
    assert o.absolute_tolerance
    assert (o.cg_tolerance, o.cg_maximum_iterations) == (1e-5, 2000)


def test_split_groups_are_joined(tmp_path):
    """A part (and a boundary) stored as several groups of one name, as gmsh writes physical
    groups made of several entities: basic_mesh::meshes returns them all, and both readers join
    them into one element list and one set of boundary nodes."""
    deck, mesh_file = loaded_block_deck("hex8", "neohooke")
    groups = []
    for g in mesh_file["Elements"]:
        conn = g["NodalConnectivity"]
        half = len(conn) // 2
        groups.append(dict(g, NodalConnectivity=conn[:half]))
        groups.append(dict(g, NodalConnectivity=conn[half:]))
    split = dict(mesh_file, Elements=groups)
    whole, _ = _check_same_parse(tmp_path, deck, mesh_file)
    parts, _ = _check_same_parse(tmp_path, deck, split)
    assert np.array_equal(parts.mesh.conn, whole.mesh.conn)
    _same_tables(whole.dirichlet, [{"dofs": t.dofs, "times": t.times, "values": t.values}
                                   for t in parts.dirichlet])
    for a, b in zip(whole.loads, parts.loads):
        assert np.array_equal(a.faces, b.faces) if a.faces is not None else b.faces is None


def test_mixed_element_types_in_a_group_are_refused(tmp_path):
    """One group name holding quadrilateral and triangle faces: neither reader runs it (one
    element type per group is on this path)."""
    deck, mesh_file = loaded_block_deck("hex8", "neohooke")
    bad = copy.deepcopy(mesh_file)
    top = next(g for g in bad["Elements"] if g["Name"] == "top")
    tri = [q[:3] for q in top["NodalConnectivity"][:2]]
    bad["Elements"].append({"Name": "top", "Type": 2, "NodalConnectivity": tri})
    with pytest.raises(NotImplementedError, match="mixes element types"):
        D.problem_from_deck(deck, bad)
    out = run_adapter_driver(tmp_path, deck, bad, "--parse-only")
    if out is not None:
        assert out["error"] == "domain_error" and "mixes element types" in out["what"]
