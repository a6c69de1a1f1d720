import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (CUDA) and the built libneon_b200.so")


@pytest.fixture(scope="session")
def kats():
    with open(os.path.join(GOLDEN, "kats.json")) as fh:
        return json.load(fh)


@pytest.fixture(scope="session")
def oracle():
    from oracle import binding
    binding.lib()
    return binding


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def random_displacement(mesh, scale, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    return scale * rng.uniform(-1.0, 1.0, size=3 * mesh.num_nodes)


def cube_mesh_file():
    """The cube.mesh of the cube examples (examples/solid_mechanics/hyperelastic/neohooke/cube),
    rebuilt as parsed .mesh JSON from its golden copy."""
    data = np.load(os.path.join(GOLDEN, "neohooke_cube.npz"))
    groups = [k[6:] for k in data.files if k.startswith("group_")]
    return {"Nodes": [{"Coordinates": data["X"].tolist()}],
            "Elements": [{"Name": g, "Type": int(data["type_" + g]),
                          "NodalConnectivity": data["group_" + g].tolist()} for g in groups]}


def cube_example_deck(example: str = "neohooke_cube_example"):
    with open(os.path.join(GOLDEN, "kats.json")) as fh:
        return json.load(fh)[example]["simulation"]


def cube_example_problem(example: str = "neohooke_cube_example"):
    """A cube example on the shared cube mesh as a Problem, read from its deck: the neo-Hookean
    one (examples/.../neohooke/cube), ``affine_microsphere_cube_example`` (Langevin statistics,
    examples/.../affine_microsphere/cube) or ``nonaffine_microsphere_cube_example``
    (examples/.../nonaffine_microsphere/cube).  A deck that asks for a direct solver (PaStiX)
    gets the PCG at a tolerance well below the Newton tolerances instead."""
    from neon_b200 import deck as D
    pr = D.problem_from_deck(cube_example_deck(example), cube_mesh_file(),
                             direct_solver=(1e-10, 20000))
    pr.name = example
    return pr


def loaded_block_deck(element: str = "hex8", model: str = "neohooke"):
    """A deck and .mesh of neon's schema that uses every boundary kind on the path: a 4x3x3 box
    ("block"; hexahedron8, or tetrahedron4 stored in gmsh order) with its bottom clamped, a
    pressure on the top, a traction on x1 (x and z), a body force on the block, a nodal force
    on y1, and a two-block sinusoidal displacement on x0 (y).  Returns (deck, mesh_file)."""
    from neon_b200 import mesh as M
    m = M.structured_hex8(4, 3, 3) if element == "hex8" else M.structured_tet4(4, 3, 3)
    if element == "hex8":
        volume = {"Name": "block", "Type": 5, "NodalConnectivity": m.conn.tolist()}
        face = lambda q: {"Type": 3, "NodalConnectivity": q.tolist()}  # noqa: E731
    else:
        volume = {"Name": "block", "Type": 4,
                  "NodalConnectivity": m.conn[:, [3, 0, 1, 2]].tolist()}  # neon -> gmsh order
        face = lambda q: {"Type": 2, "NodalConnectivity": np.concatenate(  # noqa: E731
            [q[:, [0, 1, 2]], q[:, [0, 2, 3]]]).tolist()}
    groups = [volume] + [dict(face(m.faces[n]), Name=n) for n in ("bottom", "top", "x0", "x1",
                                                                   "y1")]
    mesh_file = {"Nodes": [{"Coordinates": m.X.tolist()}], "Elements": groups}
    if model == "neohooke":
        material = {"name": "rubber", "shear_modulus": 1.0, "bulk_modulus": 20.0}
        constitutive = {"name": "neohooke"}
        scale = 1.0
    else:
        material = {"name": "steel", "elastic_modulus": 200e3, "poissons_ratio": 0.3,
                    "yield_stress": 200.0, "isotropic_hardening_modulus": 1e3}
        constitutive = {"name": "J2_plasticity", "finite_strain": False}
        scale = 1e3
    deck = {
        "name": "loaded block",
        "parts": [{"name": "block", "material": material["name"]}],
        "materials": [material],
        "steps": [{
            "name": "load", "module": "solid_mechanics", "solution": "equilibrium",
            "nonlinear_options": {"residual_tolerance": 1e-8, "displacement_tolerance": 1e-8,
                                  "linear_iterations": 15},
            "time": {"period": 1.0, "increments": {"initial": 0.25, "minimum": 0.01,
                                                   "maximum": 0.5, "adaptive": True}},
            "meshes": [{
                "name": "block",
                "constitutive": constitutive,
                "element_options": {"quadrature": "full"},
                "boundaries": [
                    {"name": "bottom", "type": "displacement", "time": [0.0, 1.0],
                     "x": [0.0, 0.0], "y": [0.0, 0.0], "z": [0.0, 0.0]},
                    {"name": "top", "type": "pressure", "time": [0.0, 1.0],
                     "value": [0.0, 0.02 * scale]},
                    {"name": "x1", "type": "traction", "time": [0.0, 0.5, 1.0],
                     "x": [0.0, 0.01 * scale, 0.03 * scale], "z": [0.0, -0.01 * scale, 0.0]},
                    {"name": "block", "type": "body_force", "time": [0.0, 1.0],
                     "z": [0.0, -0.05 * scale]},
                    {"name": "y1", "type": "nodal_force", "time": [0.0, 1.0],
                     "y": [0.0, 1e-3 * scale]},
                    {"name": "x0", "type": "displacement", "generate_type": "sinusoidal",
                     "y": [2e-3, 1e-3], "period": [1.0, 1.0], "number_of_cycles": [0.5, 0.5],
                     "phase": [0.0, 3.141592653589793]}],
            }],
            "linear_solver": {"type": "iterative", "tolerance": 1e-12,
                              "maximum_iterations": 20000},
        }],
    }
    return deck, mesh_file


def run_adapter_driver(tmp_path, deck, mesh_file, *args):
    """Run the C++ driver's deck mode on a deck and .mesh (written under tmp_path); returns its
    JSON output, or None when the driver was built without nlohmann/json.hpp."""
    import subprocess
    from neon_b200 import build
    exe = build.build_adapter_driver()
    dp, mp = os.path.join(tmp_path, "deck.json"), os.path.join(tmp_path, "part.mesh")
    with open(dp, "w") as fh:
        json.dump(deck, fh)
    with open(mp, "w") as fh:
        json.dump(mesh_file, fh)
    r = subprocess.run([exe, "--deck", dp, "--mesh", mp, *args], capture_output=True,
                       text=True, timeout=600)
    if r.returncode == 2 and "nlohmann" in r.stdout:
        return None
    assert r.returncode == 0, r.stdout + r.stderr
    return json.loads(r.stdout)
