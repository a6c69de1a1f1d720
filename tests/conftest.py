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


def cube_example_problem(example: str = "neohooke_cube_example"):
    """A cube example on the shared cube mesh as a Problem: the neo-Hookean one
    (examples/.../neohooke/cube), ``affine_microsphere_cube_example`` (Langevin statistics,
    examples/.../affine_microsphere/cube) or ``nonaffine_microsphere_cube_example``
    (examples/.../nonaffine_microsphere/cube)."""
    from neon_b200 import mesh as M
    from neon_b200 import problem as P
    with open(os.path.join(GOLDEN, "kats.json")) as fh:
        sim = json.load(fh)[example]["simulation"]
    data = np.load(os.path.join(GOLDEN, "neohooke_cube.npz"))
    faces = {k[6:]: data[k] for k in data.files if k.startswith("group_") and k != "group_cube"}
    mesh = M.Mesh(X=data["X"], conn=M.convert_from_gmsh(data["group_cube"],
                                                         int(data["type_cube"])), faces=faces)
    step = sim["steps"][0]
    part = step["meshes"][0]
    material = P.make_material(sim["materials"][0], part["constitutive"])
    bcs = P.dirichlet_boundaries(mesh, part["boundaries"])
    inc = step["time"]["increments"]
    nl = step["nonlinear_options"]
    ls = step["linear_solver"]
    # the path's linear solver is the PCG: a deck that asks for a direct solver (PaStiX) gets
    # the PCG at a tolerance well below the Newton tolerances instead
    iterative = ls.get("type") == "iterative"
    opts = P.Options(residual_tolerance=nl["residual_tolerance"],
                     displacement_tolerance=nl["displacement_tolerance"],
                     linear_iterations=nl.get("linear_iterations", 10),
                     period=step["time"]["period"], initial=inc["initial"], minimum=inc["minimum"],
                     maximum=inc["maximum"], adaptive=inc["adaptive"],
                     cg_tolerance=ls["tolerance"] if iterative else 1e-10,
                     cg_maximum_iterations=ls["maximum_iterations"] if iterative else 20000)
    return P.Problem(example, mesh, material, bcs, opts)
