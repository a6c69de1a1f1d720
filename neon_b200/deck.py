"""neon input decks: a simulation ``.json`` and a part's ``.mesh`` file to a Problem.

Follows the reader side of neon's solid-mechanics path:

* simulation_parser.cpp:60-135, 226-295 -- the deck's ``name`` / ``materials`` / ``parts`` /
  ``steps``, unique material and part names, one mesh per step;
* basic_mesh.cpp:8-19, nodal_coordinates.cpp:13-33, node_ordering_adapter.cpp:46-68 -- the mesh
  file (``Nodes[0].Coordinates``, ``Elements[{Name, Type, NodalConnectivity}]``) with gmsh
  ordering converted to neon's;
* solid_mechanics_module.cpp:9-17 and mechanics/solid/mesh.cpp:24-143, 229-248 -- the part's
  element groups, the boundary checks, Dirichlet boundaries and non-follower loads;
* static_matrix.hpp:109-143, adaptive_time_step.cpp:108-160, linear_solver_factory.cpp:20-120
  -- nonlinear options, time increments and the linear solver.

The C++ header ``include/neon_b200_json.hpp`` does the same for a C++ caller holding
``nlohmann::json`` values.
"""
from __future__ import annotations

import json
import os

import numpy as np

from . import problem as P
from .mesh import Mesh, convert_from_gmsh

# gmsh type -> nodes per element, for the element types on this path
# (mesh/element_topology.hpp: 2 triangle3, 3 quadrilateral4, 4 tetrahedron4, 5 hexahedron8)
GMSH_NODES = {2: 3, 3: 4, 4: 4, 5: 8}
VOLUME_TYPES = (4, 5)


class BasicMesh:
    """The contents of a ``.mesh`` file: coordinates [N, 3] and the element groups by name, each
    a list of (gmsh type, connectivity in neon's local order) as basic_mesh keeps them."""

    def __init__(self, mesh_file):
        if isinstance(mesh_file, (str, os.PathLike)):
            with open(mesh_file) as fh:
                mesh_file = json.load(fh)
        for key in ("Nodes", "Elements"):
            if key not in mesh_file:
                raise ValueError(f'The mesh file is missing the "{key}" field')
        self.X = np.asarray(mesh_file["Nodes"][0]["Coordinates"], dtype=np.float64)
        if self.X.ndim != 2 or self.X.shape[1] != 3:
            raise ValueError('"Coordinates" must be a list of [x, y, z] triples')
        self.groups: dict[str, list] = {}
        for group in mesh_file["Elements"]:
            gtype = int(group["Type"])
            if gtype not in GMSH_NODES:
                raise NotImplementedError(f"gmsh element type {gtype} is not on this path "
                                          "(hexahedron8, tetrahedron4 and their faces are)")
            conn = np.asarray(group["NodalConnectivity"], dtype=np.int32)
            if conn.ndim != 2 or conn.shape[1] != GMSH_NODES[gtype]:
                raise ValueError(f'group "{group["Name"]}": type {gtype} needs '
                                 f"{GMSH_NODES[gtype]} nodes per element")
            if conn.size and (conn.min() < 0 or conn.max() >= len(self.X)):
                raise ValueError(f'group "{group["Name"]}" refers to a node that does not exist')
            self.groups.setdefault(group["Name"], []).append(
                (gtype, convert_from_gmsh(conn, gtype)))

    def meshes(self, name: str) -> list:
        """basic_mesh::meshes: every group of that name (an error when there is none)."""
        if name not in self.groups:
            raise ValueError(f'The mesh name "{name}" does not exist in the mesh file')
        return self.groups[name]

    def connectivity(self, name: str) -> tuple[int, np.ndarray]:
        """The groups of one name joined into one [E, npe] array (one element type)."""
        items = self.meshes(name)
        types = {t for t, _ in items}
        if len(types) != 1:
            raise NotImplementedError(f'group "{name}" mixes element types {sorted(types)}; '
                                      "one element type per group is on this path")
        return items[0][0], np.concatenate([c for _, c in items]).astype(np.int32)


def check_deck(deck: dict) -> None:
    """simulation_parser: the required top-level fields, unique material names, parts that name
    an existing material, unique part names (simulation_parser.cpp:60-76, 226-295)."""
    for key in ("name", "materials", "parts", "steps"):
        if key not in deck:
            raise ValueError(f'"{key}" is not in input file')
    names = set()
    for material in deck["materials"]:
        if "name" not in material:
            raise ValueError('"material" is missing the "name" field')
        if material["name"] in names:
            raise ValueError("The material name must be unique")
        names.add(material["name"])
    parts = set()
    for part in deck["parts"]:
        if "name" not in part:
            raise ValueError('"part" : {"name" : ""} is missing')
        if part.get("material") not in names:
            raise ValueError("The part material was not found in the provided materials")
        if part["name"] in parts:
            raise ValueError("A part is defined more than once")
        parts.add(part["name"])
    for step in deck["steps"]:
        for field in ("name", "time", "solution"):
            if field not in step:
                raise ValueError(f'A simulation case needs a "{field}" field')
        if len(step.get("meshes", [])) != 1:
            raise ValueError("Multibody simulation are not yet supported")
        if step["meshes"][0]["name"] not in parts:
            raise ValueError(f'Mesh name "{step["meshes"][0]["name"]}" was not found in the '
                             "mesh store")


def solver_options(step: dict, direct_solver: tuple | None = None) -> P.Options:
    """static_matrix's nonlinear options, adaptive_time_step's increments and the iterative
    linear solver's tolerance / iteration limit, with neon's defaults and errors.

    The path's linear solver is the Jacobi PCG; a deck asking for a direct solver ("direct",
    "PaStiX", "MUMPS") is refused unless ``direct_solver`` = (tolerance, maximum iterations)
    gives the PCG settings to use in its place."""
    nl = step.get("nonlinear_options", {})
    for key in ("displacement_tolerance", "residual_tolerance"):
        if key not in nl:
            raise ValueError(f"{key} not specified in nonlinear_options")
    time = step["time"]
    if "period" not in time:
        raise ValueError('Time data requires a "period" value')
    if "increments" not in time:
        raise ValueError('"increments" not provided!')
    inc = time["increments"]
    for key in ("initial", "minimum", "maximum"):
        if key not in inc:
            raise ValueError(f"increment {key} value not provided!")
    if "adaptive" not in inc:
        raise ValueError('"adaptive" (true or false) not provided in "increments"')
    adaptive = bool(inc["adaptive"])
    initial = float(inc["initial"])
    ls = step.get("linear_solver")
    if ls is None or "type" not in ls:
        raise ValueError('A "linear_solver" "type" must be specified')
    kind = ls["type"]
    if kind not in ("PaStiX", "MUMPS", "direct", "iterative"):
        raise ValueError(f'Linear solver {kind} is not recognised.  Please use "PaStiX", '
                         '"MUMPS", "direct" or "iterative"')
    if kind == "iterative":
        cg_tol = float(ls.get("tolerance", 1.0e-5))
        cg_maxit = int(ls.get("maximum_iterations", 2000))
    elif direct_solver is not None:
        cg_tol, cg_maxit = float(direct_solver[0]), int(direct_solver[1])
    else:
        raise NotImplementedError(f'linear solver "{kind}": the path solves with the Jacobi '
                                  'PCG ("type": "iterative")')
    return P.Options(residual_tolerance=float(nl["residual_tolerance"]),
                     displacement_tolerance=float(nl["displacement_tolerance"]),
                     linear_iterations=int(nl.get("linear_iterations", 10)),
                     absolute_tolerance="absolute_tolerance" in nl,
                     period=float(time["period"]), initial=initial,
                     minimum=float(inc["minimum"]) if adaptive else initial,
                     maximum=float(inc["maximum"]) if adaptive else initial,
                     adaptive=adaptive, cg_tolerance=cg_tol, cg_maximum_iterations=cg_maxit)


def _is_reduced(mesh_data: dict) -> bool:
    """interpolation_factory.cpp:20-33: "element_options" must exist; "quadrature": "reduced"
    selects the reduced rules."""
    if "element_options" not in mesh_data:
        raise ValueError('Missing "part": {"element_options" : {}}')
    return mesh_data["element_options"].get("quadrature") == "reduced"


def problem_from_deck(deck, mesh_file, step: int = 0,
                      direct_solver: tuple | None = None) -> P.Problem:
    """One load step of a neon deck as a Problem (solid_mechanics_module: the part's mesh with
    its material, the step's ``meshes[0]`` entry, ``time.increments.initial`` as the generate
    time step of sinusoidal boundaries).  ``deck`` is the parsed ``.json`` (or its path),
    ``mesh_file`` the part's ``.mesh`` (a path, parsed JSON or a BasicMesh)."""
    if isinstance(deck, (str, os.PathLike)):
        with open(deck) as fh:
            deck = json.load(fh)
    check_deck(deck)
    sim = deck["steps"][step]
    mesh_data = sim["meshes"][0]
    part = next(p for p in deck["parts"] if p["name"] == mesh_data["name"])
    material_data = next(m for m in deck["materials"] if m["name"] == part["material"])
    if "constitutive" not in mesh_data:
        raise ValueError('Missing "constitutive" in "mesh"')
    material = P.make_material(material_data, mesh_data["constitutive"])
    basic = mesh_file if isinstance(mesh_file, BasicMesh) else BasicMesh(mesh_file)
    gtype, conn = basic.connectivity(mesh_data["name"])
    if gtype not in VOLUME_TYPES:
        raise ValueError(f'part "{mesh_data["name"]}" is not a volume mesh')
    reduced = _is_reduced(mesh_data)
    if reduced and gtype == 5:
        raise NotImplementedError("reduced (one-point) hexahedron8 quadrature is not on this "
                                  "path; the element kernels integrate hexahedron8 with eight "
                                  "points")
    boundaries = mesh_data.get("boundaries", [])
    for b in boundaries:
        for field in ("name", "type"):
            if field not in b:
                raise ValueError(f'"{field}" was not specified in "boundary".')
        if "time" not in b and "generate_type" not in b:
            raise ValueError('Neither "time" nor "generate_type" was specified in "boundary".')
        if b["type"] not in ("displacement", "traction", "pressure", "body_force",
                             "nodal_force"):
            raise ValueError(f'boundary "{b["type"]}" is not recognised')
    faces = {}
    for b in boundaries:
        if b["type"] == "body_force":
            if b["name"] != mesh_data["name"]:
                raise NotImplementedError("a body force acts on the part's own elements on this "
                                          f'path; "{b["name"]}" is another group')
            continue
        if b["name"] in faces:
            continue
        ftype, fconn = basic.connectivity(b["name"])
        if b["type"] in ("traction", "pressure") and ftype not in (2, 3):
            raise ValueError(f'surface load "{b["name"]}" is not a group of faces')
        faces[b["name"]] = fconn
    mesh = Mesh(X=basic.X, conn=conn, faces=faces)
    dt = float(sim["time"]["increments"]["initial"])
    dirichlet = P.dirichlet_boundaries(mesh, boundaries, dt)
    loads = P.nonfollower_loads(mesh, boundaries, dt, reduced=reduced)
    nodal = []
    for b in boundaries:
        if b["type"] != "nodal_force":
            continue
        nodes = mesh.boundary_nodes(b["name"])
        for comp, key in enumerate("xyz"):
            if key in b:
                t, v = P.boundary_table(b, key, dt)
                nodal.append(P.DofTable((3 * nodes + comp).astype(np.int32), t, v,
                                        name=b["name"]))
    options = solver_options(sim, direct_solver)
    return P.Problem(deck["name"], mesh, material, dirichlet, options, nodal_forces=nodal,
                     loads=loads)
