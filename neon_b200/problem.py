"""Problem description in neon's terms: material, constitutive model, Dirichlet boundaries,
nodal forces, nonlinear / time / linear-solver options.

The JSON keys follow neon's input schema (e.g. examples/solid_mechanics/hyperelastic/neohooke/
cube/cube.json:1-72) so the same dictionaries drive the oracle and the device path.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .mesh import Mesh, quad4_consistent_forces, structured_hex8, structured_tet4

# Model identifiers of the C-ABI (include/neon_b200.h, enum nb2_model)
LINEAR_ELASTIC, NEO_HOOKE, J2_SMALL_STRAIN, GAUSS_AFFINE_MICROSPHERE = 0, 1, 2, 3
LANGEVIN_AFFINE_MICROSPHERE, NONAFFINE_MICROSPHERE = 4, 5

MODEL_NAMES = {
    LINEAR_ELASTIC: "isotropic_linear_elasticity",
    NEO_HOOKE: "neohooke",
    J2_SMALL_STRAIN: "J2_plasticity",
    GAUSS_AFFINE_MICROSPHERE: "microsphere",
    LANGEVIN_AFFINE_MICROSPHERE: "microsphere",
    NONAFFINE_MICROSPHERE: "microsphere",
}


@dataclasses.dataclass
class Material:
    """Isotropic parameters as neon stores them: bulk and shear modulus
    (material/isotropic_elastic_property.cpp:10-43), yield stress and linear isotropic hardening
    (material/isotropic_elastic_plastic.cpp:10-38), segments per chain
    (material/micromechanical_elastomer.cpp:13-21), the non-affine stretch parameter
    (constitutive/mechanics/solid/nonaffine_microsphere.cpp:17-25)."""
    model: int
    K: float
    G: float
    yield_stress: float = 0.0
    hardening: float = 0.0
    segments_per_chain: float = 0.0
    nonaffine_stretch_parameter: float = 0.0
    unit_sphere_points: int = 21  # microsphere quadrature: BO21 or BO33

    @property
    def lam(self) -> float:
        return self.K - 2.0 * self.G / 3.0

    def params(self) -> np.ndarray:
        return np.array([self.K, self.G, self.yield_stress, self.hardening,
                         self.segments_per_chain, self.nonaffine_stretch_parameter,
                         float(self.unit_sphere_points)], dtype=np.float64)


def _check_microsphere_options(constitutive: dict):
    """The microsphere branch of make_constitutive_model (constitutive_model_factory.cpp:48-120):
    type and quadrature present and known, then the chain statistics of the affine model."""
    for key, msg in (("type", 'Missing "type" as "affine" or "nonaffine" in microsphere model'),
                     ("quadrature", 'Missing "quadrature" as "BO21", "BO33" or "FM900" in '
                                    'microsphere model')):
        if key not in constitutive:
            raise ValueError(msg)
    if constitutive["quadrature"] not in ("BO21", "BO33", "FM900"):
        raise ValueError('"quadrature" field must be "BO21", "BO33" or "FM900"')
    if constitutive["type"] == "affine":
        if "statistics" not in constitutive:
            raise ValueError('Missing "statistics" as "gaussian" or "langevin" in the '
                             'microsphere model')
        if constitutive["statistics"] not in ("gaussian", "langevin"):
            raise ValueError('"statistics" for the microsphere model must be either '
                             '"gaussian" or "langevin"')
    elif constitutive["type"] != "nonaffine":
        raise ValueError('microsphere model options are "affine" or "nonaffine"')


def make_material(material: dict, constitutive: dict) -> Material:
    """Restates the factory make_constitutive_model (constitutive_model_factory.cpp:26-161) for the
    five models on the path, and the parameter parsing of isotropic_elastic_property."""
    if "name" not in constitutive:
        raise ValueError('Missing "name" in "constitutive"')
    name = constitutive["name"]
    if name == "microsphere":
        _check_microsphere_options(constitutive)
    if "bulk_modulus" in material and "shear_modulus" in material:
        K, G = float(material["bulk_modulus"]), float(material["shear_modulus"])
    elif "elastic_modulus" in material and "poissons_ratio" in material:
        E, nu = float(material["elastic_modulus"]), float(material["poissons_ratio"])
        if nu >= 0.5:
            raise ValueError('"poissons_ratio" must be less than or equal to 0.5')
        K = E / (3.0 * (1.0 - 2.0 * nu))
        G = E / (2.0 * (1.0 + nu))
    else:
        raise ValueError('"elastic_modulus" and "poissons_ratio" or "bulk_modulus" and '
                         '"shear_modulus" need to be specified as material properties')
    if name in ("neohooke", "compressible_neohooke"):
        return Material(NEO_HOOKE, K, G)
    if name == "isotropic_linear_elasticity":
        return Material(LINEAR_ELASTIC, K, G)
    if name == "J2_plasticity":
        if "finite_strain" not in constitutive:
            raise ValueError('"small_strain_J2_plasticity" must have a boolean value for '
                             '"finite_strain"')
        if constitutive["finite_strain"]:
            raise NotImplementedError("finite-strain J2 is not on this path")
        if "yield_stress" not in material:
            raise ValueError('"yield_stress" was not specified in material properties')
        return Material(J2_SMALL_STRAIN, K, G, float(material["yield_stress"]),
                        float(material.get("isotropic_hardening_modulus", 0.0)))
    if name == "microsphere":
        affine = constitutive["type"] == "affine"
        if constitutive["quadrature"] == "FM900" or \
                (affine and "ageing" in constitutive and constitutive["statistics"] == "gaussian"):
            raise NotImplementedError("the microsphere models (affine Gaussian, affine Langevin, "
                                      "non-affine) are on this path with the BO21 and BO33 rules")
        points = 33 if constitutive["quadrature"] == "BO33" else 21
        if "segments_per_chain" not in material:
            raise ValueError("segments_per_chain not specified in material data")
        N = float(material["segments_per_chain"])
        if not affine:
            if "nonaffine_stretch_parameter" not in material:
                raise ValueError('"nonaffine_stretch_parameter" not specified in material data')
            return Material(NONAFFINE_MICROSPHERE, K, G, segments_per_chain=N,
                            nonaffine_stretch_parameter=float(
                                material["nonaffine_stretch_parameter"]),
                            unit_sphere_points=points)
        model = GAUSS_AFFINE_MICROSPHERE if constitutive["statistics"] == "gaussian" \
            else LANGEVIN_AFFINE_MICROSPHERE
        return Material(model, K, G, segments_per_chain=N, unit_sphere_points=points)
    raise ValueError(f"The model name {name} is not recognised")


@dataclasses.dataclass
class DofTable:
    """A Dirichlet boundary (nodal_value, mesh/boundary/nodal_value.cpp) or a nodal force: DOFs
    and a time/value table interpolated linearly (mesh/boundary/boundary.cpp:55-85).  For forces,
    ``weights`` scales the value per DOF (consistent forces of a unit traction)."""
    dofs: np.ndarray
    times: np.ndarray
    values: np.ndarray
    weights: np.ndarray | None = None
    name: str = ""


def sinusoidal_table(amplitude, period, number_of_cycles, phase, generate_time_step):
    """boundary::generate_sinusoidal (mesh/boundary/boundary.cpp:87-147): a time/value table that
    starts at (0, 0) and appends one block of sampled sine cycles per entry of the four lists
    (scalars are one block).  Each block has floor(cycles * period / generate_time_step) samples
    spread evenly over its cycles and starts where the previous block ended."""
    lists = [np.atleast_1d(np.asarray(a, dtype=np.float64))
             for a in (amplitude, period, number_of_cycles, phase)]
    if len({len(a) for a in lists}) != 1:
        raise ValueError("The amplitude, period, number_of_cycles, time_step and phase vectors "
                         "must be of the same size.")
    times, values = [0.0], [0.0]
    for A, T, n, ph in zip(*lists):
        omega = 2.0 * math.pi / T
        steps = int(n * T / generate_time_step)
        block = np.arange(1, steps + 1, dtype=np.float64)
        t = block * (n * T / block[-1]) + times[-1]
        times.extend(t.tolist())
        values.extend((A * np.sin(omega * t + ph)).tolist())
    return np.asarray(times), np.asarray(values)


def time_value_table(times, values):
    """boundary::allocate_time_load (mesh/boundary/boundary.cpp:150-176): at least two points,
    equal lengths, times non-decreasing."""
    t = np.asarray(times, dtype=np.float64).reshape(-1)
    v = np.asarray(values, dtype=np.float64).reshape(-1)
    if t.size < 2:
        raise ValueError('"time" is not a vector of at least two elements')
    if v.size < 2:
        raise ValueError("The specified boundary values do not contain at least two elements")
    if t.size != v.size:
        raise ValueError("The time and load vectors must be of the same size.")
    if np.any(np.diff(t) < 0.0):
        raise ValueError("Load times must be monotonically increasing.")
    return t, v


def boundary_table(boundary: dict, key: str, generate_time_step: float):
    """The time/value table of one component of a boundary (boundary.cpp:20-34): neon's
    sinusoidal generator when ``generate_type`` is "sinusoidal", else ``time`` and the
    component's values."""
    if "generate_type" in boundary:
        if boundary["generate_type"] != "sinusoidal":
            raise ValueError(f'"generate_type" {boundary["generate_type"]!r} is not supported')
        for field in ("period", "phase", "number_of_cycles"):
            if field not in boundary:
                raise ValueError(f'"{field}" was not specified in "boundaries".')
        t, v = sinusoidal_table(boundary[key], boundary["period"], boundary["number_of_cycles"],
                                boundary["phase"], generate_time_step)
        return time_value_table(t, v)
    return time_value_table(boundary["time"], boundary[key])


def dirichlet_boundaries(mesh: Mesh, boundaries: list, generate_time_step: float = 1.0):
    """mesh<submesh>::allocate_displacement_boundary (mesh/mechanics/solid/mesh.cpp:116-143).

    Returns DofTables in the order static_matrix iterates them: boundary names sorted (std::map),
    and within a name the components x, y, z (the dof_table map)."""
    out = []
    for b in sorted(boundaries, key=lambda b: b["name"]):
        if b.get("type", "displacement") != "displacement":
            continue
        nodes = mesh.boundary_nodes(b["name"])
        for comp, key in enumerate("xyz"):
            if key not in b:
                continue
            t, v = boundary_table(b, key, generate_time_step)
            out.append(DofTable((3 * nodes + comp).astype(np.int32), t, v, name=b["name"]))
    return out


TRACTION, PRESSURE, BODY_FORCE = 0, 1, 2


@dataclasses.dataclass
class LoadSpec:
    """One non-follower load boundary (nonfollower_load_boundary, mechanics/solid/boundary/
    nonfollower_load.cpp:12-121): a traction (component) or a pressure on a group of boundary
    faces, or a body force (component) over the volume elements, scaled by its time table.
    Its nodal vector per unit value is computed by whichever implementation solves the problem
    (the device, or the oracle when it checks the device)."""
    kind: int
    times: np.ndarray
    values: np.ndarray
    component: int = 0
    faces: np.ndarray | None = None   # int32 [F, 3 or 4] (surface loads)
    reduced: bool = False             # quad4 faces on the 1-point rule ("quadrature": "reduced")
    name: str = ""


def nonfollower_loads(mesh: Mesh, boundaries: list, generate_time_step: float = 1.0,
                      reduced: bool = False) -> list:
    """The traction / pressure / body_force boundaries of a neon deck as LoadSpecs, in the order
    neon builds them (nonfollower_load.cpp:21-72: per boundary, traction and body force once per
    listed component x, y, z; pressure reads its "value" array)."""
    out = []
    for b in boundaries:
        kind = b.get("type", "displacement")
        if kind not in ("traction", "pressure", "body_force"):
            continue
        if kind == "pressure":
            if "value" not in b:
                raise ValueError('Pressure boundary condition must specify a "value" array')
            t, v = time_value_table(b["time"], b["value"])
            out.append(LoadSpec(PRESSURE, t, v, 0, mesh.faces[b["name"]],
                                reduced, b["name"]))
            continue
        for comp, key in enumerate("xyz"):
            if key not in b:
                continue
            t, v = boundary_table(b, key, generate_time_step)
            if kind == "traction":
                out.append(LoadSpec(TRACTION, t, v, comp, mesh.faces[b["name"]], reduced,
                                    b["name"]))
            else:
                out.append(LoadSpec(BODY_FORCE, t, v, comp, None, False, b["name"]))
    return out


def load_tables(spec: LoadSpec, f: np.ndarray) -> DofTable:
    """A LoadSpec with its unit-load nodal vector f [3N] as a weighted DOF table."""
    if spec.kind == BODY_FORCE:
        nodes = np.arange(len(f) // 3)
    else:
        nodes = np.unique(np.asarray(spec.faces).reshape(-1))
    comps = (0, 1, 2) if spec.kind == PRESSURE else (spec.component,)
    dofs = np.sort(np.concatenate([3 * nodes + k for k in comps])).astype(np.int32)
    return DofTable(dofs, np.asarray(spec.times, float), np.asarray(spec.values, float),
                    weights=f[dofs].copy(), name=spec.name)


@dataclasses.dataclass
class Options:
    """nonlinear_options (static_matrix.hpp:109-143), time/increments
    (solver/adaptive_time_step.cpp:12-165) and linear_solver (linear_solver_factory.cpp:27-65)."""
    residual_tolerance: float = 1e-3
    displacement_tolerance: float = 1e-3
    linear_iterations: int = 10
    absolute_tolerance: bool = False
    period: float = 1.0
    initial: float = 1.0
    minimum: float = 1.0
    maximum: float = 1.0
    adaptive: bool = False
    cg_tolerance: float = 1e-5
    cg_maximum_iterations: int = 2000
    use_rcm: bool = True


@dataclasses.dataclass
class Problem:
    name: str
    mesh: Mesh
    material: Material
    dirichlet: list
    options: Options
    nodal_forces: list = dataclasses.field(default_factory=list)
    element_shear_modulus: np.ndarray | None = None
    loads: list = dataclasses.field(default_factory=list)  # LoadSpec (non-follower loads)

    @property
    def ndofs(self) -> int:
        return 3 * self.mesh.num_nodes


def _rollers(extra):
    b = [{"name": "x0", "type": "displacement", "time": [0.0, 1.0], "x": [0.0, 0.0]},
         {"name": "y0", "type": "displacement", "time": [0.0, 1.0], "y": [0.0, 0.0]},
         {"name": "bottom", "type": "displacement", "time": [0.0, 1.0], "z": [0.0, 0.0]}]
    return b + extra


def config_c1(n: int = 20) -> Problem:
    """Small-strain isotropic linear elasticity, E=200e3, nu=0.3, unit cube n^3 hex8, z=0 fully
    fixed, uz=1e-3 on z=1, one increment, Jacobi-PCG rtol 1e-10."""
    mesh = structured_hex8(n)
    mat = make_material({"elastic_modulus": 200e3, "poissons_ratio": 0.3},
                        {"name": "isotropic_linear_elasticity"})
    bcs = [{"name": "bottom", "time": [0.0, 1.0], "x": [0.0, 0.0], "y": [0.0, 0.0],
            "z": [0.0, 0.0]},
           {"name": "top", "time": [0.0, 1.0], "z": [0.0, 1e-3]}]
    opts = Options(residual_tolerance=1e-6, displacement_tolerance=1e-6, linear_iterations=10,
                   period=1.0, initial=1.0, minimum=1.0, maximum=1.0, adaptive=False,
                   cg_tolerance=1e-10, cg_maximum_iterations=100000)
    return Problem("c1_linear_elastic_hex8_%d" % n, mesh, mat, dirichlet_boundaries(mesh, bcs), opts)


def config_c2(n: int = 64, seed: int = 20240601, increments: int = 10) -> Problem:
    """Compressible neo-Hooke (mu=1, K=10), n^3 hex8 with interior nodes jittered by U(+-0.1h)
    (PCG64 seed), symmetry rollers on x=0/y=0/z=0, top stretch to 1.3 in equal increments."""
    mesh = structured_hex8(n, jitter=0.1, seed=seed)
    mat = make_material({"shear_modulus": 1.0, "bulk_modulus": 10.0}, {"name": "neohooke"})
    bcs = _rollers([{"name": "top", "type": "displacement", "time": [0.0, 1.0], "z": [0.0, 0.3]}])
    dt = 1.0 / increments
    opts = Options(residual_tolerance=1e-8, displacement_tolerance=1e-8, linear_iterations=15,
                   period=1.0, initial=dt, minimum=dt, maximum=dt, adaptive=False,
                   cg_tolerance=1e-10, cg_maximum_iterations=200000)
    return Problem("c2_neohooke_hex8_%d" % n, mesh, mat, dirichlet_boundaries(mesh, bcs), opts)


def config_c3(n: int = 100, steps: int = 20, increments_per_step: int = 4) -> Problem:
    """Small-strain J2 plasticity with linear isotropic hardening (E=200e3, nu=0.3, sigma_y=200,
    H=1e3), n^3 hex8, bottom clamped, top uz = 5e-3 sin(2 pi t / steps): one +-5e-3 cycle over
    `steps` time units (neon's sinusoidal generator, period = steps), each unit split into
    `increments_per_step` load increments (generate_time_step = 1 / increments_per_step).

    With neon's J2 update (plastic strain accumulated at every Newton iteration,
    small_strain_J2_plasticity.cpp:35-86) full Newton diverges on 1.56e-3 increments of the top
    displacement once the mesh is 40^3 or finer.  At 4 increments per unit most increments
    converge, but at 100^3 some do not (the first at t = 1.25), so the time stepping is neon's
    adaptive one (adaptive_time_step.cpp:25-92): a failed increment is halved, down to 1/16 of
    the initial one, and the step grows back to at most the initial increment."""
    mesh = structured_hex8(n)
    mat = make_material({"elastic_modulus": 200e3, "poissons_ratio": 0.3, "yield_stress": 200.0,
                         "isotropic_hardening_modulus": 1e3},
                        {"name": "J2_plasticity", "finite_strain": False})
    bcs = [{"name": "bottom", "time": [0.0, float(steps)], "x": [0.0, 0.0], "y": [0.0, 0.0],
            "z": [0.0, 0.0]},
           {"name": "top", "generate_type": "sinusoidal", "z": [5e-3], "period": [float(steps)],
            "phase": [0.0], "number_of_cycles": [1.0]}]
    dt = 1.0 / increments_per_step
    opts = Options(residual_tolerance=1e-8, displacement_tolerance=1e-8, linear_iterations=15,
                   period=float(steps), initial=dt, minimum=dt / 16.0, maximum=dt, adaptive=True,
                   cg_tolerance=1e-10, cg_maximum_iterations=200000)
    return Problem("c3_j2_hex8_%d" % n, mesh, mat, dirichlet_boundaries(mesh, bcs, dt), opts)


def config_c4(n: int = 48, seed_field: int = 7, traction: float = 0.05,
              statistics: str = "gaussian", segments_per_chain: float = 50.0,
              nonaffine_stretch_parameter: float = 1.0) -> Problem:
    """Affine microsphere (BO21, K=100, G=1 scaled by a per-element lognormal(0, 0.3) field;
    Gaussian chains, or Langevin chains of ``segments_per_chain`` segments; ``statistics=
    "nonaffine"`` for the non-affine model), n^3 hex8, bottom clamped, uniform top traction in z
    (consistent quad4 forces)."""
    mesh = structured_hex8(n)
    constitutive = {"name": "microsphere", "type": "affine", "statistics": statistics,
                    "quadrature": "BO21"}
    if statistics == "nonaffine":
        constitutive = {"name": "microsphere", "type": "nonaffine", "quadrature": "BO21"}
    mat = make_material({"bulk_modulus": 100.0, "shear_modulus": 1.0,
                         "segments_per_chain": segments_per_chain,
                         "nonaffine_stretch_parameter": nonaffine_stretch_parameter},
                        constitutive)
    rng = np.random.Generator(np.random.PCG64(seed_field))
    Ge = rng.lognormal(mean=0.0, sigma=0.3, size=mesh.num_elements) * mat.G
    bcs = [{"name": "bottom", "time": [0.0, 1.0], "x": [0.0, 0.0], "y": [0.0, 0.0],
            "z": [0.0, 0.0]}]
    dofs, w = quad4_consistent_forces(mesh, "top", (0.0, 0.0, 1.0))
    nf = [DofTable(dofs, np.array([0.0, 1.0]), np.array([0.0, traction]), weights=w, name="top")]
    opts = Options(residual_tolerance=1e-9, displacement_tolerance=1e-9, linear_iterations=15,
                   period=1.0, initial=1.0, minimum=1.0, maximum=1.0, adaptive=False,
                   cg_tolerance=1e-10, cg_maximum_iterations=200000)
    name = "c4_microsphere_hex8_%d" % n if statistics == "gaussian" else \
        "c4_%s_microsphere_hex8_%d" % (statistics, n)
    return Problem(name, mesh, mat, dirichlet_boundaries(mesh, bcs), opts,
                   nodal_forces=nf, element_shear_modulus=Ge)


def config_c5_instance(m: int, mu: float, increments: int = 5) -> Problem:
    """One instance of the batched set: m^3 cubes x 6 tet4, neo-Hooke mu, K = 20 mu, rollers +
    top stretch 1.1 in equal increments."""
    mesh = structured_tet4(m)
    mat = make_material({"shear_modulus": mu, "bulk_modulus": 20.0 * mu}, {"name": "neohooke"})
    bcs = _rollers([{"name": "top", "type": "displacement", "time": [0.0, 1.0], "z": [0.0, 0.1]}])
    dt = 1.0 / increments
    opts = Options(residual_tolerance=1e-8, displacement_tolerance=1e-8, linear_iterations=15,
                   period=1.0, initial=dt, minimum=dt, maximum=dt, adaptive=False,
                   cg_tolerance=1e-10, cg_maximum_iterations=200000)
    return Problem("c5_neohooke_tet4_%d" % m, mesh, mat, dirichlet_boundaries(mesh, bcs), opts)


def config_c5_sizes(count: int = 256, seed: int = 11, lo: int = 8, hi: int = 40):
    """Seeded (cells per side, mu) pairs of the batched workload."""
    rng = np.random.Generator(np.random.PCG64(seed))
    m = rng.integers(lo, hi + 1, size=count)
    mu = rng.uniform(0.5, 2.0, size=count)
    return [(int(a), float(b)) for a, b in zip(m, mu)]
