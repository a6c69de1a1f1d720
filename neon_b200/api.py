"""Python host mirror of neon's interfaces on the solid Newton path, over the C-ABI
(include/neon_b200.h).

* ``Mesh``-level drop-ins: ``SolidMesh`` ~ mechanics::solid::mesh<submesh>
  (update_internal_variables, save_internal_variables, tangent stiffness / internal force
  assembly, sparsity pattern).
* ``ConjugateGradient`` ~ neon's conjugate_gradient linear_solver plugin
  (src/solver/linear/linear_solver.hpp:13-71): ``solve(A, x, b)`` on a CSR matrix.
* ``StaticMatrix`` ~ mechanics::static_matrix (static_matrix.hpp:29-467): ``solve()``.

Errors follow neon: recoverable numerical failures raise ``ComputationalError``
(src/exceptions.hpp:14-17), bad input raises ``ValueError`` (neon's std::domain_error).
The CUDA library must be present: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .problem import Problem

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libneon_b200.so")

OK, E_NEG_DETJ, E_NAN, E_RETURN_MAP, E_CG_MAXIT, E_CG_BREAKDOWN, E_TIMEOUT, E_INPUT, E_CUDA, \
    E_NEWTON_MAXIT, E_CUTBACK_LIMIT = range(11)
RECOVERABLE = {E_NEG_DETJ, E_NAN, E_RETURN_MAP, E_CG_MAXIT, E_CG_BREAKDOWN, E_NEWTON_MAXIT}
FP64, MIXED = 0, 1
# element-pass scatter modes (nb2_set_scatter_mode)
SCATTER_RED, SCATTER_COLOURED = 0, 1


class ComputationalError(RuntimeError):
    """neon::computational_error: a recoverable numerical failure (cutback in static_matrix)."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


class CudaError(RuntimeError):
    """neon::cuda_error."""


class MeshDesc(C.Structure):
    _fields_ = [("num_nodes", C.c_int32), ("coordinates", C.c_void_p),
                ("num_elements", C.c_int32), ("nodes_per_element", C.c_int32),
                ("connectivity", C.c_void_p)]


class MaterialDesc(C.Structure):
    _fields_ = [("model", C.c_int32), ("bulk_modulus", C.c_double),
                ("shear_modulus", C.c_double), ("yield_stress", C.c_double),
                ("isotropic_hardening_modulus", C.c_double),
                ("segments_per_chain", C.c_double),
                ("nonaffine_stretch_parameter", C.c_double),
                ("unit_sphere_points", C.c_int32)]


class DofTableDesc(C.Structure):
    _fields_ = [("dofs", C.c_void_p), ("num_dofs", C.c_int32), ("times", C.c_void_p),
                ("values", C.c_void_p), ("num_points", C.c_int32), ("weights", C.c_void_p)]


class SolverOptions(C.Structure):
    _fields_ = [("residual_tolerance", C.c_double), ("displacement_tolerance", C.c_double),
                ("linear_iterations", C.c_int32), ("absolute_tolerance", C.c_int32),
                ("period", C.c_double), ("initial_increment", C.c_double),
                ("minimum_increment", C.c_double), ("maximum_increment", C.c_double),
                ("adaptive", C.c_int32), ("cg_tolerance", C.c_double),
                ("cg_maximum_iterations", C.c_int32), ("precision", C.c_int32),
                ("mixed_inner_tolerance", C.c_double), ("use_graphs", C.c_int32)]


class SolveReport(C.Structure):
    _fields_ = [("status", C.c_int32), ("load_steps", C.c_int32),
                ("newton_iterations", C.c_int64), ("cg_iterations", C.c_int64),
                ("seconds_total", C.c_double), ("seconds_update_assembly", C.c_double),
                ("seconds_solve", C.c_double), ("message", C.c_char * 256)]


class NewtonLog(C.Structure):
    _fields_ = [("step_time", C.c_double), ("iteration", C.c_int32),
                ("cg_iterations", C.c_int32), ("displacement_norm", C.c_double),
                ("force_norm", C.c_double)]


# symbol -> (restype, argtypes)
P = C.c_void_p
_SIGS = {
    "nb2_create": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(MaterialDesc), C.POINTER(P)]),
    "nb2_destroy": (C.c_int, [P]),
    "nb2_last_error": (C.c_int, [P, C.c_char_p, C.c_size_t]),
    "nb2_set_stream": (C.c_int, [P, P]),
    "nb2_set_scatter_mode": (C.c_int, [P, C.c_int32]),
    "nb2_element_stiffness": (C.c_int, [P, C.c_int64, P]),
    "nb2_get_sizes": (C.c_int, [P, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                C.POINTER(C.c_int64)]),
    "nb2_launch_count": (C.c_int, [P, C.POINTER(C.c_int64)]),
    "nb2_set_element_shear_modulus": (C.c_int, [P, P]),
    "nb2_set_element_moduli": (C.c_int, [P, P, P]),
    "nb2_export_pattern": (C.c_int, [P, P, P]),
    "nb2_update_internal_variables": (C.c_int, [P, P, C.c_double]),
    "nb2_assemble": (C.c_int, [P, P, P]),
    "nb2_save_internal_variables": (C.c_int, [P, C.c_int32]),
    "nb2_apply_tangent": (C.c_int, [P, P, P]),
    "nb2_apply_tangent_fp32": (C.c_int, [P, P, P]),
    "nb2_get_quadrature_values": (C.c_int, [P, C.c_int32, P]),
    "nb2_nodal_averaged_variable": (C.c_int, [P, C.c_int32, P]),
    "nb2_nonfollower_load": (C.c_int, [P, C.c_int32, C.c_int32, P, C.c_int32, C.c_int32,
                                       C.c_int32, P]),
    "nb2_apply_dirichlet": (C.c_int, [P, P, C.c_int32, P, P]),
    "nb2_pcg_solve": (C.c_int, [C.c_int32, P, P, P, P, P, C.c_double, C.c_int32,
                                C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "nb2_static_solve": (C.c_int, [P, C.POINTER(SolverOptions), P, C.c_int32, P, C.c_int32, P,
                                   C.POINTER(SolveReport), P, C.c_int32]),
    "nb2_set_displacement": (C.c_int, [P, P]),
    "nb2_get_displacement": (C.c_int, [P, P]),
    "nb2_update_assemble_device": (C.c_int, [P, C.c_int32]),
    "nb2_download_system": (C.c_int, [P, P, P]),
    "nb2_synchronize": (C.c_int, [P]),
    "nb2_set_dirichlet_mask": (C.c_int, [P, P, C.c_int32]),
    "nb2_solve_device": (C.c_int, [P, C.c_int32, C.c_double, C.c_int32, C.POINTER(C.c_int32),
                                   C.POINTER(C.c_double)]),
    "nb2_adjoint_shear_gradient": (C.c_int, [P, P, C.c_int32, C.c_double, C.c_int32, P,
                                             C.POINTER(C.c_int32)]),
    "nb2_pcg_solve_noalloc": (C.c_int, [C.c_int32, P, P, P, P, P, C.c_double, C.c_int32, P,
                                        C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "nb2_probe_fma_throughput": (C.c_int, [C.c_int32, C.POINTER(C.c_double)]),
    "nb2_batch_static_solve": (C.c_int, [P, C.c_int32, P, C.POINTER(SolverOptions), P, P, P, P,
                                         P, P, P, C.c_int32]),
    "nb2_batch_autotune": (C.c_int, [P, C.c_int32, P, C.c_int32, C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
}

_lib = None


def lib():
    """Load the in-tree CUDA library; raise if it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"neon_b200 CUDA library not built: {LIB_PATH} "
                               "(run python -m neon_b200.build)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def _check(status, ctx=None, what=""):
    if status == OK:
        return
    buf = C.create_string_buffer(512)
    lib().nb2_last_error(ctx, buf, 512)
    msg = f"{what}: {buf.value.decode()} (status {status})"
    if status in RECOVERABLE:
        raise ComputationalError(status, msg)
    if status == E_INPUT:
        raise ValueError(msg)
    raise CudaError(msg)


class SolidMesh:
    """Device-resident mesh + internal variables (neon's solid::mesh with one submesh)."""

    def __init__(self, X, conn, material, element_shear_modulus=None):
        L = lib()
        self.X = np.ascontiguousarray(X, dtype=np.float64)
        self.conn = np.ascontiguousarray(conn, dtype=np.int32)
        self.material = material
        desc = MeshDesc(self.X.shape[0], self.X.ctypes.data, self.conn.shape[0],
                        self.conn.shape[1], self.conn.ctypes.data)
        mat = MaterialDesc(int(material.model), material.K, material.G, material.yield_stress,
                           material.hardening, material.segments_per_chain,
                           material.nonaffine_stretch_parameter, material.unit_sphere_points)
        h = P()
        _check(L.nb2_create(C.byref(desc), C.byref(mat), C.byref(h)), None, "nb2_create")
        self.h = h
        n = C.c_int32()
        nnz = C.c_int64()
        nb = C.c_int64()
        L.nb2_get_sizes(self.h, C.byref(n), C.byref(nnz), C.byref(nb))
        self.ndofs, self.nnz, self.nnzb = n.value, nnz.value, nb.value
        self.nq = 8 if self.conn.shape[1] == 8 else 1
        self.nqp = self.conn.shape[0] * self.nq
        if element_shear_modulus is not None:
            g = np.ascontiguousarray(element_shear_modulus, dtype=np.float64)
            _check(L.nb2_set_element_shear_modulus(self.h, g.ctypes.data), self.h, "shear")

    def set_element_moduli(self, bulk_modulus=None, shear_modulus=None):
        """Per-element K and G ([num_elements] each, either may be None) in place of the
        material's (linear elasticity, neo-Hooke, microsphere)."""
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                for a in (bulk_modulus, shear_modulus)]
        ptr = [None if a is None else a.ctypes.data for a in arrs]
        _check(lib().nb2_set_element_moduli(self.h, ptr[0], ptr[1]), self.h, "moduli")

    def close(self):
        if getattr(self, "h", None):
            lib().nb2_destroy(self.h)
            self.h = None

    def __del__(self):
        # at interpreter exit the module globals (lib, _lib) may already be gone
        try:
            self.close()
        except (TypeError, AttributeError):
            pass

    # --- neon mesh / submesh API -----------------------------------------------------------
    def sparsity_pattern(self):
        rp = np.zeros(self.ndofs + 1, np.int32)
        col = np.zeros(self.nnz, np.int32)
        _check(lib().nb2_export_pattern(self.h, rp.ctypes.data, col.ctypes.data), self.h,
               "pattern")
        return rp, col

    def update_internal_variables(self, u, time_step_size=0.0):
        u = np.ascontiguousarray(u, dtype=np.float64)
        _check(lib().nb2_update_internal_variables(self.h, u.ctypes.data, time_step_size),
               self.h, "update_internal_variables")

    def assemble(self):
        """(K values in neon CSR order, f_int) from the last update."""
        K = np.zeros(self.nnz)
        f = np.zeros(self.ndofs)
        _check(lib().nb2_assemble(self.h, K.ctypes.data, f.ctypes.data), self.h, "assemble")
        return K, f

    def apply_tangent(self, v):
        """K v, matrix-free, with the tangent of the last update."""
        v = np.ascontiguousarray(v, dtype=np.float64)
        y = np.zeros(self.ndofs)
        _check(lib().nb2_apply_tangent(self.h, v.ctypes.data, y.ctypes.data), self.h, "apply")
        return y

    def apply_tangent_fp32(self, v):
        """K v with the FP32 matrix-free operator of the mixed-precision PCG."""
        v = np.ascontiguousarray(v, dtype=np.float64)
        y = np.zeros(self.ndofs)
        _check(lib().nb2_apply_tangent_fp32(self.h, v.ctypes.data, y.ctypes.data), self.h,
               "apply_tangent_fp32")
        return y

    def save_internal_variables(self, converged: bool):
        _check(lib().nb2_save_internal_variables(self.h, int(bool(converged))), self.h, "save")

    def quadrature_values(self, which: str):
        idx = {"cauchy_stress": 0, "DetF": 1, "plastic_strain": 2,
               "accumulated_plastic_strain": 3}[which]
        k = 9 if idx in (0, 2) else 1
        out = np.zeros(self.nqp * k)
        _check(lib().nb2_get_quadrature_values(self.h, idx, out.ctypes.data), self.h, which)
        return out.reshape(self.nqp, k) if k > 1 else out

    NODAL = {"cauchy_stress": (0, 9), "DetF": (1, 1), "plastic_strain": (2, 9),
             "accumulated_plastic_strain": (3, 1), "von_mises_stress": (4, 1)}

    def nodal_averaged(self, which: str):
        """A quadrature variable extrapolated to the nodes and averaged (neon's output fields)."""
        idx, k = self.NODAL[which]
        out = np.zeros(self.X.shape[0] * k)
        _check(lib().nb2_nodal_averaged_variable(self.h, idx, out.ctypes.data), self.h, which)
        return out.reshape(-1, k) if k > 1 else out

    def nonfollower_load(self, kind, component=0, faces=None, reduced=False):
        """The nodal vector [3N] per unit value of a traction / pressure on boundary faces or of
        a body force over the elements, computed on the device (nb2_nonfollower_load)."""
        out = np.zeros(self.ndofs)
        fc = None if faces is None else np.ascontiguousarray(faces, dtype=np.int32)
        nf, npf = (0, 0) if fc is None else (fc.shape[0], fc.shape[1])
        _check(lib().nb2_nonfollower_load(self.h, int(kind), int(component), _ptr(fc), nf, npf,
                                          int(bool(reduced)), out.ctypes.data), self.h,
               "nonfollower_load")
        return out

    def apply_dirichlet(self, dofs, K, b):
        dofs = np.ascontiguousarray(dofs, dtype=np.int32)
        _check(lib().nb2_apply_dirichlet(self.h, dofs.ctypes.data, len(dofs), K.ctypes.data,
                                         b.ctypes.data), self.h, "apply_dirichlet")

    # --- device-resident stepping ----------------------------------------------------------
    def set_displacement(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        _check(lib().nb2_set_displacement(self.h, u.ctypes.data), self.h, "set_displacement")

    def displacement(self):
        u = np.zeros(self.ndofs)
        _check(lib().nb2_get_displacement(self.h, u.ctypes.data), self.h, "get_displacement")
        return u

    def update_assemble_device(self, precision=FP64):
        _check(lib().nb2_update_assemble_device(self.h, int(precision)), self.h, "assemble")

    def download_system(self, K=True, f=True):
        Kv = np.zeros(self.nnz) if K else None
        fv = np.zeros(self.ndofs) if f else None
        _check(lib().nb2_download_system(self.h, _ptr(Kv), _ptr(fv)), self.h, "download")
        return Kv, fv

    def synchronize(self):
        _check(lib().nb2_synchronize(self.h), self.h, "synchronize")

    def set_dirichlet_mask(self, dofs):
        dofs = np.ascontiguousarray(dofs, dtype=np.int32)
        _check(lib().nb2_set_dirichlet_mask(self.h, dofs.ctypes.data, len(dofs)), self.h, "mask")

    def solve_device(self, precision=FP64, tolerance=0.0, maximum_iterations=100):
        it = C.c_int32()
        err = C.c_double()
        _check(lib().nb2_solve_device(self.h, int(precision), float(tolerance),
                                      int(maximum_iterations), C.byref(it), C.byref(err)),
               self.h, "solve_device")
        return it.value, err.value

    def element_stiffness(self, e: int):
        """submesh::tangent_stiffness(e): element e's dense tangent [3 npe][3 npe] at the state
        of the last update_internal_variables (neon's local DOF order 3a + k)."""
        nd = 3 * self.conn.shape[1]
        out = np.zeros((nd, nd))
        _check(lib().nb2_element_stiffness(self.h, int(e), out.ctypes.data), self.h,
               "element_stiffness")
        return out

    def set_scatter_mode(self, mode: int):
        """SCATTER_RED (fast, run-to-run last-bit differences) or SCATTER_COLOURED (one launch
        per element colour, bit-reproducible) for this mesh's update / assembly calls; the
        Newton driver always uses the coloured scatter."""
        _check(lib().nb2_set_scatter_mode(self.h, int(mode)), self.h, "set_scatter_mode")

    def set_stream(self, stream_handle: int):
        _check(lib().nb2_set_stream(self.h, stream_handle), self.h, "set_stream")

    def adjoint_shear_gradient(self, dJdu, precision=FP64, tolerance=1e-12,
                               maximum_iterations=200000):
        """dJ/dG_e at the equilibrium of the last StaticMatrix.solve on this mesh."""
        g = np.ascontiguousarray(dJdu, dtype=np.float64)
        out = np.zeros(self.conn.shape[0])
        it = C.c_int32()
        _check(lib().nb2_adjoint_shear_gradient(self.h, g.ctypes.data, int(precision),
                                                float(tolerance), int(maximum_iterations),
                                                out.ctypes.data, C.byref(it)), self.h, "adjoint")
        self.adjoint_iterations = it.value
        return out

    def launches(self) -> int:
        v = C.c_int64()
        lib().nb2_launch_count(self.h, C.byref(v))
        return v.value


def probe_fma_throughput(fp64: bool = True) -> float:
    """Measured CUDA-core FMA throughput of device 0 in FLOP/s (2 per FMA)."""
    v = C.c_double()
    _check(lib().nb2_probe_fma_throughput(int(bool(fp64)), C.byref(v)), None, "probe")
    return v.value


class ConjugateGradient:
    """neon's conjugate_gradient linear_solver (tolerance, maximum_iterations) on the device."""

    def __init__(self, tolerance=1e-5, maximum_iterations=2000):
        self.tolerance = float(tolerance)
        self.maximum_iterations = int(maximum_iterations)
        self.iterations = 0
        self.error = 0.0

    def solve(self, A, x, b):
        """A: scipy CSR (or (indptr, indices, data)); x is overwritten with the solution."""
        if hasattr(A, "indptr"):
            rp, ci, v = A.indptr, A.indices, A.data
        else:
            rp, ci, v = A
        rp = np.ascontiguousarray(rp, np.int32)
        ci = np.ascontiguousarray(ci, np.int32)
        v = np.ascontiguousarray(v, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        out = np.zeros(len(rp) - 1)
        it = C.c_int32()
        err = C.c_double()
        st = lib().nb2_pcg_solve(len(rp) - 1, rp.ctypes.data, ci.ctypes.data, v.ctypes.data,
                                 b.ctypes.data, out.ctypes.data, self.tolerance,
                                 self.maximum_iterations, C.byref(it), C.byref(err))
        self.iterations, self.error = it.value, err.value
        x[...] = out
        if st == E_CG_MAXIT:
            raise ComputationalError(st, "Conjugate gradient solver maximum iterations reached")
        if st == E_NAN:
            raise ComputationalError(st, "Floating point error reported")
        _check(st, None, "pcg")
        return x


def _tables(tables, keep):
    descs = (DofTableDesc * max(1, len(tables)))()
    for i, t in enumerate(tables):
        d = np.ascontiguousarray(t.dofs, np.int32)
        tt = np.ascontiguousarray(t.times, np.float64)
        vv = np.ascontiguousarray(t.values, np.float64)
        w = None if t.weights is None else np.ascontiguousarray(t.weights, np.float64)
        keep += [d, tt, vv, w]
        descs[i] = DofTableDesc(d.ctypes.data, len(d), tt.ctypes.data, vv.ctypes.data, len(tt),
                                _ptr(w))
    return descs


class StaticMatrix:
    """mechanics::static_matrix: full Newton with adaptive load stepping on the device."""

    def __init__(self, problem: Problem, precision=FP64, mixed_inner_tolerance=1e-2,
                 use_graphs=True, mesh: SolidMesh | None = None):
        self.problem = problem
        m = problem.mesh
        self.mesh = mesh or SolidMesh(m.X, m.conn, problem.material,
                                      problem.element_shear_modulus)
        o = problem.options
        self.options = SolverOptions(o.residual_tolerance, o.displacement_tolerance,
                                     o.linear_iterations, int(o.absolute_tolerance), o.period,
                                     o.initial, o.minimum, o.maximum, int(o.adaptive),
                                     o.cg_tolerance, o.cg_maximum_iterations, int(precision),
                                     mixed_inner_tolerance, int(bool(use_graphs)))
        self.report = None
        self.log = None
        self.displacement = None

    def external_force_tables(self):
        """The problem's nodal-force tables plus its non-follower loads, their nodal vectors
        computed on the device."""
        from .problem import load_tables
        tables = list(self.problem.nodal_forces)
        for spec in self.problem.loads:
            f = self.mesh.nonfollower_load(spec.kind, spec.component, spec.faces, spec.reduced)
            tables.append(load_tables(spec, f))
        return tables

    def solve(self, max_log=100000, raise_on_error=True):
        keep = []
        dt = _tables(self.problem.dirichlet, keep)
        forces = self.external_force_tables()
        nf = _tables(forces, keep)
        u = np.zeros(self.mesh.ndofs)
        rep = SolveReport()
        log = (NewtonLog * max_log)()
        st = lib().nb2_static_solve(self.mesh.h, C.byref(self.options), C.cast(dt, P),
                                    len(self.problem.dirichlet), C.cast(nf, P),
                                    len(forces), u.ctypes.data, C.byref(rep),
                                    C.cast(log, P), max_log)
        self.displacement = u
        self.report = {k: getattr(rep, k) for k, _ in SolveReport._fields_}
        self.report["message"] = rep.message.decode()
        n = min(int(rep.newton_iterations), max_log)
        self.log = np.array([[log[i].step_time, log[i].iteration, log[i].cg_iterations,
                              log[i].displacement_norm, log[i].force_norm] for i in range(n)])
        if raise_on_error and st != OK:
            if st in RECOVERABLE or st == E_CUTBACK_LIMIT:
                raise ComputationalError(st, self.report["message"])
            _check(st, self.mesh.h, "static_solve")
        return u


def batch_layout(problems):
    """The block-diagonal mesh of a batch: concatenated coordinates, connectivity shifted by each
    instance's node offset, per-element K and G, and every boundary table with its DOFs shifted
    to the global numbering (tables of instance i at [offsets[i], offsets[i+1]))."""
    if not problems:
        raise ValueError("no problems")
    model = problems[0].material.model
    npe = problems[0].mesh.conn.shape[1]
    for pr in problems:
        if pr.material.model != model or pr.mesh.conn.shape[1] != npe:
            raise ValueError("batched problems share one model and one element type")
    node_offsets = np.zeros(len(problems) + 1, np.int32)
    Xs, conns, Ks, Gs = [], [], [], []
    tables = {"dirichlet": ([], [0]), "nodal_forces": ([], [0])}
    for i, pr in enumerate(problems):
        off = int(node_offsets[i])
        Xs.append(pr.mesh.X)
        conns.append(pr.mesh.conn + off)
        E = pr.mesh.conn.shape[0]
        Ks.append(np.full(E, pr.material.K))
        Gs.append(pr.element_shear_modulus if pr.element_shear_modulus is not None
                  else np.full(E, pr.material.G))
        node_offsets[i + 1] = off + pr.mesh.num_nodes
        for which, (lst, offs) in tables.items():
            for t in getattr(pr, which):
                lst.append(type(t)(np.asarray(t.dofs, np.int64) + 3 * off, t.times, t.values,
                                   t.weights, t.name))
            offs.append(len(lst))
    if 3 * int(node_offsets[-1]) >= 2 ** 31:
        raise ValueError("the batch has more DOFs than int32 indices address")
    return {"X": np.concatenate(Xs), "conn": np.concatenate(conns).astype(np.int32),
            "K": np.concatenate(Ks), "G": np.concatenate(Gs), "node_offsets": node_offsets,
            "element_offsets": np.concatenate([[0], np.cumsum([c.shape[0] for c in conns])]),
            "dirichlet": tables["dirichlet"][0],
            "dirichlet_offsets": np.asarray(tables["dirichlet"][1], np.int32),
            "nodal_forces": tables["nodal_forces"][0],
            "force_offsets": np.asarray(tables["nodal_forces"][1], np.int32)}


class BatchedStaticMatrix:
    """Many independent static_matrix solves of uneven size in one context: the instances'
    meshes are concatenated into one block-diagonal mesh, each instance keeps its own material
    (per-element moduli), boundary tables, load stepping, Newton decisions and PCG.  All problems
    share one constitutive model and one set of solver options (those of the first problem)."""

    def __init__(self, problems, precision=FP64, mixed_inner_tolerance=1e-2, use_graphs=True,
                 autotune=True):
        self.problems = list(problems)
        self.layout = batch_layout(self.problems)
        lay = self.layout
        self.node_offsets = lay["node_offsets"]
        self.element_offsets = lay["element_offsets"]
        self.mesh = SolidMesh(lay["X"], lay["conn"], self.problems[0].material)
        self.mesh.set_element_moduli(lay["K"], lay["G"])
        o = problems[0].options
        self.options = SolverOptions(o.residual_tolerance, o.displacement_tolerance,
                                     o.linear_iterations, int(o.absolute_tolerance), o.period,
                                     o.initial, o.minimum, o.maximum, int(o.adaptive),
                                     o.cg_tolerance, o.cg_maximum_iterations, int(precision),
                                     mixed_inner_tolerance, int(bool(use_graphs)))
        self.precision = precision
        self.tuned = None
        if autotune:
            self.autotune()
        self.reports = None
        self.logs = None
        self.displacement = None

    @property
    def num_instances(self):
        return len(self.problems)

    def autotune(self):
        """Pick the batched PCG's rows per chunk and lanes per block row by timing."""
        R, L, ms = C.c_int32(), C.c_int32(), C.c_double()
        _check(lib().nb2_batch_autotune(self.mesh.h, self.num_instances,
                                        self.node_offsets.ctypes.data, int(self.precision),
                                        C.byref(R), C.byref(L), C.byref(ms)), self.mesh.h,
               "autotune")
        self.tuned = {"rows_per_chunk": R.value, "lanes_per_row": L.value, "ms_per_spmv": ms.value}
        return self.tuned

    def solve(self, max_log=64, raise_on_error=True):
        keep = []
        lay = self.layout
        dir_t, dir_off = lay["dirichlet"], lay["dirichlet_offsets"]
        frc_t, frc_off = lay["nodal_forces"], lay["force_offsets"]
        dt = _tables(dir_t, keep)
        nf = _tables(frc_t, keep)
        n = self.num_instances
        u = np.zeros(self.mesh.ndofs)
        reps = (SolveReport * n)()
        log = (NewtonLog * (n * max_log))()
        st = lib().nb2_batch_static_solve(self.mesh.h, n, self.node_offsets.ctypes.data,
                                          C.byref(self.options), C.cast(dt, P),
                                          dir_off.ctypes.data, C.cast(nf, P), frc_off.ctypes.data,
                                          u.ctypes.data, C.cast(reps, P), C.cast(log, P), max_log)
        self.displacement = u
        self.reports = []
        self.logs = []
        for i in range(n):
            r = {k: getattr(reps[i], k) for k, _ in SolveReport._fields_}
            r["message"] = reps[i].message.decode()
            self.reports.append(r)
            m = min(int(r["newton_iterations"]), max_log)
            self.logs.append(np.array([[log[i * max_log + j].step_time,
                                        log[i * max_log + j].iteration,
                                        log[i * max_log + j].cg_iterations,
                                        log[i * max_log + j].displacement_norm,
                                        log[i * max_log + j].force_norm] for j in range(m)]))
        if raise_on_error and st != OK:
            if st in RECOVERABLE or st == E_CUTBACK_LIMIT:
                bad = [i for i, r in enumerate(self.reports) if r["status"] != OK]
                raise ComputationalError(st, "instance %s: %s" % (
                    bad[:1], self.reports[bad[0]]["message"] if bad else ""))
            _check(st, self.mesh.h, "batch_static_solve")
        return u

    def instance_displacement(self, i, u=None):
        u = self.displacement if u is None else u
        return u[3 * self.node_offsets[i]:3 * self.node_offsets[i + 1]]
