"""ctypes binding of the CPU oracle (oracle/neon_oracle.cpp).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline.  The product package (neon_b200) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libneon_oracle.so")

_lib = None


STAMP = os.path.join(HERE, "_build", "cpu.txt")


def _cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name") or line.startswith("flags"):
                    return line.strip()
    except OSError:
        pass
    return "unknown"


def build(force: bool = False):
    """Compile the oracle with its Makefile (g++ -O3 -march=native -fopenmp).  -march=native
    binaries are tied to the host CPU, so a build made on another machine is redone."""
    stale = force or not os.path.exists(STAMP) or open(STAMP).read() != _cpu_model()
    subprocess.run(["make", "-s", "-C", HERE] + (["-B"] if stale else []), check=True)
    with open(STAMP, "w") as fh:
        fh.write(_cpu_model())


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or not os.path.exists(STAMP) or \
                open(STAMP).read() != _cpu_model():
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        L.orc_create.restype = P
        L.orc_create.argtypes = [C.c_int, dp, C.c_int, C.c_int, ip, C.c_int, dp, P]
        L.orc_destroy.argtypes = [P]
        L.orc_ndofs.argtypes = [P]
        L.orc_nnz.argtypes = [P]
        L.orc_nnz.restype = C.c_longlong
        L.orc_pattern.argtypes = [P, ip, ip]
        L.orc_update.argtypes = [P, dp, C.c_char_p, C.c_int]
        L.orc_assemble.argtypes = [P, dp]
        L.orc_internal_force.argtypes = [P, dp]
        L.orc_element_stiffness.argtypes = [P, C.c_int, dp]
        L.orc_save.argtypes = [P, C.c_int]
        L.orc_get_qp.argtypes = [P, C.c_int, dp]
        L.orc_set_qp.argtypes = [P, C.c_int, dp]
        L.orc_nodal_average.argtypes = [P, C.c_int, dp]
        L.orc_nonfollower_load.argtypes = [P, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                           C.c_int, dp]
        L.orc_constitutive_only.argtypes = [P]
        L.orc_cg_solve.argtypes = [C.c_int, ip, ip, dp, dp, dp, C.c_double, C.c_int, C.c_int,
                                   C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.orc_cg_sample.restype = C.c_double
        L.orc_cg_sample.argtypes = [C.c_int, ip, ip, dp, dp, C.c_int, C.c_int,
                                    C.POINTER(C.c_double)]
        L.orc_sphere_rule.argtypes = [C.c_int, dp, dp]
        L.orc_sphere_rule.restype = C.c_int
        L.orc_shape.argtypes = [C.c_int, dp, dp]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_max_threads.restype = C.c_int
        L.orc_static_solve.argtypes = [P, C.c_void_p, C.c_int, ip, ip, ip, dp, dp,
                                       C.c_int, ip, ip, ip, dp, dp, C.c_void_p,
                                       dp, dp, C.c_void_p, dp, C.c_int]
        _lib = L
    return _lib


QP = {"sigma": (0, 9), "D": (1, 36), "detF": (2, 1), "ep": (3, 9), "epbar": (4, 1), "vm": (5, 1),
      "F": (6, 9), "H": (7, 9)}


class OrcOptions(C.Structure):
    _fields_ = [("residual_tolerance", C.c_double), ("displacement_tolerance", C.c_double),
                ("linear_iterations", C.c_int), ("absolute_tolerance", C.c_int),
                ("period", C.c_double), ("initial", C.c_double), ("minimum", C.c_double),
                ("maximum", C.c_double), ("adaptive", C.c_int), ("cg_tolerance", C.c_double),
                ("cg_maximum_iterations", C.c_int), ("use_rcm", C.c_int)]


class OrcReport(C.Structure):
    _fields_ = [("status", C.c_int), ("load_steps", C.c_int),
                ("newton_iterations", C.c_longlong), ("cg_iterations", C.c_longlong),
                ("seconds_assembly", C.c_double), ("seconds_update", C.c_double),
                ("seconds_solve", C.c_double), ("message", C.c_char * 256)]


def sphere_rule(points: int = 21):
    """Directions [n][3] and weights [n] of the BO21 (points=21) or BO33 (points=33) rule."""
    r = np.zeros(33 * 3)
    w = np.zeros(33)
    n = lib().orc_sphere_rule(int(points), r, w)
    return r[:3 * n].reshape(n, 3), w[:n]


def shape(npe: int):
    nq = 8 if npe == 8 else 1
    dN = np.zeros(nq * npe * 3)
    w = np.zeros(nq)
    lib().orc_shape(npe, dN, w)
    return dN.reshape(nq, npe, 3), w


def set_threads(n: int):
    lib().orc_set_threads(int(n))


def max_threads() -> int:
    return int(lib().orc_max_threads())


class OracleMesh:
    """One oracle instance = neon's solid::mesh with one submesh + its internal variables."""

    def __init__(self, X, conn, material, element_shear_modulus=None):
        L = lib()
        self.X = np.ascontiguousarray(X, dtype=np.float64)
        self.conn = np.ascontiguousarray(conn, dtype=np.int32)
        self.N, self.E, self.npe = self.X.shape[0], self.conn.shape[0], self.conn.shape[1]
        self.nq = 8 if self.npe == 8 else 1
        params = np.ascontiguousarray(material.params())
        self._Ge = None
        gp = None
        if element_shear_modulus is not None:
            self._Ge = np.ascontiguousarray(element_shear_modulus, dtype=np.float64)
            gp = self._Ge.ctypes.data
        self.h = L.orc_create(self.N, self.X.reshape(-1), self.E, self.npe, self.conn.reshape(-1),
                              int(material.model), params, gp)
        if not self.h:
            raise ValueError("oracle: unsupported element")
        self.ndofs = L.orc_ndofs(self.h)
        self.nnz = L.orc_nnz(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def pattern(self):
        rp = np.zeros(self.ndofs + 1, np.int32)
        col = np.zeros(self.nnz, np.int32)
        lib().orc_pattern(self.h, rp, col)
        return rp, col

    def update(self, u):
        msg = C.create_string_buffer(256)
        st = lib().orc_update(self.h, np.ascontiguousarray(u, dtype=np.float64), msg, 256)
        return st, msg.value.decode()

    def assemble(self):
        K = np.zeros(self.nnz)
        lib().orc_assemble(self.h, K)
        return K

    def internal_force(self):
        f = np.zeros(self.ndofs)
        lib().orc_internal_force(self.h, f)
        return f

    def element_stiffness(self, e):
        ke = np.zeros((3 * self.npe) ** 2)
        lib().orc_element_stiffness(self.h, int(e), ke)
        return ke.reshape(3 * self.npe, 3 * self.npe)

    def save(self, converged=True):
        lib().orc_save(self.h, int(bool(converged)))

    def get(self, name):
        which, k = QP[name]
        out = np.zeros(self.E * self.nq * k)
        lib().orc_get_qp(self.h, which, out)
        return out.reshape(self.E * self.nq, k) if k > 1 else out

    # submesh::nodal_averaged_variable + average_internal_variable (value / count per node)
    NODAL = {"cauchy_stress": (0, 9), "DetF": (1, 1), "plastic_strain": (2, 9),
             "accumulated_plastic_strain": (3, 1), "von_mises_stress": (4, 1)}

    def nodal_average(self, name):
        which, k = self.NODAL[name]
        out = np.zeros(self.N * k)
        lib().orc_nodal_average(self.h, which, out)
        return out.reshape(self.N, k) if k > 1 else out

    def set(self, name, values):
        which, _ = QP[name]
        lib().orc_set_qp(self.h, which, np.ascontiguousarray(values, dtype=np.float64).reshape(-1))

    def nonfollower_load(self, kind, component=0, faces=None, reduced=False):
        """Unit-load nodal vector of a traction / pressure (faces) or a body force (volume),
        neumann.hpp:69-192 and pressure.cpp:9-37 restated."""
        f = np.zeros(self.ndofs)
        fc = None if faces is None else np.ascontiguousarray(faces, dtype=np.int32)
        nf, npf = (0, 0) if fc is None else fc.shape
        lib().orc_nonfollower_load(self.h, int(kind), int(component),
                                   None if fc is None else fc.ctypes.data, int(nf), int(npf),
                                   int(bool(reduced)), f)
        return f

    def constitutive_only(self):
        return lib().orc_constitutive_only(self.h)


def cg_solve(rowptr, col, val, b, tol, maxit, use_rcm=True):
    """neon's conjugate_gradient::solve restated; returns (status, x, iterations, error)."""
    n = len(rowptr) - 1
    x = np.zeros(n)
    it = C.c_int(0)
    err = C.c_double(0)
    st = lib().orc_cg_solve(n, np.ascontiguousarray(rowptr, np.int32),
                            np.ascontiguousarray(col, np.int32),
                            np.ascontiguousarray(val, np.float64),
                            np.ascontiguousarray(b, np.float64), x, float(tol), int(maxit),
                            int(bool(use_rcm)), C.byref(it), C.byref(err))
    return st, x, it.value, err.value


def cg_sample_seconds(rowptr, col, val, b, iterations, use_rcm=True):
    """Seconds of `iterations` reference PCG iterations (+ P^T A P rebuild when use_rcm)."""
    tp = C.c_double(0)
    s = lib().orc_cg_sample(len(rowptr) - 1, np.ascontiguousarray(rowptr, np.int32),
                            np.ascontiguousarray(col, np.int32),
                            np.ascontiguousarray(val, np.float64),
                            np.ascontiguousarray(b, np.float64), int(iterations),
                            int(bool(use_rcm)), C.byref(tp))
    return s, tp.value


def _pack_tables(tables, weighted=False):
    doff = np.zeros(len(tables) + 1, np.int32)
    poff = np.zeros(len(tables) + 1, np.int32)
    for i, t in enumerate(tables):
        doff[i + 1] = doff[i] + len(t.dofs)
        poff[i + 1] = poff[i] + len(t.times)
    cat = lambda xs, dt: (np.ascontiguousarray(np.concatenate(xs), dt)  # noqa: E731
                          if xs else np.zeros(1, dt))
    dofs = cat([t.dofs for t in tables], np.int32)
    ts = cat([t.times for t in tables], np.float64)
    vs = cat([t.values for t in tables], np.float64)
    w = None
    if weighted:
        w = cat([t.weights if t.weights is not None else np.ones(len(t.dofs)) for t in tables],
                np.float64)
    return doff, dofs, poff, ts, vs, w


def static_solve(problem, max_log=100000):
    """static_matrix<mesh>::solve() on the oracle.  Returns (report dict, u, f_int, log)."""
    m = problem.mesh
    om = OracleMesh(m.X, m.conn, problem.material, problem.element_shear_modulus)
    o = problem.options
    opt = OrcOptions(o.residual_tolerance, o.displacement_tolerance, o.linear_iterations,
                     int(o.absolute_tolerance), o.period, o.initial, o.minimum, o.maximum,
                     int(o.adaptive), o.cg_tolerance, o.cg_maximum_iterations, int(o.use_rcm))
    rep = OrcReport()
    bd = _pack_tables(problem.dirichlet)
    # non-follower loads: the oracle forms their nodal vectors itself
    from neon_b200.problem import load_tables
    forces = list(problem.nodal_forces) + [
        load_tables(sp, om.nonfollower_load(sp.kind, sp.component, sp.faces, sp.reduced))
        for sp in getattr(problem, "loads", [])]
    nf = _pack_tables(forces, weighted=True)
    u = np.zeros(om.ndofs)
    f = np.zeros(om.ndofs)
    log = np.zeros((max_log, 5))
    lib().orc_static_solve(om.h, C.byref(opt), len(problem.dirichlet), bd[0], bd[1], bd[2], bd[3],
                           bd[4], len(forces), nf[0], nf[1], nf[2], nf[3], nf[4],
                           nf[5].ctypes.data if nf[5] is not None else None, u, f, C.byref(rep),
                           log, max_log)
    report = {k: getattr(rep, k) for k, _ in OrcReport._fields_}
    report["message"] = rep.message.decode()
    nlog = min(int(report["newton_iterations"]), max_log)
    return report, u, f, log[:nlog], om
