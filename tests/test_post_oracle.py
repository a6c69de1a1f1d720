"""The oracle's nodal averaging (neon's nodal_averaged_variable + average_internal_variable), on
CPU: extrapolation reproduces trilinear point fields at the corners, and a uniform state
averages to itself."""
import numpy as np

from conftest import random_displacement
from neon_b200 import mesh as M
from neon_b200 import problem as P


def test_extrapolation_recovers_linear_stress_field(oracle):
    m = M.structured_hex8(3, 2, 2, jitter=0.1, seed=4)
    mat = P.make_material({"elastic_modulus": 200e3, "poissons_ratio": 0.3},
                          {"name": "isotropic_linear_elasticity"})
    om = oracle.OracleMesh(m.X, m.conn, mat)
    # a point field that is trilinear in the reference coordinates of every element takes, at
    # each corner, the value of that trilinear field: use sigma = nodal coordinates interpolated
    rng = np.random.Generator(np.random.PCG64(2))
    nodal = rng.standard_normal((m.num_nodes, 9))
    g = 1 / np.sqrt(3)
    lc = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                   [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)
    N = np.prod(1 + (g * lc)[:, None, :] * lc[None, :, :], axis=2) / 8  # [point][corner]
    sig = np.einsum("la,eak->elk", N, nodal[m.conn]).reshape(-1, 9)
    om.set("sigma", sig)
    avg = om.nodal_average("cauchy_stress")
    np.testing.assert_allclose(avg, nodal, rtol=1e-12, atol=1e-12)


def test_uniform_state_averages_to_itself(oracle):
    m = M.structured_tet4(2, 2, 1)
    mat = P.make_material({"shear_modulus": 1.0, "bulk_modulus": 10.0}, {"name": "neohooke"})
    om = oracle.OracleMesh(m.X, m.conn, mat)
    om.update(random_displacement(m, 0.0, 1))
    F = om.nodal_average("DetF")
    np.testing.assert_allclose(F, 1.0, rtol=1e-14)
