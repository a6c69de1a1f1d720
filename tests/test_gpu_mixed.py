"""The pieces of the mixed-precision path: the matrix-free FP64 tangent product (the defect
residual) equals the assembled K times v, and the FP32-bulk Newton reaches the FP64 device
solution on problems without path dependence (neo-Hooke, linear elasticity)."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import random_displacement, rel_err
from neon_b200 import mesh as M
from neon_b200 import problem as P
from test_gpu_parity import FIELD_MODELS, MATERIALS, SCALE

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from neon_b200 import api, build
    build.build()
    return api


@pytest.mark.parametrize("topo", ["hex8", "tet4"])
@pytest.mark.parametrize("model", list(MATERIALS))
def test_matrix_free_tangent_equals_assembled(api, topo, model):
    m = M.structured_hex8(4, 3, 3, jitter=0.1, seed=3) if topo == "hex8" else \
        M.structured_tet4(3, 2, 2)
    Ge = None
    if model in FIELD_MODELS:
        Ge = np.random.Generator(np.random.PCG64(5)).lognormal(0.0, 0.3, m.num_elements)
    g = api.SolidMesh(m.X, m.conn, MATERIALS[model], Ge)
    g.update_internal_variables(random_displacement(m, SCALE[model], 11))
    K, _ = g.assemble()
    rp, col = g.sparsity_pattern()
    A = sp.csr_matrix((K, col, rp), shape=(g.ndofs, g.ndofs))
    v = np.random.Generator(np.random.PCG64(9)).standard_normal(g.ndofs)
    assert rel_err(g.apply_tangent(v), A @ v) < 1e-12


@pytest.mark.parametrize("make", [lambda: P.config_c1(6), lambda: P.config_c2(5, increments=3),
                                  lambda: P.config_c4(4), lambda: P.config_c5_instance(3, 1.3),
                                  lambda: P.config_c4(4, traction=0.2, statistics="langevin",
                                                      segments_per_chain=5),
                                  lambda: P.config_c4(4, traction=0.2, statistics="nonaffine",
                                                      segments_per_chain=5,
                                                      nonaffine_stretch_parameter=1.5)],
                         ids=["c1_le_hex8", "c2_nh_hex8", "c4_microsphere_hex8", "c5_nh_tet4",
                              "c4_langevin_hex8", "c4_nonaffine_hex8"])
def test_mixed_newton_reaches_fp64_solution(api, make):
    pr = make()
    pr.options.residual_tolerance = pr.options.displacement_tolerance = 1e-10
    u64 = api.StaticMatrix(pr).solve()
    u32 = api.StaticMatrix(pr, precision=api.MIXED, mixed_inner_tolerance=1e-4).solve()
    assert rel_err(u32, u64) < 1e-9


@pytest.mark.parametrize("topo", ["hex8", "tet4"])
@pytest.mark.parametrize("model", list(MATERIALS))
def test_fp32_matrix_free_tangent(api, topo, model):
    """The FP32 operator of the mixed PCG equals the assembled FP64 K v to FP32 rounding."""
    m = M.structured_hex8(4, 3, 3, jitter=0.1, seed=3) if topo == "hex8" else \
        M.structured_tet4(3, 2, 2)
    g = api.SolidMesh(m.X, m.conn, MATERIALS[model])
    g.update_internal_variables(random_displacement(m, SCALE[model], 11))
    K, _ = g.assemble()
    rp, col = g.sparsity_pattern()
    A = sp.csr_matrix((K, col, rp), shape=(g.ndofs, g.ndofs))
    v = np.random.Generator(np.random.PCG64(9)).standard_normal(g.ndofs)
    y = g.apply_tangent_fp32(v)
    assert rel_err(y, A @ v) < 2e-5
    # the Jacobi diagonal it forms is the assembled diagonal (checked through e_i products)
    e = np.zeros(g.ndofs)
    e[7] = 1.0
    assert abs(g.apply_tangent_fp32(e)[7] - A[7, 7]) <= 1e-5 * abs(A[7, 7])
