"""Parity of the sm_100a path (through the C-ABI) with the CPU oracle on the same seeded inputs.

Bars: CSR pattern and DOF numbering bit-exact; K, f_int and the quadrature-point state within
1e-12 relative (FP64); Newton solutions within 1e-10 relative (both Newton loops converge to the
same equilibrium with CG at rtol 1e-10, so the remaining difference is CG round-off amplified by
the conditioning); the mixed-precision path within 1e-8 of the FP64 device path.
"""
import numpy as np
import pytest

from conftest import cube_example_problem, random_displacement, rel_err
from neon_b200 import mesh as M
from neon_b200 import problem as P

pytestmark = pytest.mark.gpu

TOL_K = 1e-12


@pytest.fixture(scope="module")
def api():
    from neon_b200 import api, build
    build.build()
    api.lib()
    return api


MATERIALS = {
    "linear_elastic": P.make_material({"elastic_modulus": 200e3, "poissons_ratio": 0.3},
                                      {"name": "isotropic_linear_elasticity"}),
    "neohooke": P.make_material({"shear_modulus": 1.0, "bulk_modulus": 10.0},
                                {"name": "neohooke"}),
    "j2": P.make_material({"elastic_modulus": 200e3, "poissons_ratio": 0.3, "yield_stress": 200.0,
                           "isotropic_hardening_modulus": 1e3},
                          {"name": "J2_plasticity", "finite_strain": False}),
    "microsphere": P.make_material({"bulk_modulus": 100.0, "shear_modulus": 1.0,
                                    "segments_per_chain": 50},
                                   {"name": "microsphere", "type": "affine",
                                    "statistics": "gaussian", "quadrature": "BO21"}),
    # short chains (5 segments) so the Langevin terms are far from the Gaussian limit
    "langevin": P.make_material({"bulk_modulus": 100.0, "shear_modulus": 1.0,
                                 "segments_per_chain": 5},
                                {"name": "microsphere", "type": "affine",
                                 "statistics": "langevin", "quadrature": "BO21"}),
    "nonaffine": P.make_material({"bulk_modulus": 100.0, "shear_modulus": 1.0,
                                  "segments_per_chain": 5, "nonaffine_stretch_parameter": 1.5},
                                 {"name": "microsphere", "type": "nonaffine",
                                  "quadrature": "BO21"}),
    # the 33-point unit-sphere rule on the affine and on the anisotropic tangent path
    "microsphere_bo33": P.make_material({"bulk_modulus": 100.0, "shear_modulus": 1.0,
                                         "segments_per_chain": 50},
                                        {"name": "microsphere", "type": "affine",
                                         "statistics": "gaussian", "quadrature": "BO33"}),
    "nonaffine_bo33": P.make_material({"bulk_modulus": 100.0, "shear_modulus": 1.0,
                                       "segments_per_chain": 5,
                                       "nonaffine_stretch_parameter": 1.5},
                                      {"name": "microsphere", "type": "nonaffine",
                                       "quadrature": "BO33"}),
}
# displacement amplitudes that keep det F > 0 and put J2 points in the plastic range
SCALE = {"linear_elastic": 1e-3, "neohooke": 0.02, "j2": 4e-3, "microsphere": 0.02,
         "langevin": 0.03, "nonaffine": 0.03, "microsphere_bo33": 0.02, "nonaffine_bo33": 0.03}
# models with a per-element shear modulus field in the tests
FIELD_MODELS = ("microsphere", "langevin", "nonaffine", "microsphere_bo33", "nonaffine_bo33")


def _meshes():
    return {"hex8": M.structured_hex8(5, 4, 3, jitter=0.1, seed=3),
            "tet4": M.structured_tet4(3, 2, 3)}


@pytest.mark.parametrize("topo", ["hex8", "tet4"])
def test_pattern_bit_exact(api, oracle, topo):
    m = _meshes()[topo]
    g = api.SolidMesh(m.X, m.conn, MATERIALS["linear_elastic"])
    om = oracle.OracleMesh(m.X, m.conn, MATERIALS["linear_elastic"])
    rp, col = g.sparsity_pattern()
    orp, ocol = om.pattern()
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)


def test_pattern_bit_exact_full_size_c1(api, oracle):
    pr = P.config_c1(20)
    g = api.SolidMesh(pr.mesh.X, pr.mesh.conn, pr.material)
    om = oracle.OracleMesh(pr.mesh.X, pr.mesh.conn, pr.material)
    assert g.nnz == om.nnz == 2042829
    rp, col = g.sparsity_pattern()
    orp, ocol = om.pattern()
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)


@pytest.mark.parametrize("topo", ["hex8", "tet4"])
@pytest.mark.parametrize("model", list(MATERIALS))
def test_update_and_assembly_parity(api, oracle, topo, model):
    m = _meshes()[topo]
    mat = MATERIALS[model]
    Ge = None
    if model in FIELD_MODELS:
        Ge = np.random.Generator(np.random.PCG64(5)).lognormal(0.0, 0.3, m.num_elements)
    g = api.SolidMesh(m.X, m.conn, mat, Ge)
    om = oracle.OracleMesh(m.X, m.conn, mat, Ge)
    for it, seed in enumerate((11, 12)):  # two updates: J2 state carries over
        u = random_displacement(m, SCALE[model], seed) * (1 + it)
        st, msg = om.update(u)
        assert st == 0, msg
        g.update_internal_variables(u)
        K, f = g.assemble()
        Ko = om.assemble()
        fo = om.internal_force()
        assert rel_err(K, Ko) < TOL_K
        assert rel_err(f, fo) < TOL_K
        sig = g.quadrature_values("cauchy_stress")
        assert rel_err(sig, om.get("sigma")) < TOL_K
        assert rel_err(g.quadrature_values("DetF"), om.get("detF")) < TOL_K
        if model == "j2":
            assert om.get("epbar").max() > 0  # the case is plastic
            assert rel_err(g.quadrature_values("plastic_strain"), om.get("ep")) < TOL_K
            assert rel_err(g.quadrature_values("accumulated_plastic_strain"),
                           om.get("epbar")) < TOL_K


def test_commit_revert(api, oracle):
    m = M.structured_hex8(3)
    mat = MATERIALS["j2"]
    g = api.SolidMesh(m.X, m.conn, mat)
    u1 = random_displacement(m, 4e-3, 1)
    g.update_internal_variables(u1)
    g.save_internal_variables(True)
    ep1 = g.quadrature_values("accumulated_plastic_strain").copy()
    g.update_internal_variables(2 * u1)
    assert g.quadrature_values("accumulated_plastic_strain").max() > ep1.max()
    g.save_internal_variables(False)
    g.update_internal_variables(u1)
    # reverted state + same u: the return map from the committed state is (nearly) elastic
    assert rel_err(g.quadrature_values("accumulated_plastic_strain"), ep1) < 1e-6


def test_dirichlet_application_parity(api):
    pr = P.config_c1(4)
    g = api.SolidMesh(pr.mesh.X, pr.mesh.conn, pr.material)
    g.update_internal_variables(np.zeros(g.ndofs))
    K, f = g.assemble()
    dofs = np.concatenate([t.dofs for t in pr.dirichlet])
    b = np.ones(g.ndofs)
    K2, b2 = K.copy(), b.copy()
    g.apply_dirichlet(dofs, K2, b2)
    import scipy.sparse as sp
    rp, col = g.sparsity_pattern()
    A = sp.csr_matrix((K, col, rp)).toarray()
    A2 = sp.csr_matrix((K2, col, rp)).toarray()
    ref = A.copy()
    ref[dofs, :] = 0
    ref[:, dofs] = 0
    ref[dofs, dofs] = A[dofs, dofs]
    assert np.array_equal(A2, ref)
    assert np.all(b2[dofs] == 0) and np.all(np.delete(b2, dofs) == 1)


def test_pcg_three_by_three_kat(api, kats):
    k = kats["cg_3x3"]
    rp = np.array([0, 3, 6, 9], np.int32)
    col = np.tile(np.arange(3, dtype=np.int32), 3)
    val = np.zeros(9)
    for i, j, v in k["triplets"]:
        val[3 * i + j] = v
    for tol in (1e-5, 1e-12):
        x = np.zeros(3)
        api.ConjugateGradient(tol, 2000).solve((rp, col, val), x, np.array(k["b"]))
        np.testing.assert_allclose(x, k["x"], atol=k["margin"])


def test_pcg_matches_reference_algorithm(api, oracle):
    pr = P.config_c1(8)
    om = oracle.OracleMesh(pr.mesh.X, pr.mesh.conn, pr.material)
    om.update(random_displacement(pr.mesh, 1e-4, 2))
    K = om.assemble()
    rp, col = om.pattern()
    rng = np.random.Generator(np.random.PCG64(4))
    b = rng.standard_normal(om.ndofs)
    # SPD: fix the first face so K is nonsingular
    g = api.SolidMesh(pr.mesh.X, pr.mesh.conn, pr.material)
    dofs = np.concatenate([t.dofs for t in pr.dirichlet])
    g.apply_dirichlet(dofs, K, b)
    st, xo, ito, erro = oracle.cg_solve(rp, col, K, b, 1e-12, 20000, use_rcm=False)
    assert st == 0
    cg = api.ConjugateGradient(1e-12, 20000)
    x = np.zeros(om.ndofs)
    cg.solve((rp, col, K), x, b)
    assert abs(cg.iterations - ito) <= max(2, 0.02 * ito)
    assert rel_err(x, xo) < 1e-9
    with pytest.raises(api.ComputationalError):
        api.ConjugateGradient(1e-12, 5).solve((rp, col, K), x, b)


def _solve_both(api, oracle, pr, **kw):
    rep_o, u_o, f_o, log_o, _ = oracle.static_solve(pr)
    sm = api.StaticMatrix(pr, **kw)
    u = sm.solve()
    return rep_o, u_o, log_o, sm, u


@pytest.mark.parametrize("name,make", [
    ("c1_linear_elastic", lambda: P.config_c1(6)),
    ("c2_neohooke_jitter", lambda: P.config_c2(5, increments=3)),
    ("c3_j2_cyclic", lambda: P.config_c3(4, steps=20)),
    ("c4_microsphere_traction", lambda: P.config_c4(4)),
    ("c4_langevin_traction", lambda: P.config_c4(4, traction=0.2, statistics="langevin",
                                                 segments_per_chain=5)),
    ("affine_microsphere_cube_example",
     lambda: cube_example_problem("affine_microsphere_cube_example")),
    ("c4_nonaffine_traction", lambda: P.config_c4(4, traction=0.2, statistics="nonaffine",
                                                  segments_per_chain=5,
                                                  nonaffine_stretch_parameter=1.5)),
    ("nonaffine_microsphere_cube_example",
     lambda: cube_example_problem("nonaffine_microsphere_cube_example")),
    ("c5_neohooke_tet4", lambda: P.config_c5_instance(3, 1.3, increments=2)),
    ("neohooke_cube_example", cube_example_problem),
])
def test_static_solve_parity(api, oracle, name, make):
    pr = make()
    rep_o, u_o, log_o, sm, u = _solve_both(api, oracle, pr)
    assert rep_o["status"] == 0, rep_o["message"]
    assert sm.report["status"] == 0, sm.report["message"]
    assert sm.report["load_steps"] == rep_o["load_steps"]
    assert sm.report["newton_iterations"] == rep_o["newton_iterations"]
    assert rel_err(u, u_o) < 1e-10
    # same Newton trajectory: iteration numbers and the norms the convergence test reads
    assert np.array_equal(sm.log[:, :2], log_o[:, :2])
    # norms near the CG noise floor (rtol 1e-10 of the step's first residual) differ by CG
    # round-off; the rest agree to 1e-6
    for col in (3, 4):
        floor = 1e-8 * np.abs(log_o[:, col]).max()
        np.testing.assert_allclose(sm.log[:, col], log_o[:, col], rtol=1e-6, atol=floor)


def test_mixed_precision_matches_fp64_device(api):
    pr = P.config_c3(6, steps=20)
    pr.options.period = 5.0  # first five increments of the cycle (into the plastic range)
    u64 = api.StaticMatrix(pr).solve()
    sm = api.StaticMatrix(pr, precision=api.MIXED, mixed_inner_tolerance=1e-4)
    u32 = sm.solve()
    assert rel_err(u32, u64) < 1e-8


def test_negative_jacobian_is_a_computational_error(api):
    """Failure detection without a GPU fault: an inverting displacement sets the device status
    word; the host maps it to neon's computational_error message."""
    m = M.structured_hex8(2)
    g = api.SolidMesh(m.X, m.conn, MATERIALS["neohooke"])
    u = np.zeros(g.ndofs)
    u[2::3] = -2.0 * m.X[:, 2]  # z -> -z: inverts every element
    with pytest.raises(api.ComputationalError, match="Positive Jacobian assumption violated"):
        g.update_internal_variables(u)
    # the context stays usable
    g.update_internal_variables(np.zeros(g.ndofs))


def test_cutback_then_failure_reports_status(api, oracle):
    """Newton limit 1 on a nonlinear step: both paths cut back until the limit and report."""
    pr = P.config_c2(3, increments=1)
    pr.options.linear_iterations = 1
    rep_o, u_o, f_o, log_o, _ = oracle.static_solve(pr)
    sm = api.StaticMatrix(pr)
    with pytest.raises(api.ComputationalError):
        sm.solve()
    assert sm.report["status"] == rep_o["status"] != 0
    assert sm.report["newton_iterations"] == rep_o["newton_iterations"]


def test_full_size_c3_assembly_properties(api):
    """Size-independent properties at the full 100^3 J2 size: K symmetric, rigid translations in
    its null space at u = 0, f_int = 0 at u = 0, and the device pattern size of the config."""
    pr = P.config_c3(100)
    g = api.SolidMesh(pr.mesh.X, pr.mesh.conn, pr.material)
    assert g.ndofs == 3090903 and g.nnz == 245438109
    g.set_displacement(np.zeros(g.ndofs))
    g.update_assemble_device(api.FP64)
    K, f = g.download_system()
    assert np.abs(f).max() == 0.0
    import scipy.sparse as sp
    rp, col = g.sparsity_pattern()
    A = sp.csr_matrix((K, col, rp), shape=(g.ndofs, g.ndofs))
    asym = abs(A - A.T).max()
    assert asym <= 1e-12 * abs(K).max()
    for k in range(3):
        t = np.zeros(g.ndofs)
        t[k::3] = 1.0
        assert np.abs(A @ t).max() <= 1e-9 * abs(K).max()


def test_cpp_adapter_driver(api, oracle):
    """The C++ adapter (include/neon_b200.hpp) used from a C++ program, as neon would."""
    import json
    import subprocess
    from neon_b200 import build
    exe = build.build_adapter_driver()
    out = json.loads(subprocess.run([exe, "4"], check=True, capture_output=True,
                                    text=True).stdout)
    np.testing.assert_allclose(out["cg_x"], [1.375, 1.75, 1.625], atol=1e-5)
    assert out["maxit_threw"] is True
    pr = P.config_c1(4)
    rep, u_o, _, _, _ = oracle.static_solve(pr)
    assert rep["status"] == 0
    assert out["newton_iterations"] == rep["newton_iterations"]
    assert rel_err(np.array(out["u"]), u_o) < 1e-10


@pytest.mark.parametrize("topo", ["hex8", "tet4"])
@pytest.mark.parametrize("model", ["linear_elastic", "neohooke", "j2", "microsphere", "langevin",
                                   "nonaffine"])
def test_element_stiffness_getter(api, oracle, topo, model):
    """nb2_element_stiffness (submesh::tangent_stiffness(e)) equals the oracle's element matrix
    in neon's local DOF order; an element index past the end is refused."""
    m = _meshes()[topo]
    mat = MATERIALS[model]
    Ge = None
    if model in FIELD_MODELS:
        Ge = np.random.Generator(np.random.PCG64(5)).lognormal(0.0, 0.3, m.num_elements)
    g = api.SolidMesh(m.X, m.conn, mat, Ge)
    om = oracle.OracleMesh(m.X, m.conn, mat, Ge)
    u = random_displacement(m, SCALE[model], 21)
    assert om.update(u)[0] == 0
    g.update_internal_variables(u)
    for e in (0, m.num_elements // 2, m.num_elements - 1):
        Ke = g.element_stiffness(e)
        Ko = om.element_stiffness(e)
        assert Ke.shape == Ko.shape == (3 * m.nodes_per_element,) * 2
        assert rel_err(Ke, Ko) < TOL_K
    with pytest.raises(ValueError):
        g.element_stiffness(m.num_elements)
