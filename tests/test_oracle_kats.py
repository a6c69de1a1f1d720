"""Pins the CPU oracle to dbeurle/neon's own known-answer tests (tests/golden/kats.json, made by
tests/golden/make_kats.py from the reference's test sources and example)."""
import numpy as np
import pytest

from conftest import cube_example_problem
from neon_b200 import mesh as M
from neon_b200 import problem as P


def _single_point(oracle, material, n=2):
    """An oracle instance with n quadrature points worth of state (one tet4 element's worth is
    1 point, so use n tet4 elements on dummy coordinates)."""
    X = np.array([[1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0], [0, 0, 0]] * n)
    conn = np.arange(4 * n, dtype=np.int32).reshape(n, 4)
    return oracle.OracleMesh(X, conn, material)


def _is_spd(D):
    D = np.asarray(D).reshape(6, 6)
    return np.linalg.norm(D - D.T) < 1e-5 and np.all(np.linalg.eigvals(D).real > 0)


def test_dof_numbering(kats):
    k = kats["dof_numbering"]
    expand = lambda c: (3 * np.asarray(c)[:, None] + np.arange(3)).reshape(-1)  # noqa: E731
    assert expand(k["one_element"]["connectivity"]).tolist() == k["one_element"]["dofs"]
    for c, d in zip(k["two_elements"]["connectivity"], k["two_elements"]["dofs"]):
        assert expand(c).tolist() == d


def test_linear_elastic_moduli(oracle, kats):
    k = kats["linear_elastic_D"]
    mat = P.make_material({"elastic_modulus": k["E"], "poissons_ratio": k["nu"]},
                          {"name": "isotropic_linear_elasticity"})
    om = _single_point(oracle, mat)
    om.set("H", np.zeros((2, 9)))
    assert om.constitutive_only() == 0
    for D in om.get("D"):
        D = D.reshape(6, 6)
        assert D[0, 0] == pytest.approx(k["D00"], rel=1e-12)
        assert D[3, 3] == pytest.approx(k["D33"], rel=1e-12)
        assert D[0, 1] == pytest.approx(k["D01"], rel=1e-12)
        assert _is_spd(D)
    assert np.abs(om.get("sigma")).max() < k["margin"]
    H = np.zeros((2, 9))
    H[:, 4] = k["uniaxial_H11"]
    om.set("H", H)
    om.constitutive_only()
    for s, vm in zip(om.get("sigma"), om.get("vm")):
        assert abs(s[1]) < k["margin"] and s[0] > 0 and s[4] > 0 and vm < 200e6


def test_j2_known_answers(oracle, kats):
    k = kats["j2"]
    mat = P.make_material({"elastic_modulus": k["E"], "poissons_ratio": k["nu"],
                           "yield_stress": k["yield_stress"],
                           "isotropic_hardening_modulus": k["hardening"]},
                          {"name": "J2_plasticity", "finite_strain": False})
    # yield function helper: f(100e6, 0) <= 0, f(300e6, 0) > 0
    for vm, ebar, sign in k["yield_check"]:
        f = vm - (mat.yield_stress + ebar * mat.hardening)
        assert (f <= 0) if sign == "<=0" else (f > 0)
    for h22, plastic in ((k["elastic_H22"], False), (k["plastic_H22"], True)):
        om = _single_point(oracle, mat)
        H = np.zeros((2, 9))
        H[:, 8] = h22
        om.set("H", H)
        assert om.constitutive_only() == 0
        for s, vm, eb, D in zip(om.get("sigma"), om.get("vm"), om.get("epbar"), om.get("D")):
            assert _is_spd(D)
            assert abs(s[1]) < 1e-5 and abs(s[2]) < 1e-5 and abs(s[5]) < 1e-5
            assert s[0] > 0 and s[4] > 0 and s[8] > 0
            if plastic:
                assert eb > 0 and k["yield_stress"] < vm <= k["plastic_vm_max"]
            else:
                assert eb == pytest.approx(0.0, abs=1e-5) and vm < k["yield_stress"]


def test_neo_hooke_known_answers(oracle, kats):
    k = kats["neo_hooke"]
    mat = P.make_material({"elastic_modulus": k["E"], "poissons_ratio": k["nu"]},
                          {"name": "neohooke"})
    om = _single_point(oracle, mat)
    om.set("F", np.tile(np.eye(3).reshape(-1), (2, 1)))
    om.set("detF", np.ones(2))
    om.constitutive_only()
    assert np.abs(om.get("sigma")).max() < k["margin"]
    for D in om.get("D"):
        D = D.reshape(6, 6)
        assert D[0, 0] == pytest.approx(D[1, 1]) and D[0, 1] == pytest.approx(D[0, 2])
        assert D[3, 3] == pytest.approx(D[4, 4]) and D[5, 5] == pytest.approx(D[4, 4])
        assert _is_spd(D)


def test_microsphere_known_answers(oracle, kats):
    k = kats["gaussian_affine_microsphere"]
    mat = P.make_material({"elastic_modulus": k["E"], "poissons_ratio": k["nu"],
                           "segments_per_chain": k["segments_per_chain"]},
                          {"name": "microsphere", "type": "affine", "statistics": "gaussian",
                           "quadrature": "BO21"})
    om = _single_point(oracle, mat)
    om.set("F", np.tile(np.eye(3).reshape(-1), (2, 1)))
    om.set("detF", np.ones(2))
    om.constitutive_only()
    assert all(_is_spd(D) for D in om.get("D"))
    # BO21 is not exactly isotropic: |sigma(I)| is at the rule's truncation level
    assert np.abs(om.get("sigma")).max() / mat.G < 1e-5
    lam = k["uniaxial_stretch"]
    F = np.diag([lam, 1 / np.sqrt(lam), 1 / np.sqrt(lam)]).reshape(-1)
    om.set("F", np.tile(F, (2, 1)))
    om.set("detF", np.full(2, np.linalg.det(F.reshape(3, 3))))
    om.constitutive_only()
    assert all(_is_spd(D) for D in om.get("D"))
    assert all(np.linalg.norm(s) > 0 for s in om.get("sigma"))


def _langevin(E, nu, N):
    return P.make_material({"elastic_modulus": E, "poissons_ratio": nu, "segments_per_chain": N},
                           {"name": "microsphere", "type": "affine", "statistics": "langevin",
                            "quadrature": "BO21"})


def _uniaxial(om, lam):
    F = np.diag([lam, 1 / np.sqrt(lam), 1 / np.sqrt(lam)]).reshape(-1)
    om.set("F", np.tile(F, (2, 1)))
    om.set("detF", np.full(2, np.linalg.det(F.reshape(3, 3))))
    om.constitutive_only()


def test_langevin_microsphere_known_answers(oracle, kats):
    """test/hyperelastic_constitutive.cpp "Affine microsphere": no stress and a symmetric positive
    definite tangent at F = I, a symmetric positive definite tangent under uniaxial stretch."""
    k = kats["langevin_affine_microsphere"]
    mat = _langevin(k["E"], k["nu"], k["segments_per_chain"])
    assert mat.model == P.LANGEVIN_AFFINE_MICROSPHERE
    om = _single_point(oracle, mat)
    om.set("F", np.tile(np.eye(3).reshape(-1), (2, 1)))
    om.set("detF", np.ones(2))
    om.constitutive_only()
    assert all(_is_spd(D) for D in om.get("D"))
    assert np.abs(om.get("sigma")).max() / mat.G < 1e-5
    _uniaxial(om, k["uniaxial_stretch"])
    assert all(_is_spd(D) for D in om.get("D"))
    assert all(np.linalg.norm(s) > 0 for s in om.get("sigma"))


def test_langevin_tends_to_gaussian_for_long_chains(oracle):
    """pade_first -> 3 and pade_second - pade_first -> 0 as N -> infinity: the Langevin model
    becomes the Gaussian one (tau = 3 G sum w t(x)t, zero macro moduli)."""
    gauss = P.make_material({"elastic_modulus": 10e6, "poissons_ratio": 0.45,
                             "segments_per_chain": 50},
                            {"name": "microsphere", "type": "affine", "statistics": "gaussian",
                             "quadrature": "BO21"})
    og, ol = _single_point(oracle, gauss), _single_point(oracle, _langevin(10e6, 0.45, 1e12))
    for om in (og, ol):
        _uniaxial(om, 1.3)
    assert np.abs(ol.get("sigma") - og.get("sigma")).max() < 1e-9 * np.abs(og.get("sigma")).max()
    assert np.abs(ol.get("D") - og.get("D")).max() < 1e-9 * np.abs(og.get("D")).max()


def test_langevin_chains_stiffen_with_stretch(oracle):
    """Finite chains lock: the ratio of the Langevin to the Gaussian uniaxial stress grows with
    the stretch and with fewer segments per chain."""
    gauss = P.make_material({"elastic_modulus": 1.0, "poissons_ratio": 0.45,
                             "segments_per_chain": 50},
                            {"name": "microsphere", "type": "affine", "statistics": "gaussian",
                             "quadrature": "BO21"})
    ratios = {}
    for N in (5.0, 20.0):
        for lam in (1.2, 1.6):
            og, ol = _single_point(oracle, gauss), _single_point(oracle, _langevin(1.0, 0.45, N))
            _uniaxial(og, lam)
            _uniaxial(ol, lam)
            ratios[N, lam] = ol.get("sigma")[0][0] / og.get("sigma")[0][0]
    assert ratios[5.0, 1.6] > ratios[5.0, 1.2] > 1.0
    assert ratios[5.0, 1.6] > ratios[20.0, 1.6] > 1.0


def test_nonaffine_microsphere_known_answers(oracle, kats):
    """test/hyperelastic_constitutive.cpp "Nonaffine microsphere": no stress and a symmetric
    positive definite tangent at F = I, a symmetric positive definite tangent under uniaxial
    stretch."""
    k = kats["nonaffine_microsphere"]
    mat = P.make_material({"elastic_modulus": k["E"], "poissons_ratio": k["nu"],
                           "nonaffine_stretch_parameter": k["nonaffine_stretch_parameter"],
                           "segments_per_chain": k["segments_per_chain"]},
                          {"name": "microsphere", "type": "nonaffine", "quadrature": "BO21"})
    assert mat.model == P.NONAFFINE_MICROSPHERE
    om = _single_point(oracle, mat)
    om.set("F", np.tile(np.eye(3).reshape(-1), (2, 1)))
    om.set("detF", np.ones(2))
    om.constitutive_only()
    assert all(_is_spd(D) for D in om.get("D"))
    assert np.abs(om.get("sigma")).max() / mat.G < 1e-5
    _uniaxial(om, k["uniaxial_stretch"])
    assert all(_is_spd(D) for D in om.get("D"))
    assert all(np.linalg.norm(s) > 0 for s in om.get("sigma"))


def test_nonaffine_stress_is_objective_and_isochoric(oracle):
    """The non-affine model depends on F only through Fbar, and through Fbar by stretches:
    a rotation R F gives R sigma R^T, a dilatation leaves the deviatoric stress unchanged."""
    mat = P.make_material({"bulk_modulus": 100.0, "shear_modulus": 1.0,
                           "nonaffine_stretch_parameter": 1.0, "segments_per_chain": 50},
                          {"name": "microsphere", "type": "nonaffine", "quadrature": "BO21"})
    F = np.array([[1.2, 0.1, 0.0], [0.05, 0.9, 0.1], [0.0, -0.1, 1.05]])
    c, s_ = np.cos(0.4), np.sin(0.4)
    R = np.array([[c, -s_, 0], [s_, c, 0], [0, 0, 1.0]])
    out = {}
    for key, Fq in (("F", F), ("RF", R @ F), ("aF", 1.1 * F)):
        om = _single_point(oracle, mat)
        om.set("F", np.tile(Fq.reshape(-1), (2, 1)))
        om.set("detF", np.full(2, np.linalg.det(Fq)))
        om.constitutive_only()
        out[key] = om.get("sigma")[0].reshape(3, 3)
    scale = np.abs(out["F"]).max()
    assert np.abs(R @ out["F"] @ R.T - out["RF"]).max() < 1e-12 * scale
    dev = lambda s: s - np.trace(s) / 3 * np.eye(3)  # noqa: E731
    # the deviatoric Kirchhoff stress J dev(sigma) is the same for F and a F
    assert np.abs(np.linalg.det(F) * dev(out["F"]) -
                  np.linalg.det(1.1 * F) * dev(out["aF"])).max() < 1e-12 * scale


def test_langevin_cube_example_deck(kats):
    """The affine microsphere cube example's deck builds the Langevin model on the shared cube
    mesh (examples/.../affine_microsphere/cube/cube.json)."""
    pr = cube_example_problem("affine_microsphere_cube_example")
    assert pr.material.model == P.LANGEVIN_AFFINE_MICROSPHERE
    assert pr.material.segments_per_chain == 45
    assert pr.mesh.conn.shape[1] == 8
    pn = cube_example_problem("nonaffine_microsphere_cube_example")
    assert pn.material.model == P.NONAFFINE_MICROSPHERE
    assert pn.material.nonaffine_stretch_parameter == 1.0 and pn.options.linear_iterations == 15


def test_cg_three_by_three(oracle, kats):
    k = kats["cg_3x3"]
    import scipy.sparse as sp
    t = np.array(k["triplets"])
    A = sp.csr_matrix((t[:, 2], (t[:, 0].astype(int), t[:, 1].astype(int))), shape=(3, 3))
    A.sort_indices()
    # setFromTriplets keeps explicit zeros: the pattern is the full 3x3
    rp = np.array([0, 3, 6, 9], np.int32)
    col = np.tile(np.arange(3, dtype=np.int32), 3)
    val = np.array([A[i, j] for i in range(3) for j in range(3)])
    for tol, rcm in ((1e-5, True), (1e-5, False), (1e-12, True)):
        st, x, it, err = oracle.cg_solve(rp, col, val, np.array(k["b"]), tol, 2000, rcm)
        assert st == 0
        np.testing.assert_allclose(x, k["x"], atol=k["margin"])


def test_quadrature_rules(oracle, kats):
    k = kats["quadrature"]
    dN, w = oracle.shape(8)
    assert w.sum() == pytest.approx(k["hex8_weight_sum"])
    assert np.abs(dN.sum(axis=1)).max() < 1e-14  # sum_a dN_a = 0 (partition of unity)
    dN4, w4 = oracle.shape(4)
    assert w4.sum() == pytest.approx(k["tet1_weight_sum"])
    assert np.abs(dN4.sum(axis=1)).max() < 1e-14
    r, ws = oracle.sphere_rule()
    assert len(ws) == k["bo21_points"] and ws.sum() == pytest.approx(k["bo21_weight_sum"])
    np.testing.assert_allclose(np.linalg.norm(r, axis=1), 1.0, rtol=1e-11)
    # unit cube volume: sum_q det(X dN) w
    m = M.structured_hex8(1)
    vol = sum(np.linalg.det(m.X[m.conn[0]].T @ dN[l]) * w[l] for l in range(8))
    assert vol == pytest.approx(k["unit_cube_volume"])


def test_bo33_unit_sphere_rule(oracle):
    """The 33-point rule (Bazant and Oh 1986, unit_sphere_quadrature.cpp:33-91): unit directions,
    weights summing to 1, isotropic second moment, and the microsphere models on it stress-free
    at F = I and close to the 21-point rule under stretch (both integrate the same sphere)."""
    r, w = oracle.sphere_rule(33)
    assert len(w) == 33 and w.sum() == pytest.approx(1.0, abs=1e-11)
    np.testing.assert_allclose(np.linalg.norm(r, axis=1), 1.0, rtol=1e-11)
    np.testing.assert_allclose((w[:, None, None] * r[:, :, None] * r[:, None, :]).sum(0),
                               np.eye(3) / 3.0, atol=1e-11)
    sig = {}
    for q in ("BO21", "BO33"):
        mat = P.make_material({"bulk_modulus": 100.0, "shear_modulus": 1.0,
                               "segments_per_chain": 8},
                              {"name": "microsphere", "type": "affine", "statistics": "langevin",
                               "quadrature": q})
        assert mat.unit_sphere_points == int(q[2:])
        om = _single_point(oracle, mat)
        om.set("F", np.tile(np.eye(3).reshape(-1), (2, 1)))
        om.set("detF", np.ones(2))
        om.constitutive_only()
        assert np.abs(om.get("sigma")).max() < 1e-5
        assert all(_is_spd(D) for D in om.get("D"))
        _uniaxial(om, 1.3)
        sig[q] = om.get("sigma")[0].reshape(3, 3)
    assert np.abs(sig["BO33"] - sig["BO21"]).max() < 0.02 * np.abs(sig["BO21"]).max()


def test_cube_fixture_element_symmetry(oracle, kats):
    k = kats["cube_fixture"]
    m = M.structured_hex8(3)
    assert m.num_nodes == k["nodes"] and m.num_elements == k["hex8"]
    mat = P.make_material({"elastic_modulus": 200e6, "poissons_ratio": 0.45}, {"name": "neohooke"})
    om = oracle.OracleMesh(m.X, m.conn, mat)
    assert om.ndofs == k["active_dofs"]
    assert om.update(np.zeros(om.ndofs))[0] == 0
    for e in range(m.num_elements):
        ke = om.element_stiffness(e)
        assert np.abs(ke).max() > 0
        assert np.abs(ke - ke.T).max() <= 1e-9 * np.abs(ke).max()


def test_pattern_equals_triplet_pattern(oracle):
    """setFromTriplets semantics: sorted unique columns per row from every element DOF pair."""
    import scipy.sparse as sp
    for m in (M.structured_hex8(3, 2, 2), M.structured_tet4(2)):
        mat = P.make_material({"elastic_modulus": 1.0, "poissons_ratio": 0.3},
                              {"name": "isotropic_linear_elasticity"})
        om = oracle.OracleMesh(m.X, m.conn, mat)
        rp, col = om.pattern()
        dofs = (3 * m.conn[:, :, None] + np.arange(3)).reshape(m.num_elements, -1)
        i = np.repeat(dofs, dofs.shape[1], axis=1).ravel()
        j = np.tile(dofs, (1, dofs.shape[1])).ravel()
        A = sp.csr_matrix((np.ones(len(i)), (i, j)), shape=(om.ndofs, om.ndofs))
        A.sum_duplicates()
        A.sort_indices()
        assert np.array_equal(A.indptr, rp) and np.array_equal(A.indices, col)


def test_neohooke_cube_example_verify_criteria(oracle, kats):
    """examples/.../neohooke/cube: u_z max 0.5 and du_z/dz = 0.5 (verify.py)."""
    k = kats["neohooke_cube_example"]
    pr = cube_example_problem()
    rep, u, f, log, om = oracle.static_solve(pr)
    assert rep["status"] == 0, rep["message"]
    uz = u[2::3]
    z = pr.mesh.X[:, 2]
    assert uz.max() == pytest.approx(k["max_displacement"], rel=k["rel_tol"])
    slope, icpt = np.polyfit(z, uz, 1)
    assert slope == pytest.approx(k["slope"], rel=1e-6)


def test_uniaxial_patch_neo_hooke_jittered(oracle):
    """Homogeneous uniaxial stretch on a jittered mesh: u_z = (lambda - 1) z exactly and the
    lateral stretch solves lambda ln(lambda l^2) + mu (l^2 - 1) = 0 (compressible_neohooke.cpp)."""
    pr = P.config_c2(4, increments=3)
    rep, u, f, log, om = oracle.static_solve(pr)
    assert rep["status"] == 0, rep["message"]
    X = pr.mesh.X
    np.testing.assert_allclose(u[2::3], 0.3 * X[:, 2], atol=1e-9)
    from scipy.optimize import brentq
    lam, mu, s = pr.material.lam, pr.material.G, 1.3
    # sigma_xx = 0: lam ln J + mu (l^2 - 1) = 0 with J = s l^2
    l = brentq(lambda l: lam * np.log(s * l * l) + mu * (l * l - 1.0), 0.5, 1.0)
    np.testing.assert_allclose(u[0::3], (l - 1.0) * X[:, 0], atol=1e-8)


def _triangle_mesh(oracle):
    """The reference's right triangle (0,0,0), (1,0,0), (0,1,0) as face 0-1-2 of a tet4."""
    X = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
    mat = P.make_material({"elastic_modulus": 1.0, "poissons_ratio": 0.3},
                          {"name": "isotropic_linear_elasticity"})
    return oracle.OracleMesh(X, np.array([[0, 1, 2, 3]], np.int32), mat)


def test_triangle_traction_and_pressure_known_answers(oracle):
    """test/boundary.cpp:72-112 (traction 1 on the triangle: 1/6 per node, 2 -> 2/6) and
    :114-166 (pressure -1: z components 1/6, -2 -> 2/6)."""
    om = _triangle_mesh(oracle)
    tri = np.array([[0, 1, 2]], np.int32)
    t = om.nonfollower_load(P.TRACTION, 0, tri)
    np.testing.assert_allclose(t[[0, 3, 6]], 1.0 / 6.0, atol=1e-15)
    np.testing.assert_allclose(2.0 * t[[0, 3, 6]], 2.0 / 6.0, atol=1e-15)
    assert np.count_nonzero(t) == 3
    p = om.nonfollower_load(P.PRESSURE, 0, tri)
    np.testing.assert_allclose(-1.0 * p[[2, 5, 8]], 1.0 / 6.0, atol=1e-15)
    np.testing.assert_allclose(-2.0 * p[[2, 5, 8]], 2.0 / 6.0, atol=1e-15)
    np.testing.assert_allclose(p[[0, 1, 3, 4, 6, 7, 9, 10, 11]], 0.0, atol=1e-15)


def test_nonfollower_load_integrals(oracle):
    """Consistent loads integrate exactly: the traction vector sums to the face area, the body
    force to the volume, and a pressure on a closed surface to zero (divergence theorem), on a
    cube whose boundary is warped so the faces are not planar."""
    m = M.structured_hex8(4, 3, 5)
    X = m.X.copy()
    X += 0.03 * np.sin(np.pi * X[:, [1, 2, 0]]) * np.sin(np.pi * X[:, [2, 0, 1]])
    mat = P.make_material({"elastic_modulus": 1.0, "poissons_ratio": 0.3},
                          {"name": "isotropic_linear_elasticity"})
    om = oracle.OracleMesh(X, m.conn, mat)
    closed = np.concatenate([m.faces[k] for k in ("bottom", "top", "x0", "x1", "y0", "y1")])
    p = om.nonfollower_load(P.PRESSURE, 0, closed).reshape(-1, 3)
    assert np.abs(p.sum(axis=0)).max() < 1e-13
    # volume: det J summed over the 8-point rule (exact for trilinear maps)
    b = om.nonfollower_load(P.BODY_FORCE, 2, None)
    q = om.nonfollower_load(P.BODY_FORCE, 0, None)
    assert abs(b.sum() - q.sum()) < 1e-14 and b.sum() > 0.9
    top = m.faces["top"]
    t = om.nonfollower_load(P.TRACTION, 2, top)
    tr = om.nonfollower_load(P.TRACTION, 2, top, reduced=True)
    assert abs(t.sum() - tr.sum()) < 0.05 * t.sum()  # 1-point vs 4-point area of a warped face
    # a flat face (the structured mesh): the area is exact on both rules
    om0 = oracle.OracleMesh(m.X, m.conn, mat)
    a4 = om0.nonfollower_load(P.TRACTION, 2, top).sum()
    a1 = om0.nonfollower_load(P.TRACTION, 2, top, reduced=True).sum()
    assert abs(a4 - 1.0) < 1e-14 and abs(a1 - 1.0) < 1e-14
    assert abs(om0.nonfollower_load(P.BODY_FORCE, 1, None).sum() - 1.0) < 1e-14
