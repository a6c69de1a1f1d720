"""Adjoint gradient of the microsphere problem (config 4 shape, small mesh): against central
finite differences of the forward solve and against the mixed-precision adjoint; the
torch.autograd harness gives the same gradient."""
import numpy as np
import pytest

from conftest import rel_err
from neon_b200 import problem as P

pytestmark = pytest.mark.gpu


def _problem(n=4, seed=7):
    pr = P.config_c4(n, seed_field=seed)
    o = pr.options
    o.residual_tolerance = o.displacement_tolerance = 1e-13
    o.cg_tolerance = 1e-13
    o.linear_iterations = 25
    return pr


def _objective(pr, u, u_target):
    top = np.unique(pr.mesh.faces["top"].reshape(-1))
    dofs = (3 * top[:, None] + np.arange(3)).reshape(-1)
    d = u[dofs] - u_target[dofs]
    g = np.zeros_like(u)
    g[dofs] = d
    return 0.5 * float(d @ d), g


@pytest.fixture(scope="module")
def setup():
    from neon_b200 import api, build
    build.build()
    pr = _problem()
    target = P.config_c4(4, seed_field=99)
    u_target = api.StaticMatrix(target).solve()
    return api, pr, u_target


def test_adjoint_matches_central_differences(setup):
    api, pr, u_target = setup
    sm = api.StaticMatrix(pr)
    u = sm.solve()
    J, g = _objective(pr, u, u_target)
    grad = sm.mesh.adjoint_shear_gradient(g, api.FP64, 1e-13)
    rng = np.random.Generator(np.random.PCG64(3))
    picks = rng.choice(pr.mesh.num_elements, size=8, replace=False)
    G0 = pr.element_shear_modulus.copy()
    for e in picks:
        h = 1e-4 * G0[e]
        vals = []
        for sgn in (1.0, -1.0):
            pr.element_shear_modulus = G0.copy()
            pr.element_shear_modulus[e] += sgn * h
            up = api.StaticMatrix(pr).solve()
            vals.append(_objective(pr, up, u_target)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(grad[e] - fd) <= 1e-5 * abs(fd) + 1e-9 * np.abs(grad).max(), (e, grad[e], fd)
    pr.element_shear_modulus = G0


def test_mixed_adjoint_matches_fp64(setup):
    api, pr, u_target = setup
    sm = api.StaticMatrix(pr)
    u = sm.solve()
    _, g = _objective(pr, u, u_target)
    g64 = sm.mesh.adjoint_shear_gradient(g, api.FP64, 1e-12)
    g32 = sm.mesh.adjoint_shear_gradient(g, api.MIXED, 1e-12)
    assert rel_err(g32, g64) < 1e-9


def test_torch_autograd_harness(setup):
    import torch
    from neon_b200.autograd import equilibrium_displacement
    api, pr, u_target = setup
    G = torch.tensor(pr.element_shear_modulus, dtype=torch.float64, requires_grad=True)
    u = equilibrium_displacement(G, pr)
    top = np.unique(pr.mesh.faces["top"].reshape(-1))
    dofs = torch.from_numpy((3 * top[:, None] + np.arange(3)).reshape(-1))
    d = u[dofs] - torch.from_numpy(u_target)[dofs]
    J = 0.5 * (d * d).sum()
    J.backward()
    sm = api.StaticMatrix(pr)
    _, g = _objective(pr, sm.solve(), u_target)
    ref = sm.mesh.adjoint_shear_gradient(g, api.FP64, 1e-12)
    assert rel_err(G.grad.numpy(), ref) < 1e-10


def test_langevin_adjoint_matches_central_differences(setup):
    """The same adjoint for the Langevin affine microsphere: d sigma / dG carries the Pade chain
    weight, and the defect-corrected transpose solve uses the Langevin force's forward-mode
    product."""
    api = setup[0]

    def langevin(seed):
        pr = P.config_c4(4, seed_field=seed, statistics="langevin", segments_per_chain=5)
        o = pr.options
        o.residual_tolerance = o.displacement_tolerance = 1e-13
        o.cg_tolerance = 1e-13
        o.linear_iterations = 25
        return pr

    pr = langevin(7)
    u_target = api.StaticMatrix(langevin(99)).solve()
    sm = api.StaticMatrix(pr)
    u = sm.solve()
    _, g = _objective(pr, u, u_target)
    grad = sm.mesh.adjoint_shear_gradient(g, api.FP64, 1e-13)
    rng = np.random.Generator(np.random.PCG64(5))
    G0 = pr.element_shear_modulus.copy()
    for e in rng.choice(pr.mesh.num_elements, size=6, replace=False):
        h = 1e-4 * G0[e]
        vals = []
        for sgn in (1.0, -1.0):
            pr.element_shear_modulus = G0.copy()
            pr.element_shear_modulus[e] += sgn * h
            vals.append(_objective(pr, api.StaticMatrix(pr).solve(), u_target)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(grad[e] - fd) <= 1e-5 * abs(fd) + 1e-9 * np.abs(grad).max(), (e, grad[e], fd)
    pr.element_shear_modulus = G0
    assert pr.material.model == P.LANGEVIN_AFFINE_MICROSPHERE


def test_c4_full_size_adjoint(setup):
    """Config 4 at its own size: 48^3 hex8 (110,592 elements), lognormal(0, 0.3) shear-modulus
    field, top traction; the gradient of J = 1/2 |u_top - u_target|^2 with respect to all
    110,592 moduli against central differences (h = 1e-4 G_e) on 8 random elements (the
    configuration asks for 64; each difference is two full forward solves), and the FP32-bulk
    adjoint against the FP64 one."""
    api = setup[0]
    pr = _problem(48, seed=7)
    assert pr.mesh.num_elements == 110592
    target = P.config_c4(48, seed_field=99)
    u_target = api.StaticMatrix(target).solve()
    sm = api.StaticMatrix(pr)
    u = sm.solve()
    _, g = _objective(pr, u, u_target)
    # the transpose solve at rtol 1e-11 (1e-13 is below what the FP64 PCG reaches at this size)
    grad = sm.mesh.adjoint_shear_gradient(g, api.FP64, 1e-11)
    g32 = sm.mesh.adjoint_shear_gradient(g, api.MIXED, 1e-11)
    assert rel_err(g32, grad) < 1e-8
    rng = np.random.Generator(np.random.PCG64(11))
    G0 = pr.element_shear_modulus.copy()
    # the elements whose moduli move the top face most, and random ones
    top_elems = np.argsort(-np.abs(grad))[:4]
    picks = np.concatenate([top_elems, rng.choice(pr.mesh.num_elements, size=4, replace=False)])
    for e in picks:
        h = 1e-4 * G0[e]
        vals = []
        for sgn in (1.0, -1.0):
            pr.element_shear_modulus = G0.copy()
            pr.element_shear_modulus[e] += sgn * h
            vals.append(_objective(pr, api.StaticMatrix(pr).solve(), u_target)[0])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(grad[e] - fd) <= 1e-4 * abs(fd) + 1e-6 * np.abs(grad).max(), (e, grad[e], fd)
    pr.element_shear_modulus = G0
