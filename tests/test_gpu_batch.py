"""Batched solves of uneven instances in one context: every instance must reach the solution of
its own single-instance solve (which is pinned to the oracle), with the same load steps and
Newton iterations, in FP64 and in mixed precision; a failing instance must not disturb the
others."""
import numpy as np
import pytest

from conftest import rel_err
from neon_b200 import problem as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from neon_b200 import api, build
    build.build()
    return api


SIZES = [(3, 0.7), (2, 1.9), (5, 1.2), (1, 0.5), (4, 1.0)]


def _instances(sizes=SIZES):
    return [P.config_c5_instance(m, mu) for m, mu in sizes]


@pytest.fixture(scope="module")
def singles(api):
    out = []
    for pr in _instances():
        sm = api.StaticMatrix(pr)
        u = sm.solve()
        out.append((u, sm.report, sm.log))
    return out


def test_batched_fp64_equals_single_solves(api, singles):
    bs = api.BatchedStaticMatrix(_instances())
    u = bs.solve()
    for i, (u1, rep, log) in enumerate(singles):
        ui = bs.instance_displacement(i, u)
        assert rel_err(ui, u1) < 1e-10, i
        r = bs.reports[i]
        assert r["status"] == 0
        assert r["load_steps"] == rep["load_steps"]
        assert r["newton_iterations"] == rep["newton_iterations"]
        # same Newton trajectory: step times and iteration indices
        np.testing.assert_array_equal(bs.logs[i][:, :2], log[:, :2])
    assert bs.tuned["rows_per_chunk"] in (16, 32, 64, 128)
    assert bs.tuned["lanes_per_row"] in (4, 8, 16, 32)


def test_batched_matches_oracle(api, oracle):
    pr = _instances([(3, 0.7), (2, 1.9)])
    bs = api.BatchedStaticMatrix(pr, autotune=False)
    u = bs.solve()
    for i, p in enumerate(pr):
        rep, uo, _, _, _ = oracle.static_solve(p)
        assert rep["status"] == 0
        assert rel_err(bs.instance_displacement(i, u), uo) < 1e-10


def test_batched_mixed_reaches_fp64(api, singles):
    bs = api.BatchedStaticMatrix(_instances(), precision=api.MIXED, mixed_inner_tolerance=1e-4)
    u = bs.solve()
    for i, (u1, rep, _) in enumerate(singles):
        assert bs.reports[i]["status"] == 0
        assert rel_err(bs.instance_displacement(i, u), u1) < 1e-8, i


def test_failing_instance_is_isolated(api, singles):
    probs = _instances()
    bad = P.config_c5_instance(2, 1.0)
    # crush the box through itself in one increment: inverted elements, cutbacks, give-up
    for t in bad.dirichlet:
        if t.name == "top":
            t.values = np.array([0.0, -1.5])
    probs.insert(2, bad)
    bs = api.BatchedStaticMatrix(probs, autotune=False)
    with pytest.raises(api.ComputationalError):
        bs.solve()
    assert bs.reports[2]["status"] == api.E_CUTBACK_LIMIT
    single = api.StaticMatrix(bad)
    with pytest.raises(api.ComputationalError):
        single.solve()
    assert single.report["status"] == api.E_CUTBACK_LIMIT
    good = [i for i in range(len(probs)) if i != 2]
    for j, i in enumerate(good):
        assert bs.reports[i]["status"] == 0
        assert rel_err(bs.instance_displacement(i), singles[j][0]) < 1e-10


def test_coupled_instances_are_rejected(api):
    pr = _instances([(2, 1.0), (2, 1.0)])
    bs = api.BatchedStaticMatrix(pr, autotune=False)
    bs.node_offsets = np.array([0, 5, bs.node_offsets[-1]], np.int32)  # cuts instance 0
    with pytest.raises(ValueError):
        bs.solve()


def test_batched_hex8_linear_elastic_instances(api):
    """hex8 instances of different sizes and moduli (config 1 shape) against single solves."""
    probs = []
    for n, E in ((3, 200e3), (5, 70e3), (2, 120e3)):
        pr = P.config_c1(n)
        nu = 0.3
        pr.material.K = E / (3 * (1 - 2 * nu))
        pr.material.G = E / (2 * (1 + nu))
        probs.append(pr)
    bs = api.BatchedStaticMatrix(probs, autotune=False)
    u = bs.solve()
    for i, pr in enumerate(probs):
        u1 = api.StaticMatrix(pr).solve()
        assert rel_err(bs.instance_displacement(i, u), u1) < 1e-10
