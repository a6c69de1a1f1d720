"""Host logic of the batched solves (no GPU): the block-diagonal layout of uneven instances."""
import numpy as np

from neon_b200 import problem as P
from neon_b200.api import batch_layout


def test_layout_offsets_and_shifted_tables():
    probs = [P.config_c5_instance(m, mu) for m, mu in [(2, 0.5), (3, 1.0), (1, 2.0)]]
    lay = batch_layout(probs)
    nodes = [p.mesh.num_nodes for p in probs]
    assert list(lay["node_offsets"]) == [0, nodes[0], nodes[0] + nodes[1], sum(nodes)]
    assert lay["X"].shape == (sum(nodes), 3)
    # connectivity of instance i lies inside its node range
    eo = lay["element_offsets"]
    for i in range(len(probs)):
        c = lay["conn"][eo[i]:eo[i + 1]]
        assert c.min() >= lay["node_offsets"][i] and c.max() < lay["node_offsets"][i + 1]
        np.testing.assert_array_equal(c - lay["node_offsets"][i], probs[i].mesh.conn)
        np.testing.assert_allclose(lay["G"][eo[i]:eo[i + 1]], probs[i].material.G)
        np.testing.assert_allclose(lay["K"][eo[i]:eo[i + 1]], probs[i].material.K)
    # tables: same count per instance, DOFs shifted by 3 x node offset
    do = lay["dirichlet_offsets"]
    for i, p in enumerate(probs):
        assert do[i + 1] - do[i] == len(p.dirichlet)
        for t0, t1 in zip(p.dirichlet, lay["dirichlet"][do[i]:do[i + 1]]):
            np.testing.assert_array_equal(np.asarray(t1.dofs) - 3 * lay["node_offsets"][i],
                                          t0.dofs)
            np.testing.assert_array_equal(t1.values, t0.values)


def test_layout_rejects_mixed_models():
    a = P.config_c5_instance(2, 1.0)
    b = P.config_c1(2)
    try:
        batch_layout([a, b])
    except ValueError:
        return
    raise AssertionError("a batch of two models must be rejected")


def test_c5_sizes_are_seeded_and_in_range():
    s1 = P.config_c5_sizes()
    assert s1 == P.config_c5_sizes()
    assert len(s1) == 256
    assert all(8 <= m <= 40 and 0.5 <= mu <= 2.0 for m, mu in s1)
