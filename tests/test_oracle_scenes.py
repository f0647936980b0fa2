"""The oracle-side scene builder (oracle/scenes.py), which feeds the CPU
reference arm of the benchmark, produces exactly the product's scene: every
array bit for bit, the Schwarz subdomain choice and the seeded initial state."""
import numpy as np
import pytest

import higher_order_embedded_fem_b200 as H
from oracle import scenes as OS


@pytest.mark.parametrize("n,seed", [(6, 2), (24, 2)])
def test_oracle_cylinder_scene_matches_product(n, seed):
    e = H.scenes.embedded_cylinder(n, 0.3, 0.4, 8, 27, seed)
    o = OS.embedded_cylinder(n, 0.3, 0.4, 8, 27, seed)
    b0, b1 = e.blocks
    assert np.array_equal(o.vertices, e.vertices)
    assert np.array_equal(o.interior_conn, b0.connectivity)
    assert np.array_equal(o.interface_conn, b1.connectivity)
    assert np.array_equal(o.interior_rule[0], b0.weights)
    assert np.array_equal(o.interior_rule[1], b0.points)
    assert np.array_equal(o.iface_offsets, b1.offsets)
    assert np.array_equal(o.iface_weights, b1.weights)
    assert np.array_equal(o.iface_points, b1.points)
    assert np.array_equal(o.volume_fractions, e.volume_fractions)
    assert o.cell_size == e.cell_size


def test_oracle_schwarz_choice_and_state_match_product():
    e = H.scenes.embedded_cylinder(8, 0.3, 0.4, 8, 27, 2)
    o = OS.embedded_cylinder(8, 0.3, 0.4, 8, 27, 2)
    b0, b1 = e.blocks
    model = H.EmbeddedModel3d(e.vertices, b0.connectivity, b1.connectivity, (b0.weights, b0.points),
                              (b1.offsets, b1.weights, b1.points))
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(model, e.volume_fractions, 0.5)
    subs, untreated = o.schwarz_subdomains(0.5)
    assert len(subs) == len(comp.schwarz_connectivity)
    assert all(np.array_equal(a, b) for a, b in zip(subs, comp.schwarz_connectivity))
    assert np.array_equal(untreated, comp.untreated_nodes)
    for seed, nn in [(1000, 7), (1002, 3 * e.vertices.shape[0])]:
        assert np.array_equal(OS.random_normal(seed, nn, 0.25), H.scenes.random_normal(seed, nn, 0.25))
