"""Oracle: embedded-quadrature construction (embed_mesh_3d, cut-cell
quadrature, moment-fitting simplification), fenris/src/embedding/*.

Checks that need no GPU: the restatement's classification and cut volumes
against exact geometry, polynomial exactness of the cut-cell rules (volume,
first and second moments of the embedded mesh), the single-tet case against
the directly mapped tet rule, and the simplification's invariants.  Also the
product's tet rules against the reference's tables and the product's input
checks that run before any device call.
"""
import numpy as np
import pytest

import higher_order_embedded_fem_b200 as H
from oracle import oracle as O

from test_oracle_golden import GOLD


def _grid(n):
    bg = H.scenes.hex27_box(1.0, 1, 1, 1, n)
    return bg.vertices, bg.blocks[0].connectivity


def _cell_box(V, conn, c):
    Hc = V[conn[c, :8]]
    return Hc.min(0), Hc.max(0)


def _physical_moments(V, conn, emb, off, w, p):
    """Volume, first and second moments over interior + interface cells."""
    tot, m1, m2 = 0.0, np.zeros(3), np.zeros((3, 3))
    for k, c in enumerate(emb.interface_cells):
        lo, hi = _cell_box(V, conn, c)
        ww = w[off[k]:off[k + 1]] * np.prod((hi - lo) / 2)
        x = lo + (p[off[k]:off[k + 1]] + 1) / 2 * (hi - lo)
        tot += ww.sum()
        m1 += ww @ x
        m2 += np.einsum("q,qi,qj->ij", ww, x, x)
    for c in emb.interior_cells:
        lo, hi = _cell_box(V, conn, c)
        v, c0 = np.prod(hi - lo), (lo + hi) / 2
        tot += v
        m1 += v * c0
        m2 += v * (np.outer(c0, c0) + np.diag((hi - lo) ** 2 / 12))
    return tot, m1, m2


@pytest.mark.parametrize("strength", [1, 2, 3, 5])
def test_product_tet_rules_match_reference_tables(strength):
    q = GOLD["quadrature"]["tet_quadrature_strength_%d" % strength]
    w, p = H.tet_quadrature_strength(strength)
    assert np.array_equal(w, np.array(q["weights"]))
    assert np.array_equal(p, np.array(q["points"]))


def test_hollow_cylinder_volume_and_moments_are_exact():
    V, conn = _grid(8)
    X, T = H.scenes.hollow_cylinder_tets(0.3, 0.4, 1.0, 2, 48, 24)
    vol, m1, m2 = H.scenes.tet_mesh_volume_moments(X, T)
    emb = O.Embedding(V, conn, X, T)
    assert len(emb.interface_cells) > 0 and len(emb.exterior_cells) > 0
    assert abs(emb.cut_volume.sum() / vol - 1) < 1e-13
    # classification thresholds (EmbedOptions defaults)
    cellv = (1 / 8) ** 3
    f = emb.cut_volume / cellv
    assert np.all(f[emb.exterior_cells] < 1e-4)
    assert np.all((f[emb.interface_cells] >= 1e-4) & (f[emb.interface_cells] < 0.999))
    assert np.all(f[emb.interior_cells] >= 0.999)
    off, w, p = emb.interface_quadratures(*H.tet_quadrature_strength(2))
    assert np.all(np.abs(p) <= 1 + 1e-12) and np.all(w >= 0)  # degenerate slivers carry weight 0
    tot, mm1, mm2 = _physical_moments(V, conn, emb, off, w, p)
    assert abs(tot / vol - 1) < 1e-13
    assert np.abs(mm1 - m1).max() < 1e-13 * np.abs(m1).max()
    assert np.abs(mm2 - m2).max() < 1e-13 * np.abs(m2).max()


def test_grid_aligned_box_has_no_interface_cells():
    V, conn = _grid(4)
    box = H.scenes.tet10_box(0.25, 2, 2, 2, 1)  # [0, 0.5]^3 in 2^3 hexes, 6 tets each
    X = box.vertices + 0.25  # -> [0.25, 0.75]^3, aligned with the 4^3 grid
    T = box.blocks[0].connectivity[:, :4]
    emb = O.Embedding(V, conn, X, T)
    assert len(emb.interface_cells) == 0
    assert len(emb.interior_cells) == 8
    assert abs(emb.cut_volume.sum() - 0.125) < 1e-15
    for c in emb.interior_cells:
        lo, hi = _cell_box(V, conn, c)
        assert np.all(lo >= 0.25 - 1e-15) and np.all(hi <= 0.75 + 1e-15)


def test_single_tet_inside_a_cell_gets_the_mapped_tet_rule():
    V, conn = _grid(2)
    X = np.array([[0.1, 0.1, 0.1], [0.4, 0.15, 0.12], [0.12, 0.35, 0.2], [0.2, 0.18, 0.45]])
    T = np.array([[0, 1, 2, 3]])
    emb = O.Embedding(V, conn, X, T)
    assert len(emb.interface_cells) == 1
    c = emb.interface_cells[0]
    tw, tp = H.tet_quadrature_strength(5)
    off, w, p = emb.interface_quadratures(tw, tp)
    lo, hi = _cell_box(V, conn, c)
    N = np.stack([-0.5 * tp.sum(1) - 0.5, 0.5 * tp[:, 0] + 0.5, 0.5 * tp[:, 1] + 0.5, 0.5 * tp[:, 2] + 0.5], 1)
    x = N @ X
    xi = (x - lo) / (hi - lo) * 2 - 1
    vol = abs(np.linalg.det(np.stack([X[1] - X[0], X[2] - X[0], X[3] - X[0]]))) / 6
    wref = tw * (vol / (4 / 3)) / np.prod((hi - lo) / 2)
    # a symmetric rule: the same point set whatever the vertex order
    assert len(w) == len(tw)
    match = [int(np.argmin(np.linalg.norm(p - q, axis=1))) for q in xi]
    assert sorted(match) == list(range(len(tw)))
    assert np.abs(p[match] - xi).max() < 1e-14 and np.abs(w[match] - wref).max() < 1e-14 * wref.max()


def test_stabilization_is_appended():
    V, conn = _grid(4)
    X, T = H.scenes.hollow_cylinder_tets(0.3, 0.4, 1.0, 1, 24, 8)
    emb = O.Embedding(V, conn, X, T)
    tw, tp = H.tet_quadrature_strength(1)
    hw, hp = GOLD["quadrature"]["hex_quadrature_strength_5"]["weights"], \
        GOLD["quadrature"]["hex_quadrature_strength_5"]["points"]
    off0, w0, p0 = emb.interface_quadratures(tw, tp)
    off, w, p = emb.interface_quadratures(tw, tp, (1e-3, hw, hp))
    assert np.array_equal(np.diff(off), np.diff(off0) + len(hw))
    for k in range(len(off) - 1):
        n0 = off0[k + 1] - off0[k]
        assert np.array_equal(w[off[k]:off[k] + n0], w0[off0[k]:off0[k + 1]])
        assert np.array_equal(w[off[k] + n0:off[k + 1]], 1e-3 * np.array(hw))
        assert np.array_equal(p[off[k] + n0:off[k + 1]], np.array(hp))


@pytest.mark.parametrize("strength", [1, 2, 3, 4])
def test_simplification_keeps_moments_with_at_most_r_points(strength):
    V, conn = _grid(4)
    X, T = H.scenes.hollow_cylinder_tets(0.3, 0.4, 1.0, 1, 24, 8)
    emb = O.Embedding(V, conn, X, T)
    off, w, p = emb.interface_quadratures(*H.tet_quadrature_strength(3))
    oo, ow, op = O.simplify_quadratures(off, w, p, strength)
    r = O.moment_matrix(p[:1], strength).shape[0]
    assert r == sum((k + 1) * (k + 2) // 2 for k in range(strength + 1))
    assert np.all(ow > 0)
    for k in range(len(off) - 1):
        pk, wk = p[off[k]:off[k + 1]], w[off[k]:off[k + 1]]
        sel, ws = op[oo[k]:oo[k + 1]], ow[oo[k]:oo[k + 1]]
        assert len(ws) <= max(r, 0) or len(ws) == len(wk)
        # the kept points are a subset, in their original order
        idx = [int(np.nonzero((pk == q).all(1))[0][0]) for q in sel]
        assert idx == sorted(idx)
        P = O.moment_matrix(pk, strength)
        m0 = P @ wk
        assert np.abs(P[:, idx] @ ws - m0).max() <= 1e-12 * np.abs(m0).max()


def test_simplification_leaves_small_rules_unchanged():
    tw, tp = H.tet_quadrature_strength(3)
    off = np.array([0, 8])
    oo, ow, op = O.simplify_quadratures(off, tw, tp, 3)  # 8 points <= r = 20
    assert np.array_equal(oo, off) and np.array_equal(ow, tw) and np.array_equal(op, tp)


def test_product_rejects_bad_embedding_input_before_device_use():
    V, conn = _grid(2)
    X = np.array([[0.1, 0.1, 0.1], [0.4, 0.15, 0.12], [0.12, 0.35, 0.2], [0.2, 0.18, 0.45]])
    with pytest.raises(H.HoefemError) as e:
        H.embed_mesh_3d(V, conn, X, np.array([[0, 1, 2, 7]]))
    assert e.value.status == "INVALID_ARGUMENT"
    with pytest.raises(H.HoefemError) as e:
        H.embed_mesh_3d(V, conn, X, np.array([[0, 1, 2, 2]]))
    assert e.value.status == "INVALID_ARGUMENT"
    bad = conn.copy()
    bad[0, 3] = len(V)
    with pytest.raises(H.HoefemError) as e:
        H.embed_mesh_3d(V, bad, X, np.array([[0, 1, 2, 3]]))
    assert e.value.status == "INVALID_ARGUMENT"
    with pytest.raises(ValueError):
        H.embed_mesh_3d(V, conn[:, :10], X, np.array([[0, 1, 2, 3]]))
    with pytest.raises(H.HoefemError) as e:
        H.embedding.simplify_rules(np.array([0, 8]), np.ones(8), np.zeros((8, 3)), 6)
    assert e.value.status == "INVALID_ARGUMENT"
