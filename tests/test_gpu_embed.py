"""Embedded-quadrature construction on the GPU vs the FP64 oracle.

The GPU clips every (background cell, embedded tet) pair on its own; the
oracle restates the reference's region-level clipping.  Their triangulations
of a cut polyhedron may differ (vertex labels), so the parity bar is:
classification identical, cut volume per cell within 1e-13 of the cell
volume, and every moment sum_q w_q xi_q^a (|a| <= the tet rule's strength)
of every interface rule within 1e-12 of the rule's total weight.
Simplification: at most r points, non-negative weights, all moments kept to
1e-12.  Then a Newton step on the cut-cell model against the oracle's step.
"""
import itertools

import numpy as np
import pytest

import higher_order_embedded_fem_b200 as H
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def _grid(n):
    bg = H.scenes.hex27_box(1.0, 1, 1, 1, n)
    return bg.vertices, bg.blocks[0].connectivity


def _monomials(p, degree):
    return np.stack([p[:, 0] ** a * p[:, 1] ** b * p[:, 2] ** c
                     for a, b, c in itertools.product(range(degree + 1), repeat=3) if a + b + c <= degree], 1)


def _rule_moments(off, w, p, degree):
    M = _monomials(p, degree) * w[:, None]
    return np.stack([M[off[k]:off[k + 1]].sum(0) for k in range(len(off) - 1)])


CASES = [(8, (0.3, 0.4, 1.0, 2, 48, 24)), (12, (0.22, 0.41, 1.0, 3, 40, 16)), (5, (0.3, 0.4, 1.0, 1, 24, 8))]


@pytest.fixture(scope="module", params=range(len(CASES)))
def case(request):
    n, cyl = CASES[request.param]
    V, conn = _grid(n)
    X, T = H.scenes.hollow_cylinder_tets(*cyl)
    return V, conn, X, T, O.Embedding(V, conn, X, T), H.embed_mesh_3d(V, conn, X, T)


def test_classification_and_cut_volumes_match_oracle(case):
    V, conn, X, T, ref, emb = case
    assert np.array_equal(emb.cell_class, ref.cell_class)
    cellv = np.prod(V[conn[0, :8]].max(0) - V[conn[0, :8]].min(0))
    assert np.abs(emb.cut_volume - ref.cut_volume).max() <= 1e-13 * cellv
    vol = H.scenes.tet_mesh_volume_moments(X, T)[0]
    assert abs(emb.cut_volume.sum() / vol - 1) < 1e-13


@pytest.mark.parametrize("strength", [1, 3, 5])
def test_interface_rule_moments_match_oracle(case, strength):
    V, conn, X, T, ref, emb = case
    tq = H.tet_quadrature_strength(strength)
    o_g, w_g, p_g = H.embedding.compute_interface_quadrature_rules(emb, tq)
    o_r, w_r, p_r = ref.interface_quadratures(*tq)
    assert len(o_g) == len(o_r) == len(emb.interface_cells) + 1
    assert np.all(w_g >= 0) and np.all(np.abs(p_g) <= 1 + 1e-12)
    Mg, Mr = _rule_moments(o_g, w_g, p_g, strength), _rule_moments(o_r, w_r, p_r, strength)
    scale = Mr[:, :1]  # total weight of each rule
    assert np.all(np.abs(Mg - Mr) <= 1e-12 * scale)


def test_stabilization_points_are_appended(case):
    V, conn, X, T, ref, emb = case
    tq = H.tet_quadrature_strength(2)
    hw, hp = H.scenes.hex27_box(1.0, 1, 1, 1, 1).blocks[0].weights, H.scenes.hex27_box(1.0, 1, 1, 1, 1).blocks[0].points
    o0, w0, p0 = H.embedding.compute_interface_quadrature_rules(emb, tq)
    st = H.StabilizationOptions(1e-3, (hw, hp))
    o1, w1, p1 = H.embedding.compute_interface_quadrature_rules(emb, tq, st)
    assert np.array_equal(np.diff(o1), np.diff(o0) + len(hw))
    for k in range(len(o1) - 1):
        n0 = o0[k + 1] - o0[k]
        assert np.array_equal(w1[o1[k]:o1[k] + n0], w0[o0[k]:o0[k + 1]])
        assert np.array_equal(p1[o1[k]:o1[k] + n0], p0[o0[k]:o0[k + 1]])
        assert np.array_equal(w1[o1[k] + n0:o1[k + 1]], 1e-3 * hw)
        assert np.array_equal(p1[o1[k] + n0:o1[k + 1]], hp)


@pytest.mark.parametrize("strength", [2, 3, 5])
def test_simplification_keeps_moments(case, strength):
    V, conn, X, T, ref, emb = case
    o, w, p = H.embedding.compute_interface_quadrature_rules(emb, H.tet_quadrature_strength(3))
    oo, ow, op = H.embedding.simplify_rules(o, w, p, strength)
    r = len(list(x for x in itertools.product(range(strength + 1), repeat=3) if sum(x) <= strength))
    counts = np.diff(oo)
    assert np.all(counts <= np.maximum(r, 0)) or np.all((counts <= r) | (counts == np.diff(o)))
    assert np.all(ow > 0)
    ro, rw, rp = O.simplify_quadratures(o, w, p, strength)
    for k in range(len(o) - 1):
        pk, wk = p[o[k]:o[k + 1]], w[o[k]:o[k + 1]]
        sel = op[oo[k]:oo[k + 1]]
        idx = [int(np.nonzero((pk == q).all(1))[0][0]) for q in sel]
        assert idx == sorted(idx)
        P = O.moment_matrix(pk, strength)
        m0 = P @ wk
        assert np.abs(P[:, idx] @ ow[oo[k]:oo[k + 1]] - m0).max() <= 1e-12 * np.abs(m0).max()
        # the oracle's reduction keeps the same moments
        ridx = [int(np.nonzero((pk == q).all(1))[0][0]) for q in rp[ro[k]:ro[k + 1]]]
        assert np.abs(P[:, ridx] @ rw[ro[k]:ro[k + 1]] - m0).max() <= 1e-12 * np.abs(m0).max()


def test_empty_embedding_and_far_mesh():
    V, conn = _grid(3)
    X = np.array([[5.0, 5.0, 5.0], [6.0, 5.0, 5.0], [5.0, 6.0, 5.0], [5.0, 5.0, 6.0]])
    emb = H.embed_mesh_3d(V, conn, X, np.array([[0, 1, 2, 3]]))
    assert len(emb.exterior_cells) == 27 and emb.cut_volume.sum() == 0.0
    emb = H.embed_mesh_3d(V, conn, np.zeros((0, 3)), np.zeros((0, 4), dtype=np.int64))
    assert len(emb.exterior_cells) == 27
    o, w, p = H.embedding.compute_interface_quadrature_rules(emb, H.tet_quadrature_strength(1))
    assert len(o) == 1 and len(w) == 0


def test_cut_cell_cylinder_newton_step_matches_oracle():
    e = H.scenes.embedded_cylinder_cut(6, n_r=1, n_theta=32, n_z=12)
    b0, b1 = e.blocks
    m = H.EmbeddedModel3d(e.vertices, b0.connectivity, b1.connectivity, (b0.weights, b0.points),
                          (b1.offsets, b1.weights, b1.points))
    mat = H.StVKMaterial(H.YoungPoisson(5e5, 0.45))
    ref = O.Scene(e.vertices)
    ref.add_block(O.ELEM_HEX27, b0.connectivity, b0.weights, b0.points)
    ref.add_block(O.ELEM_HEX27, b1.connectivity, b1.weights, b1.points, qoff=b1.offsets)
    ref.finalize_pattern()
    ref.set_material(O.MAT_STVK, mat.lame.mu, mat.lame.lam, 1000.0)
    bc = e.nodes_below(2, 1e-9)
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(m, e.volume_fractions, 0.5)
    P = comp.build(m)
    integ = H.NewtonCgIntegrator3d(m, mat, 1000.0, bc, preconditioner=P)
    ref.set_bc(bc)
    ref.set_gravity(True)
    ref.set_schwarz(comp.schwarz_connectivity, comp.untreated_nodes)
    ref.set_solver(1e-5, 500, 100)
    ref.setup()
    u0 = H.scenes.random_normal(1, m.ndof(), 0.01 * e.cell_size)
    v0 = np.zeros(m.ndof())
    u, v = u0.copy(), v0.copy()
    st = integ.step(u, v, 0.0, 1e-3)
    ur, vr, rs = ref.step(u0, v0, 0.0, 1e-3)
    assert rs["status"] == 0
    assert st["newton_iterations"] == rs["newton_iters"]
    assert rel(u, ur) < 1e-8 and rel(v, vr) < 1e-8
