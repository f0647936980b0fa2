"""Pins the oracle to the reference's own known answers (tests/golden, read
from the reference's test sources) and to the consistency properties its
tests check (finite differences, batch vs pairwise contraction)."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_vectors.json")))


def test_mock_patterns_golden():
    # fenris/tests/unit_tests/assembly.rs:552-621
    for c in GOLD["mock_patterns"]:
        ro, ci = O.pattern(c["elements"], c["solution_dim"], c["num_nodes"])
        assert ro.tolist() == c["row_offsets"]
        assert ci.tolist() == c["col_indices"]


def test_dirichlet_csr_golden():
    # fenris/tests/unit_tests/assembly.rs:318-345
    d = GOLD["dirichlet_example"]
    n = d["n"]
    ro = np.arange(0, n * n + 1, n)
    ci = np.tile(np.arange(n), n)
    v = O.dirichlet_csr(ro, ci, np.full(n * n, d["fill"]), d["nodes"], d["dim"])
    expected = np.array(d["expected_column_major"]).reshape(n, n).T
    assert np.array_equal(v.reshape(n, n), expected)


def _mats():
    m = GOLD["materials"]
    Fs = [np.array(F).reshape(3, 3) for F in m["deformation_gradients_row_major"]]
    vecs = [np.array(v) for v in m["vectors"]]
    lames = [O.lame(p["young"], p["poisson"]) for p in m["young_poisson"]]
    return Fs, vecs, lames


def _fd_contraction(kind, mu, lam, F, a, b, h=1e-6):
    # approximate_stiffness_contraction, materials.rs:818-859
    r = np.zeros((3, 3))
    for i in range(3):
        for j in range(3):
            for l in range(3):
                for n in range(3):
                    e = np.zeros((3, 3))
                    e[j, n] = 1.0
                    d = (O.stress(kind, mu, lam, F + h * e)[i, l] - O.stress(kind, mu, lam, F - h * e)[i, l]) / (2 * h)
                    r[i, j] += d * a[l] * b[n]
    return r


@pytest.mark.parametrize("kind", [O.MAT_SNH, O.MAT_STVK, O.MAT_LINEAR])
def test_contraction_consistent_with_finite_difference(kind):
    # fenris/tests/unit_tests/materials.rs:12-42 (scale * h tolerance)
    Fs, vecs, lames = _mats()
    h = 1e-6
    for mu, lam in lames:
        for F in Fs:
            for a in vecs:
                for b in vecs:
                    fd = _fd_contraction(kind, mu, lam, F, a, b, h)
                    c = O.contract(kind, mu, lam, F, a, b)
                    scale = max(np.abs(fd).max(), np.abs(c).max())
                    assert np.abs(fd - c).max() <= scale * h


@pytest.mark.parametrize("kind", [O.MAT_SNH, O.MAT_STVK, O.MAT_LINEAR])
def test_contraction_batch_consistency(kind):
    # fenris/tests/unit_tests/materials.rs:45-93: batch ADDS into pre-filled output
    Fs, vecs, lames = _mats()
    A = np.array(vecs).T.copy()  # 3 x n
    n = A.shape[1]
    for mu, lam in lames:
        for F in Fs:
            ref = np.full((3 * n, 3 * n), 4.0)
            for i in range(n):
                for j in range(n):
                    ref[3 * i:3 * i + 3, 3 * j:3 * j + 3] += O.contract(kind, mu, lam, F, A[:, i], A[:, j])
            out = np.full((3 * n, 3 * n), 4.0)
            O.contract_multiple(kind, mu, lam, F, A, out)
            scale = max(np.abs(ref).max(), np.abs(out).max())
            assert np.abs(ref - out).max() <= 1e-12 * scale


def test_snh_dp_df_symmetric_and_matches_contraction():
    # materials.rs:955-989 pins dp/df through its eigen-decomposition; here the
    # matrix is checked for symmetry and against the pairwise contraction.
    s = GOLD["snh_analytic"]
    mu, lam = O.lame(s["young"], s["poisson"])
    F = np.array(s["F_row_major"]).reshape(3, 3)
    C = O.snh_dp_df(mu, lam, F)
    assert np.abs(C - C.T).max() <= 1e-12 * np.abs(C).max()
    rng = np.random.default_rng(0)
    for _ in range(5):
        a, b = rng.standard_normal(3), rng.standard_normal(3)
        via_C = np.einsum("kilj,k,l->ij", C.reshape(3, 3, 3, 3), a, b)
        assert np.allclose(via_C, O.contract(O.MAT_SNH, mu, lam, F, a, b), rtol=1e-12, atol=1e-12 * np.abs(C).max())


def test_lame_reference_conversion():
    mu, lam = O.lame(1e6, 0.4)
    assert mu == 0.5 * 1e6 / 1.4
    assert lam == 0.5 * mu * 0.4 / (1.0 - 0.8)


def test_cg_dense_golden():
    # fenris/tests/unit_tests/cg.rs:18-58
    c = GOLD["cg"]["arbitrary"]
    A = np.full((3, 3), c["off"])
    np.fill_diagonal(A, c["diag"])
    x0 = np.array(c["x0"])
    st, x, it = O.cg_dense(A, A @ x0, np.zeros(3), c["tol"])
    assert st == 0 and 0 < it <= 3 and np.abs(x - x0).max() <= 1e-12
    c = GOLD["cg"]["preconditioned"]
    A = np.array(c["A_row_major"]).reshape(3, 3)
    P = np.array(c["P_row_major"]).reshape(3, 3)
    x0 = np.array(c["x0"])
    st, x, it = O.cg_dense(A, A @ x0, np.array(c["guess"]), c["tol"], P=P)
    assert st == 0 and it == c["iterations"] and np.abs(x - x0).max() <= 1e-12


def test_cg_identity_and_error_kinds():
    # solve_identity (cg.rs tests) and SolveErrorKind outcomes
    st, x, it = O.cg_dense(np.eye(4), np.full(4, 5.0), np.zeros(4), 1e-8)
    assert st == 0 and np.array_equal(x, np.full(4, 5.0))
    A = np.diag([1.0, 2.0, 3.0, 4.0])
    st, x, it = O.cg_dense(A, np.ones(4), np.zeros(4), 1e-14, max_iter=1)
    assert st == 3 and it == 1
    st, x, it = O.cg_dense(-A, np.ones(4), np.zeros(4), 1e-14)
    assert st == 1 and it == 0


def test_block_inverse_matches_dense_inverse_on_spd():
    # The Schwarz block rule reduces to the inverse for SPD blocks
    # (schwarz_precond.rs:329-342); golden 9x9 block-preconditioner matrix
    # (newton_cg.rs:827-876) made SPD by symmetrisation + shift.
    M = np.array(GOLD["block_preconditioner"]["matrix_row_major"]).reshape(9, 9)
    S = 0.5 * (M + M.T) + 60 * np.eye(9)
    P = O.invert_block(S)
    assert np.abs(P - np.linalg.inv(S)).max() <= 1e-13 * np.abs(np.linalg.inv(S)).max()
    # indefinite block: |lambda| flip
    w, V = np.linalg.eigh(0.5 * (M + M.T))
    P = O.invert_block(0.5 * (M + M.T))
    assert np.allclose(P, (V / np.abs(w)) @ V.T, rtol=1e-10, atol=1e-12)


def test_quadrature_tables_are_exact():
    q = GOLD["quadrature"]
    t = q["tet_quadrature_strength_5"]
    assert abs(sum(t["weights"]) - 4.0 / 3.0) < 1e-14
    h = q["hex_quadrature_strength_5"]
    assert abs(sum(h["weights"]) - 8.0) < 1e-13
    # strength 5: integrates x^2 y^2 z exactly on the cube (odd -> 0), x^4 -> 8/5
    pts = np.array(h["points"])
    w = np.array(h["weights"])
    assert abs(np.sum(w * pts[:, 0] ** 4) - 8.0 / 5.0) < 1e-13
    assert abs(np.sum(w * pts[:, 0] ** 2 * pts[:, 1] ** 2) - 8.0 / 9.0) < 1e-13


@pytest.mark.parametrize("kind", [O.ELEM_TET10, O.ELEM_HEX27])
def test_lagrange_property_and_partition_of_unity(kind):
    # fenris/tests/unit_tests/element.rs:173-291,610-680
    if kind == O.ELEM_TET10:
        nodes = np.array([[-1, -1, -1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1], [0, -1, -1], [0, 0, -1], [-1, 0, -1],
                          [-1, -1, 0], [-1, 0, 0], [0, -1, 0]], dtype=float)
    else:
        from itertools import product  # noqa: F401
        nodes = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1], [-1, -1, 1], [1, -1, 1], [1, 1, 1],
                          [-1, 1, 1], [0, -1, -1], [-1, 0, -1], [-1, -1, 0], [1, 0, -1], [1, -1, 0], [0, 1, -1],
                          [1, 1, 0], [-1, 1, 0], [0, -1, 1], [-1, 0, 1], [1, 0, 1], [0, 1, 1], [0, 0, -1],
                          [0, -1, 0], [-1, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 0, 0]], dtype=float)
    for i, x in enumerate(nodes):
        N = O.basis(kind, x)
        e = np.zeros(len(nodes))
        e[i] = 1
        assert np.abs(N - e).max() < 1e-14
    rng = np.random.default_rng(1)
    for _ in range(10):
        xi = rng.uniform(-1, 1, 3)
        if kind == O.ELEM_TET10:
            xi = -1 + (xi + 1) / max(1.0, np.sum(xi + 1) / 2.0)
        assert abs(O.basis(kind, xi).sum() - 1) < 1e-13
        assert np.abs(O.gradients(kind, xi).sum(axis=1)).max() < 1e-13
        # gradient is the derivative of the basis
        h = 1e-6
        g = O.gradients(kind, xi)
        for d in range(3):
            e = np.zeros(3)
            e[d] = h
            fd = (O.basis(kind, xi + e) - O.basis(kind, xi - e)) / (2 * h)
            assert np.abs(fd - g[d]).max() < 1e-8


@pytest.mark.parametrize("kind,mat", [(O.ELEM_TET10, O.MAT_SNH), (O.ELEM_TET10, O.MAT_STVK),
                                      (O.ELEM_HEX27, O.MAT_STVK), (O.ELEM_HEX27, O.MAT_SNH)])
def test_element_stiffness_is_negative_derivative_of_forces(kind, mat):
    # fenris/tests/unit_tests/assembly.rs:390-520: K_e = -d f_e / d u
    q = GOLD["quadrature"]["tet_quadrature_strength_5" if kind == O.ELEM_TET10 else "hex_quadrature_strength_5"]
    w, p = np.array(q["weights"]), np.array(q["points"])
    n = O.NODES[kind]
    rng = np.random.default_rng(2)
    if kind == O.ELEM_TET10:
        ref = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]])
        X = np.vstack([ref, [(ref[a] + ref[b]) / 2 for a, b in [(0, 1), (1, 2), (0, 2), (0, 3), (2, 3), (1, 3)]]])
    else:
        X = (np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1.0]]))
        alpha = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1], [-1, -1, 1], [1, -1, 1], [1, 1, 1],
                          [-1, 1, 1], [0, -1, -1], [-1, 0, -1], [-1, -1, 0], [1, 0, -1], [1, -1, 0], [0, 1, -1],
                          [1, 1, 0], [-1, 1, 0], [0, -1, 1], [-1, 0, 1], [1, 0, 1], [0, 1, 1], [0, 0, -1],
                          [0, -1, 0], [-1, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0, 0, 0]], dtype=float)
        X = (alpha + 1) / 2
    X = X + 0.02 * rng.standard_normal(X.shape)
    ue = 0.05 * rng.standard_normal((3, n))
    mu, lam = O.lame(1e2, 0.3)
    K = O.element_stiffness(kind, X, ue, w, p, mat, mu, lam)
    h = 1e-6
    Kfd = np.zeros_like(K)
    for J in range(n):
        for j in range(3):
            up, um = ue.copy(), ue.copy()
            up[j, J] += h
            um[j, J] -= h
            df = (O.element_force(kind, X, up, w, p, mat, mu, lam) - O.element_force(kind, X, um, w, p, mat, mu, lam))
            Kfd[:, 3 * J + j] = -(df / (2 * h)).T.reshape(-1)
    assert np.abs(K - K.T).max() <= 1e-12 * np.abs(K).max()
    assert np.abs(K - Kfd).max() <= 1e-6 * np.abs(K).max()


def test_tet10_mesh_sizes():
    # 8x8x8 hexes -> Max triangulation -> Tet10: 4,913 nodes / 1,141,065 nnz
    t = O.tets_from_hex(O.hex_box(1.0, 1, 1, 1, 8), True)
    assert t.vertices.shape == (4913, 3) and t.cells.shape == (3072, 10)
    ro, ci = O.pattern(t.cells.tolist(), 3, 4913)
    assert ci.size == 1141065


def test_greedy_coloring_is_disjoint_and_first_fit():
    # paradis/src/coloring.rs:83-111 (disjointness) + first fit order
    rng = np.random.default_rng(3)
    for _ in range(20):
        subsets = [sorted(set(rng.integers(0, 100, rng.integers(0, 10)).tolist())) for _ in range(rng.integers(0, 10))]
        cols = O.coloring(subsets)
        assert sorted(x for c in cols for x in c) == list(range(len(subsets)))
        for c in cols:
            seen = set()
            for l in c:
                assert not (seen & set(subsets[l]))
                seen |= set(subsets[l])
        # first fit: an element is never placeable in an earlier color
        color_of = {l: k for k, c in enumerate(cols) for l in c}
        for l, s in enumerate(subsets):
            for k in range(color_of[l]):
                earlier = set(x for m in cols[k] if m < l for x in subsets[m])
                assert earlier & set(s)
