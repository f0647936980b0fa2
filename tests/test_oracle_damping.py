"""Oracle: element-wise PSD projection of the stiffness (DefaultSemidefiniteProjection,
fenris/src/assembly.rs:549-564) and the damping matrix D = gamma M + alpha K_proj
(compute_damping_matrix_into, simulation_toolbox/src/fem/system_assembly.rs:145-193)."""
import numpy as np
import scipy.sparse as sp

import higher_order_embedded_fem_b200 as H
from oracle import oracle as O


def _scene(cpu=2, mat_kind=O.MAT_SNH):
    s = H.scenes.tet10_box(1.0, 1, 1, 1, cpu)
    b = s.blocks[0]
    ref = O.Scene(s.vertices)
    ref.add_block(O.ELEM_TET10, b.connectivity, b.weights, b.points)
    ref.finalize_pattern()
    mu, lam = O.lame(1e6, 0.4)
    ref.set_material(mat_kind, mu, lam, 1000.0)
    return s, ref


def test_projection_keeps_psd_stiffness_and_makes_indefinite_psd():
    s, ref = _scene()
    n = 3 * s.vertices.shape[0]
    ro, ci = ref.pattern()
    # at rest the element tangents are PSD: the projection changes nothing beyond rounding
    K0 = ref.stiffness(np.zeros(n))
    P0 = ref.stiffness_projected(np.zeros(n))
    assert np.abs(P0 - K0).max() <= 1e-9 * np.abs(K0).max()
    # strongly compressed state: indefinite element tangents
    u = -0.45 * s.vertices.reshape(-1) + H.scenes.random_normal(3, n, 0.05 * s.cell_size)
    K = sp.csr_matrix((ref.stiffness(u), ci, ro), shape=(n, n))
    P = sp.csr_matrix((ref.stiffness_projected(u), ci, ro), shape=(n, n))
    lk = np.linalg.eigvalsh(K.toarray())
    lp = np.linalg.eigvalsh(P.toarray())
    assert lk.min() < -1e-6 * np.abs(lk).max()
    assert lp.min() >= -1e-10 * np.abs(lp).max()
    assert np.abs((P - P.T).toarray()).max() <= 1e-12 * np.abs(lp).max()


def test_damping_matrix_combination():
    s, ref = _scene()
    n = 3 * s.vertices.shape[0]
    ref.set_bc(s.nodes_below(2, 1e-9))
    ref.setup()
    u = H.scenes.random_normal(5, n, 0.01 * s.cell_size)
    ref.set_damping(mass=0.3, stiffness=0.02)
    D = ref.damping(u)
    want = 0.02 * ref.stiffness_projected(u) + 0.3 * ref.mass()
    assert np.abs(D - want).max() <= 1e-14 * np.abs(want).max()
    ref.set_damping(mass=None, stiffness=0.02)
    assert np.abs(ref.damping(u) - 0.02 * ref.stiffness_projected(u)).max() <= 1e-14 * np.abs(want).max()


def test_damped_step_dissipates():
    s, ref = _scene()
    n = 3 * s.vertices.shape[0]
    ref.set_bc(s.nodes_below(2, 1e-9))
    ref.set_gravity(False)
    ref.set_solver(1e-8, 1000, 100)
    ref.setup()
    u0 = np.zeros(n)
    v0 = H.scenes.random_normal(7, n, 0.1)
    _, v_plain, st = ref.step(u0, v0, 0.0, 1e-3)
    assert st["status"] == 0
    ref.set_damping(mass=5.0, stiffness=None)
    _, v_damped, st = ref.step(u0, v0, 0.0, 1e-3)
    assert st["status"] == 0
    M = sp.csr_matrix((ref.mass(), ref.pattern()[1], ref.pattern()[0]), shape=(n, n))
    assert v_damped @ (M @ v_damped) < v_plain @ (M @ v_plain)
