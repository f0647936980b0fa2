"""Damping on the GPU vs the FP64 oracle: element-wise PSD-projected stiffness
(DefaultSemidefiniteProjection), the damped Jacobian combination and damped
backward-Euler Newton steps (compute_damping_matrix_into)."""
import numpy as np
import pytest

import higher_order_embedded_fem_b200 as H
from oracle import oracle as O

from test_gpu_parity import embedded_setup, rel, tet10_setup

pytestmark = pytest.mark.gpu


def test_projected_stiffness_tet10_matches_oracle():
    s, m, mat, ref = tet10_setup(3)
    n = m.ndof()
    # compressed state: many element tangents indefinite
    u = -0.45 * s.vertices.reshape(-1) + H.scenes.random_normal(3, n, 0.05 * s.cell_size)
    got = m.assemble_projected_stiffness_into_par(np.zeros(m.nnz), u, mat)
    want = ref.stiffness_projected(u)
    assert rel(got, want) < 1e-10
    assert rel(m.assemble_stiffness_into_par(np.zeros(m.nnz), u, mat), want) > 1e-6  # the projection acted


def test_projected_stiffness_embedded_hex27_matches_oracle():
    e, m, mat, ref = embedded_setup(4, O.MAT_SNH)
    u = -0.3 * e.vertices.reshape(-1) + H.scenes.random_normal(4, m.ndof(), 0.02 * e.cell_size)
    got = m.assemble_projected_stiffness_into_par(np.zeros(m.nnz), u, mat)
    assert rel(got, ref.stiffness_projected(u)) < 1e-10


def test_damped_jacobian_combination():
    s, m, mat, ref = tet10_setup(3)
    bc = s.nodes_below(2, 1e-9)
    ref.set_bc(bc)
    ref.setup()
    u = H.scenes.random_normal(1, m.ndof(), 0.01 * s.cell_size)
    K, M = ref.stiffness(u), ref.mass()
    ref.set_damping(mass=0.2, stiffness=0.01)
    D = ref.damping(u)
    dt = 1e-3
    J = m.jacobian_combination_damped(np.zeros(m.nnz), dt * dt, K, dt, D, 1.0, M, bc)
    ro, ci = m.pattern()
    want = O.dirichlet_csr(ro, ci, (dt * dt) * K + dt * D + 1.0 * M, bc, 3)
    assert rel(J, want) < 1e-14


@pytest.mark.parametrize("damping", [(0.5, None), (None, 0.02), (0.3, 0.01)])
def test_damped_newton_step_tet10_matches_oracle(damping):
    s, m, mat, ref = tet10_setup(3)
    bc = s.nodes_below(2, 1e-9)
    u0 = H.scenes.random_normal(1, m.ndof(), 0.01 * s.cell_size)
    v0 = H.scenes.random_normal(2, m.ndof(), 0.05)
    integ = H.NewtonCgIntegrator3d(m, mat, 1000.0, bc)
    integ.set_damping(*damping)
    ref.set_bc(bc)
    ref.set_gravity(True)
    ref.set_solver(1e-5, 500, 100)
    ref.set_damping(*damping)
    ref.setup()
    u, v = u0.copy(), v0.copy()
    st = integ.step(u, v, 0.0, 1e-3)
    ur, vr, rs = ref.step(u0, v0, 0.0, 1e-3)
    assert rs["status"] == 0
    assert st["newton_iterations"] == rs["newton_iters"]
    assert rel(u, ur) < 1e-8 and rel(v, vr) < 1e-8
    # damping changes the step
    integ.set_damping(None, None)
    u2, v2 = u0.copy(), v0.copy()
    integ.step(u2, v2, 0.0, 1e-3)
    assert rel(v2, vr) > 1e-6


def test_damped_newton_step_embedded_schwarz_matches_oracle():
    e, m, mat, ref = embedded_setup(4)
    bc = e.nodes_below(2, 1e-9)
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(m, e.volume_fractions, 0.5)
    P = comp.build(m)
    integ = H.NewtonCgIntegrator3d(m, mat, 1000.0, bc, preconditioner=P)
    integ.set_damping(0.1, 0.005)
    ref.set_bc(bc)
    ref.set_gravity(True)
    ref.set_schwarz(comp.schwarz_connectivity, comp.untreated_nodes)
    ref.set_solver(1e-5, 500, 100)
    ref.set_damping(0.1, 0.005)
    ref.setup()
    u0 = H.scenes.random_normal(1, m.ndof(), 0.01 * e.cell_size)
    v0 = H.scenes.random_normal(2, m.ndof(), 0.05)
    u, v = u0.copy(), v0.copy()
    st = integ.step(u, v, 0.0, 1e-3)
    ur, vr, rs = ref.step(u0, v0, 0.0, 1e-3)
    assert rs["status"] == 0
    assert st["newton_iterations"] == rs["newton_iters"]
    assert rel(u, ur) < 1e-8 and rel(v, vr) < 1e-8
