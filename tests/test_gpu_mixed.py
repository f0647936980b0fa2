"""Mixed-precision variant vs the FP64 oracle: FP32 element stiffness within
1e-5 relative, FP32-operator CG inside FP64 iterative refinement reaching the
FP64 tolerance on the true residual, and the mixed Newton step."""
import numpy as np
import pytest

import higher_order_embedded_fem_b200 as H
from oracle import oracle as O

from test_gpu_parity import embedded_setup, rel, tet10_setup

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mat_kind", [O.MAT_SNH, O.MAT_STVK])
def test_fp32_stiffness_error_tet10(mat_kind):
    s, m, mat, ref = tet10_setup(8, mat_kind)
    u = H.scenes.random_normal(1, m.ndof(), 0.01 * s.cell_size)
    K32 = m.assemble_stiffness_into_precision(np.zeros(m.nnz), u, mat, True)
    err = rel(K32, ref.stiffness(u))
    assert err < 1e-5, err


@pytest.mark.parametrize("mat_kind", [O.MAT_SNH, O.MAT_STVK])
def test_fp32_stiffness_error_embedded(mat_kind):
    e, m, mat, ref = embedded_setup(8, mat_kind)
    u = H.scenes.random_normal(3, m.ndof(), 0.01 * e.cell_size)
    K32 = m.assemble_stiffness_into_precision(np.zeros(m.nnz), u, mat, True)
    err = rel(K32, ref.stiffness(u))
    assert err < 1e-5, err


def test_mixed_cg_reaches_fp64_tolerance():
    e, m, mat, ref = embedded_setup(8)
    u = H.scenes.random_normal(3, m.ndof(), 0.001 * e.cell_size)
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(m, e.volume_fractions, 0.5)
    bc = e.nodes_below(2, 1e-9)
    ref.set_bc(bc)
    ref.setup()
    J = ref.jacobian(ref.stiffness(u), 1e-3)
    P = comp.build(m)
    P.update(J)
    b = H.scenes.random_normal(6, m.ndof(), 1.0)
    b[np.repeat(3 * bc, 3) + np.tile(np.arange(3), bc.size)] = 0.0
    x = np.zeros(m.ndof())
    out = (H.ConjugateGradient(m).with_operator(J).with_preconditioner(P)
           .with_stopping_criterion(H.RelativeResidualCriterion(1e-6)).with_max_iter(2000)
           .solve_with_guess_mixed(b, x, 0.1))
    y = m.spmv(np.zeros(m.ndof()), J, x)
    assert np.linalg.norm(y - b) <= 1e-6 * np.linalg.norm(b)
    x64 = np.zeros(m.ndof())
    out64 = (H.ConjugateGradient(m).with_operator(J).with_preconditioner(P)
             .with_stopping_criterion(H.RelativeResidualCriterion(1e-6)).with_max_iter(2000)
             .solve_with_guess(b, x64))
    assert rel(x, x64) < 1e-4
    assert out.num_iterations <= 3 * out64.num_iterations


def test_mixed_newton_step_matches_oracle():
    e, m, mat, ref = embedded_setup(6)
    bc = e.nodes_below(2, 1e-9)
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(m, e.volume_fractions, 0.5)
    P = comp.build(m)
    integ = H.NewtonCgIntegrator3d(m, mat, 1000.0, bc, preconditioner=P)
    integ.set_tolerances(1e-6, 500, 100)
    integ.set_precision(True, 0.1)
    ref.set_bc(bc)
    ref.set_gravity(True)
    ref.set_schwarz(comp.schwarz_connectivity, comp.untreated_nodes)
    ref.set_solver(1e-6, 500, 100)
    ref.setup()
    X = e.vertices
    u0 = np.zeros_like(X)
    u0[:, 0] = 0.02 * X[:, 2] ** 2
    u0 = u0.reshape(-1) + H.scenes.random_normal(1, m.ndof(), 0.001 * e.cell_size)
    v0 = np.zeros(m.ndof())
    u, v = u0.copy(), v0.copy()
    st = integ.step(u, v, 0.0, 1e-3)
    ur, vr, rs = ref.step(u0, v0, 0.0, 1e-3)
    assert rs["status"] == 0
    assert st["residual_norm"] <= 1e-3 * 1e-5 * st["representative_force"]
    assert rel(u, ur) < 1e-6 and rel(v, vr) < 1e-4
