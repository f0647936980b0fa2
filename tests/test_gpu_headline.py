"""Parity at the benchmark's own sizes and on the Newton paths the small
scenes do not reach, against the FP64 oracle (the CPU restatement of the
reference path).

* The embedded Hex27 hollow cylinder 24^3 (132,888 DOFs, 22.3 M non-zeros,
  1,728 Schwarz subdomains), one backward-Euler step dt = 1e-3, CG to 1e-6:
  the plain FP64 step (both CG engines) and the mixed-precision step against
  the oracle's step on the same inputs, built independently on the oracle side
  (oracle/scenes.py).  Tolerances: Newton iteration counts equal, total CG
  iterations within 2 %; u within 1e-8 and v within 1e-6 relative (FP64) --
  both solvers stop at the reference's Newton tolerance dt 1e-5 ||M a|| with
  CG at 1e-6, so the two end states agree to that tolerance, not to rounding;
  the mixed step within 1e-6 (u) and 1e-4 (v).
* The Tet10 box 40 x 40 x 21 x 6 (201,600 elements, 846,369 DOFs, 70.9 M
  non-zeros): CSR pattern bit-exact, FP64 forces and stiffness within 1e-10,
  FP32 element stiffness within 1e-5.
* Backtracking line search (hamilton2/src/newton.rs:171-248) and substep
  retries (simulation_toolbox/src/fem/newton_cg.rs:146-228) on small Tet10
  boxes: the same number of alpha reductions, Newton iterations and substeps
  as the oracle, u and v within 1e-8.
"""
import numpy as np
import pytest

import higher_order_embedded_fem_b200 as H
from oracle import oracle as O
from oracle import scenes as OS

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


@pytest.fixture(scope="module")
def cylinder24():
    n, seed = 24, 2
    sc = OS.embedded_cylinder(n, 0.3, 0.4, 8, 27, seed)
    u0, v0 = OS.sway_state(sc, 0.02, 0.01, 1000 + seed)
    ref = OS.cylinder_reference_scene(sc, cg_tol=1e-6)
    ur, vr, rs = ref.step(u0, v0, 0.0, 1e-3)
    assert rs["status"] == 0
    e = H.scenes.embedded_cylinder(n, 0.3, 0.4, 8, 27, seed)
    b0, b1 = e.blocks
    model = H.EmbeddedModel3d(e.vertices, b0.connectivity, b1.connectivity, (b0.weights, b0.points),
                              (b1.offsets, b1.weights, b1.points))
    mat = H.StVKMaterial(H.YoungPoisson(5e5, 0.45))
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(model, e.volume_fractions, 0.5)
    P = comp.build(model)
    integ = H.NewtonCgIntegrator3d(model, mat, 1000.0, e.nodes_below(2, 1e-9), preconditioner=P)
    integ.set_tolerances(1e-6, 500, 100)
    return dict(u0=u0, v0=v0, ur=ur, vr=vr, rs=rs, integ=integ, model=model)


@pytest.mark.parametrize("engine", ["chunked", "streamed"])
def test_headline_cylinder_fp64_step_matches_oracle(cylinder24, engine):
    c = cylinder24
    integ = c["integ"]
    integ.set_precision(False, 0.1)
    integ.set_cg_engine(engine)
    u, v = c["u0"].copy(), c["v0"].copy()
    st = integ.step(u, v, 0.0, 1e-3)
    rs = c["rs"]
    assert st["newton_iterations"] == rs["newton_iters"]
    assert st["substeps"] == rs["substeps"] == 1
    assert abs(st["total_cg_iterations"] - sum(rs["cg_iters"])) <= 0.02 * sum(rs["cg_iters"])
    eu, ev = rel(u, c["ur"]), rel(v, c["vr"])
    print("cylinder 24^3 FP64 (%s): u %.2e v %.2e, CG %d vs %d" % (engine, eu, ev, st["total_cg_iterations"],
                                                                     sum(rs["cg_iters"])))
    assert eu < 1e-8 and ev < 1e-6


@pytest.mark.parametrize("fp16", [False, True])
def test_headline_cylinder_mixed_step_vs_oracle(cylinder24, fp16):
    c = cylinder24
    integ = c["integ"]
    integ.set_precision(True, 0.1)
    integ.set_cg_engine("streamed", fp16)
    u, v = c["u0"].copy(), c["v0"].copy()
    st = integ.step(u, v, 0.0, 1e-3)
    rs = c["rs"]
    assert st["residual_norm"] <= 1e-3 * 1e-5 * st["representative_force"]
    assert st["newton_iterations"] == rs["newton_iters"]
    eu, ev = rel(u, c["ur"]), rel(v, c["vr"])
    print("cylinder 24^3 mixed%s: u %.2e v %.2e, CG %d vs %d" % (" fp16" if fp16 else "", eu, ev,
                                                                  st["total_cg_iterations"], sum(rs["cg_iters"])))
    assert eu < 1e-6 and ev < 1e-4
    integ.set_precision(False, 0.1)


def test_config3_tet10_box_pattern_and_element_parity():
    s = H.scenes.tet10_box(0.025, 40, 40, 21, 1)
    b = s.blocks[0]
    model = H.NodalModel3d(s.vertices, b.connectivity, (b.weights, b.points))
    assert model.num_elements == 201600 and model.ndof() == 846369 and model.nnz == 70917201
    mat = H.StableNeoHookeanMaterial(H.YoungPoisson(1e6, 0.4))
    ref = O.Scene(s.vertices)
    ref.add_block(O.ELEM_TET10, b.connectivity, b.weights, b.points)
    ref.finalize_pattern()
    ref.set_material(O.MAT_SNH, mat.lame.mu, mat.lame.lam, 1000.0)
    ro, ci = model.pattern()
    rro, rci = ref.pattern()
    assert np.array_equal(ro, rro) and np.array_equal(ci, rci)
    del rci, ci
    u0 = H.scenes.random_normal(2, model.ndof(), 0.02 * 0.025)
    fr, Kr = ref.forces(u0), ref.stiffness(u0)
    f = model.assemble_elastic_pseudo_forces_into_par(np.zeros(model.ndof()), u0, mat)
    K64 = model.assemble_stiffness_into_par(np.zeros(model.nnz), u0, mat)
    K32 = model.assemble_stiffness_into_precision(np.zeros(model.nnz), u0, mat, True)
    ef, e64, e32 = rel(f, fr), rel(K64, Kr), rel(K32, Kr)
    print("Tet10 box 201,600: forces %.2e stiffness FP64 %.2e FP32 %.2e" % (ef, e64, e32))
    assert ef < 1e-10 and e64 < 1e-10 and e32 < 1e-5


def tet10_scene(cpu, amp):
    s = H.scenes.tet10_box(1.0, 1, 1, 1, cpu)
    b = s.blocks[0]
    model = H.NodalModel3d(s.vertices, b.connectivity, (b.weights, b.points))
    mat = H.StableNeoHookeanMaterial(H.YoungPoisson(1e6, 0.4))
    bc = s.nodes_below(2, 1e-9)
    ref = O.Scene(s.vertices)
    ref.add_block(O.ELEM_TET10, b.connectivity, b.weights, b.points)
    ref.finalize_pattern()
    ref.set_material(O.MAT_SNH, mat.lame.mu, mat.lame.lam, 1000.0)
    ref.set_bc(bc)
    ref.set_gravity(True)
    # compressed along z and swayed in x: the first Newton steps overshoot
    X = s.vertices
    u0 = np.zeros_like(X)
    u0[:, 2] = -amp * X[:, 2]
    u0[:, 0] = 0.5 * amp * X[:, 2] ** 2
    return model, mat, bc, ref, u0.reshape(-1)


@pytest.mark.parametrize("engine", ["chunked", "streamed"])
def test_line_search_backtracking_matches_oracle(engine):
    model, mat, bc, ref, u0 = tet10_scene(3, 0.2)
    dt = 5e-2
    ref.set_solver(1e-5, 500, 100)
    ref.setup()
    ur, vr, rs = ref.step(u0, np.zeros_like(u0), 0.0, dt)
    assert rs["status"] == 0 and rs["ls_backtracks"] > 0 and rs["substeps"] == 1
    integ = H.NewtonCgIntegrator3d(model, mat, 1000.0, bc)
    integ.set_cg_engine(engine)
    u, v = u0.copy(), np.zeros_like(u0)
    st = integ.step(u, v, 0.0, dt)
    assert st["line_search_backtracks"] == rs["ls_backtracks"]
    assert st["newton_iterations"] == rs["newton_iters"] and st["substeps"] == 1
    assert rel(u, ur) < 1e-8 and rel(v, vr) < 1e-8


@pytest.mark.parametrize("engine", ["chunked", "streamed"])
def test_failed_attempt_recovers_with_substeps_matches_oracle(engine):
    # Newton limited to 3 iterations: the full step needs 4, so the first
    # attempt fails and the step is retried as 5 substeps of dt / 5
    model, mat, bc, ref, u0 = tet10_scene(3, 0.1)
    dt = 5e-2
    ref.set_solver(1e-5, 500, 3)
    ref.setup()
    ur, vr, rs = ref.step(u0, np.zeros_like(u0), 0.0, dt)
    assert rs["status"] == 0 and rs["substeps"] == 5
    integ = H.NewtonCgIntegrator3d(model, mat, 1000.0, bc)
    integ.set_tolerances(1e-5, 500, 3)
    integ.set_cg_engine(engine)
    u, v = u0.copy(), np.zeros_like(u0)
    st = integ.step(u, v, 0.0, dt)
    assert st["substeps"] == 5 and st["newton_iterations"] == rs["newton_iters"]
    assert rel(u, ur) < 1e-8 and rel(v, vr) < 1e-8
