"""The persistent streamed CG (default engine) against the chunked-graph CG and
the FP64 oracle's PCG (fenris/src/cg.rs:376-482): same outcomes, iteration
counts within one, solutions to the solve's tolerance, deterministic results.

Tolerances: x within 1e-6 of the oracle's x at CG tolerance 1e-8 (as the
chunked engine's test), true residual ||b - A x|| <= tol ||b||.
"""
import numpy as np
import pytest

import higher_order_embedded_fem_b200 as H
from oracle import oracle as O

from test_gpu_parity import embedded_setup, rel, tet10_setup

pytestmark = pytest.mark.gpu


def schwarz_system(n=8, seed=3):
    # a small displacement (0.1 % of the cell size): the StVK Jacobian stays SPD
    e, m, mat, ref = embedded_setup(n)
    u = H.scenes.random_normal(seed, m.ndof(), 0.001 * e.cell_size)
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(m, e.volume_fractions, 0.5)
    bc = e.nodes_below(2, 1e-9)
    ref.set_bc(bc)
    ref.set_schwarz(comp.schwarz_connectivity, comp.untreated_nodes)
    ref.setup()
    J = ref.jacobian(ref.stiffness(u), 1e-3)
    ref.schwarz_update(J)  # the oracle's CG applies its own Schwarz values
    P = comp.build(m)
    P.update(J)
    b = H.scenes.random_normal(6, m.ndof(), 1.0)
    b[np.repeat(3 * bc, 3) + np.tile(np.arange(3), bc.size)] = 0.0
    return m, ref, P, J, b


def solve(m, J, P, b, tol, engine, mixed=False, fp16=False, max_iter=5000):
    m.set_cg_engine(engine, fp16)
    x = np.zeros(m.ndof())
    cg = (H.ConjugateGradient(m).with_operator(J).with_stopping_criterion(H.RelativeResidualCriterion(tol))
          .with_max_iter(max_iter))
    if P is not None:
        cg = cg.with_preconditioner(P)
    out = cg.solve_with_guess_mixed(b, x, 0.1) if mixed else cg.solve_with_guess(b, x)
    return x, out.num_iterations, m.cg_engine_stats()


def true_rel_residual(m, J, x, b):
    return np.linalg.norm(m.spmv(np.zeros(m.ndof()), J, x) - b) / np.linalg.norm(b)


def test_streamed_schwarz_cg_matches_chunked_and_oracle():
    m, ref, P, J, b = schwarz_system(8)
    xs, its, stats = solve(m, J, P, b, 1e-8, "streamed")
    assert stats["launches"] >= 1 and stats["iterations"] == its
    assert stats["operator_bytes"] > 8 * m.nnz
    xc, itc, stc = solve(m, J, P, b, 1e-8, "chunked")
    assert stc["launches"] == 0
    st, xr, itr = ref.cg(J, b, 1e-8, 5000)
    assert st == 0
    assert abs(its - itr) <= 1 and abs(itc - itr) <= 1
    assert rel(xs, xr) < 1e-6 and rel(xs, xc) < 1e-6
    assert true_rel_residual(m, J, xs, b) <= 1e-8 * 1.01


def test_streamed_cg_is_deterministic():
    m, ref, P, J, b = schwarz_system(6)
    x1, i1, _ = solve(m, J, P, b, 1e-8, "streamed")
    x2, i2, _ = solve(m, J, P, b, 1e-8, "streamed")
    assert i1 == i2 and np.array_equal(x1, x2)


def test_streamed_diagonal_and_identity_cg_match_oracle():
    s, m, mat, ref = tet10_setup(6)
    u = H.scenes.random_normal(1, m.ndof(), 0.01 * s.cell_size)
    bc = s.nodes_below(2, 1e-9)
    ref.set_bc(bc)
    ref.setup()
    J = ref.jacobian(ref.stiffness(u), 1e-3)
    b = H.scenes.random_normal(6, m.ndof(), 1.0)
    b[np.repeat(3 * bc, 3) + np.tile(np.arange(3), bc.size)] = 0.0
    D = H.DiagonalPreconditioner(m)
    D.update(J)
    xs, its, stats = solve(m, J, D, b, 1e-10, "streamed", max_iter=2000)
    st, xr, itr = ref.cg(J, b, 1e-10, 2000)
    assert st == 0 and stats["launches"] >= 1
    assert abs(its - itr) <= 1
    assert rel(xs, xr) < 1e-8
    # no preconditioner: against the chunked engine (the oracle's scene CG always
    # uses its preconditioner)
    xi, iti, _ = solve(m, J, None, b, 1e-8, "streamed", max_iter=5000)
    xc, itc, _ = solve(m, J, None, b, 1e-8, "chunked", max_iter=5000)
    assert abs(iti - itc) <= 1 and rel(xi, xc) < 1e-6
    assert true_rel_residual(m, J, xi, b) <= 1e-8 * 1.01


def test_streamed_cg_error_kinds():
    s, m, mat, ref = tet10_setup(3)
    ref.setup()
    J = ref.jacobian(ref.stiffness(np.zeros(m.ndof())), 1e-3)
    b = H.scenes.random_normal(6, m.ndof(), 1.0)
    m.set_cg_engine("streamed")
    with pytest.raises(H.SolveError) as ei:
        H.ConjugateGradient(m).with_operator(J).with_stopping_criterion(
            H.RelativeResidualCriterion(1e-14)).with_max_iter(2).solve_with_guess(b, np.zeros(m.ndof()))
    assert ei.value.kind == H.SolveErrorKind.MaxIterationsReached and ei.value.output.num_iterations == 2
    with pytest.raises(H.SolveError) as ei:
        H.ConjugateGradient(m).with_operator(-J).solve_with_guess(b, np.zeros(m.ndof()))
    assert ei.value.kind == H.SolveErrorKind.IndefiniteOperator and ei.value.output.num_iterations == 0


@pytest.mark.parametrize("fp16", [False, True])
def test_streamed_mixed_cg_reaches_fp64_tolerance(fp16):
    m, ref, P, J, b = schwarz_system(8)
    x64, it64, _ = solve(m, J, P, b, 1e-6, "streamed")
    xm, itm, stats = solve(m, J, P, b, 1e-6, "streamed", mixed=True, fp16=fp16)
    assert stats["launches"] >= 1
    assert true_rel_residual(m, J, xm, b) <= 1e-6
    assert rel(xm, x64) < 1e-4
    # FP32 values keep the iteration count; scaled FP16 Schwarz blocks cost a few
    assert itm <= (1.15 if fp16 else 1.05) * it64 + 3


@pytest.mark.parametrize("mixed", [False, True])
def test_streamed_and_chunked_newton_steps_agree(mixed):
    e, m, mat, ref = embedded_setup(6)
    bc = e.nodes_below(2, 1e-9)
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(m, e.volume_fractions, 0.5)
    P = comp.build(m)
    integ = H.NewtonCgIntegrator3d(m, mat, 1000.0, bc, preconditioner=P)
    integ.set_tolerances(1e-6, 500, 100)
    integ.set_precision(mixed, 0.1)
    u0 = H.scenes.random_normal(1, m.ndof(), 0.01 * e.cell_size)
    out = []
    for engine in ("streamed", "chunked"):
        integ.set_cg_engine(engine)
        u, v = u0.copy(), np.zeros(m.ndof())
        st = integ.step(u, v, 0.0, 1e-3)
        out.append((u, v, st, integ.cg_engine_stats()))
    (us, vs, ss, es), (uc, vc, sc, ec) = out
    assert es["launches"] >= ss["num_cg_solves"] and ec["launches"] == 0
    assert ss["newton_iterations"] == sc["newton_iterations"]
    assert abs(ss["total_cg_iterations"] - sc["total_cg_iterations"]) <= max(2, 0.03 * sc["total_cg_iterations"])
    assert rel(us, uc) < 1e-7 and rel(vs, vc) < 1e-5


def numpy_pcg_iterates(A, apply_p, b, k):
    """x after k iterations of the PCG recurrence of fenris/src/cg.rs:376-482."""
    x = np.zeros_like(b)
    r = b.copy()
    z = apply_p(r)
    p = z.copy()
    zr = z @ r
    for _ in range(k):
        Ap = A @ p
        alpha = zr / (p @ Ap)
        x += alpha * p
        r -= alpha * Ap
        z = apply_p(r)
        zn = z @ r
        p = z + (zn / zr) * p
        zr = zn
    return x


@pytest.mark.parametrize("engine", ["streamed", "chunked"])
@pytest.mark.parametrize("prec", ["none", "diagonal", "schwarz"])
def test_cg_first_iterates_match_numpy_recurrence(engine, prec):
    import scipy.sparse as sp

    m, ref, P, J, b = schwarz_system(6)
    ro, ci = m.pattern()
    A = sp.csr_matrix((J, ci, ro), shape=(m.ndof(), m.ndof()))
    if prec == "schwarz":
        pro, pci = P.pattern()
        Pm = sp.csr_matrix((P.values(), pci, pro), shape=(m.ndof(), m.ndof()))
        apply_p, Pd = (lambda r: Pm @ r), P
    elif prec == "diagonal":
        D = H.DiagonalPreconditioner(m)
        D.update(J)
        d = 1.0 / A.diagonal()
        apply_p, Pd = (lambda r: d * r), D
    else:
        apply_p, Pd = (lambda r: r.copy()), None
    m.set_cg_engine(engine)
    for k in (1, 2, 3):
        x = np.zeros(m.ndof())
        cg = (H.ConjugateGradient(m).with_operator(J).with_stopping_criterion(H.RelativeResidualCriterion(1e-14))
              .with_max_iter(k))
        if Pd is not None:
            cg = cg.with_preconditioner(Pd)
        with pytest.raises(H.SolveError) as ei:
            cg.solve_with_guess(b, x)
        assert ei.value.kind == H.SolveErrorKind.MaxIterationsReached and ei.value.output.num_iterations == k
        assert rel(x, numpy_pcg_iterates(A, apply_p, b, k)) < 1e-10, (k, rel(x, numpy_pcg_iterates(A, apply_p, b, k)))


def test_auto_engine_small_model_keeps_the_graphs():
    # below 32,768 nodes the automatic choice is the chunked engine, unsampled
    m, ref, P, J, b = schwarz_system(8)
    m.set_cg_engine("auto")
    xs = []
    for _ in range(3):
        x = np.zeros(m.ndof())
        (H.ConjugateGradient(m).with_operator(J).with_preconditioner(P)
         .with_stopping_criterion(H.RelativeResidualCriterion(1e-8)).with_max_iter(5000).solve_with_guess(b, x))
        xs.append(x)
    st = m.cg_engine_stats()
    assert st["auto_choice"] == 0 and st["launches"] == 0
    assert st["auto_us_per_iteration"] == [0.0, 0.0]
    # (the first solves also tune the SpMV variant, so they differ in rounding)
    for x in xs[1:]:
        assert rel(x, xs[0]) < 1e-6


def test_auto_engine_times_both_engines_and_keeps_the_faster():
    # the benchmark cylinder (44,296 nodes): per engine a set-up solve and a
    # timed whole solve, then the faster engine for the rest
    e = H.scenes.embedded_cylinder(24, 0.3, 0.4, 8, 27, 2)
    b0, b1 = e.blocks
    m = H.EmbeddedModel3d(e.vertices, b0.connectivity, b1.connectivity, (b0.weights, b0.points),
                          (b1.offsets, b1.weights, b1.points))
    mat = H.StVKMaterial(H.YoungPoisson(5e5, 0.45))
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(m, e.volume_fractions, 0.5)
    integ = H.NewtonCgIntegrator3d(m, mat, 1000.0, e.nodes_below(2, 1e-9), preconditioner=comp.build(m))
    integ.set_tolerances(1e-6, 500, 100)
    integ.set_precision(True)
    integ.set_cg_engine("auto")
    X = e.vertices
    u0 = np.zeros_like(X)
    u0[:, 0] = 0.02 * X[:, 2] ** 2
    u0 = u0.reshape(-1)
    us_ = []
    for _ in range(2):
        u, v = u0.copy(), np.zeros_like(u0)
        integ.step(u, v, 0.0, 1e-3)
        us_.append(u)
    st = integ.cg_engine_stats()
    us = st["auto_us_per_iteration"]
    assert st["auto_choice"] in (0, 1) and us[0] > 0 and us[1] > 0
    assert st["auto_choice"] == (1 if us[1] < us[0] else 0)
    assert rel(us_[1], us_[0]) < 1e-6