"""CUDA path vs the FP64 oracle (restatement of the reference CPU path).

Tolerances: FP64 assembly / SpMV / Jacobian / preconditioner values within
1e-10 relative to the largest magnitude (max|a - b| <= 1e-10 max|b|); the
pattern and colorings are compared bit-exactly in test_product_cpu.py.
"""
import numpy as np
import pytest

import higher_order_embedded_fem_b200 as H
from oracle import oracle as O

pytestmark = pytest.mark.gpu
RTOL = 1e-10


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def tet10_setup(cpu=8, mat_kind=O.MAT_SNH, young=1e6, nu=0.4):
    s = H.scenes.tet10_box(1.0, 1, 1, 1, cpu)
    b = s.blocks[0]
    m = H.NodalModel3d(s.vertices, b.connectivity, (b.weights, b.points))
    cls = H.StableNeoHookeanMaterial if mat_kind == O.MAT_SNH else H.StVKMaterial
    mat = cls(H.YoungPoisson(young, nu))
    ref = O.Scene(s.vertices)
    ref.add_block(O.ELEM_TET10, b.connectivity, b.weights, b.points)
    ref.finalize_pattern()
    ref.set_material(mat_kind, mat.lame.mu, mat.lame.lam, 1000.0)
    return s, m, mat, ref


def embedded_setup(n=8, mat_kind=O.MAT_STVK, young=5e5, nu=0.45, seed=2):
    e = H.scenes.embedded_cylinder(n, seed=seed)
    b0, b1 = e.blocks
    m = H.EmbeddedModel3d(e.vertices, b0.connectivity, b1.connectivity, (b0.weights, b0.points),
                          (b1.offsets, b1.weights, b1.points))
    cls = H.StableNeoHookeanMaterial if mat_kind == O.MAT_SNH else H.StVKMaterial
    mat = cls(H.YoungPoisson(young, nu))
    ref = O.Scene(e.vertices)
    ref.add_block(O.ELEM_HEX27, b0.connectivity, b0.weights, b0.points)
    ref.add_block(O.ELEM_HEX27, b1.connectivity, b1.weights, b1.points, qoff=b1.offsets)
    ref.finalize_pattern()
    ref.set_material(mat_kind, mat.lame.mu, mat.lame.lam, 1000.0)
    return e, m, mat, ref


@pytest.mark.parametrize("mat_kind", [O.MAT_SNH, O.MAT_STVK])
def test_tet10_forces_and_stiffness(mat_kind):
    s, m, mat, ref = tet10_setup(8, mat_kind)
    u = H.scenes.random_normal(1, m.ndof(), 0.01 * s.cell_size)
    f = m.assemble_elastic_pseudo_forces(u, mat)
    assert rel(f, ref.forces(u)) < RTOL
    K = m.assemble_stiffness(u, mat)
    Kr = ref.stiffness(u)
    assert rel(K, Kr) < RTOL
    # accumulation semantics: "_into" adds
    f2 = m.assemble_elastic_pseudo_forces_into_par(np.ones(m.ndof()), u, mat)
    assert rel(f2 - 1.0, f) < 1e-12
    K2 = m.assemble_stiffness_into_par(np.full(m.nnz, 4.0), u, mat)
    assert rel(K2 - 4.0, K) < 1e-12


@pytest.mark.parametrize("mat_kind", [O.MAT_SNH, O.MAT_STVK])
def test_embedded_hex27_forces_and_stiffness(mat_kind):
    e, m, mat, ref = embedded_setup(8, mat_kind)
    u = H.scenes.random_normal(3, m.ndof(), 0.01 * e.cell_size)
    assert rel(m.assemble_elastic_pseudo_forces(u, mat), ref.forces(u)) < RTOL
    assert rel(m.assemble_stiffness(u, mat), ref.stiffness(u)) < RTOL


def test_mass_matrix():
    s, m, mat, ref = tet10_setup(4)
    assert rel(m.assemble_mass(1000.0), ref.mass_values(1000.0)) < RTOL
    e, me, mate, refe = embedded_setup(6)
    assert rel(me.assemble_mass(1000.0), refe.mass_values(1000.0)) < RTOL


def test_device_tensors_match_host_arrays():
    torch = pytest.importorskip("torch")
    s, m, mat, ref = tet10_setup(4)
    u = H.scenes.random_normal(5, m.ndof(), 0.01 * s.cell_size)
    Kh = m.assemble_stiffness(u, mat)
    ud = torch.from_numpy(u).cuda()
    Kd = m.assemble_stiffness(ud, mat)
    assert np.array_equal(Kd.cpu().numpy(), Kh)
    fd = m.assemble_elastic_pseudo_forces(ud, mat)
    assert np.array_equal(fd.cpu().numpy(), m.assemble_elastic_pseudo_forces(u, mat))


def test_spmv_jacobian_dirichlet():
    s, m, mat, ref = tet10_setup(6)
    u = H.scenes.random_normal(1, m.ndof(), 0.01 * s.cell_size)
    K = ref.stiffness(u)
    x = H.scenes.random_normal(9, m.ndof(), 1.0)
    ro, ci = m.pattern()
    dense_y = np.zeros(m.ndof())
    for r in range(m.ndof()):
        dense_y[r] = np.dot(K[ro[r]:ro[r + 1]], x[ci[ro[r]:ro[r + 1]]])
    y = m.spmv(np.zeros(m.ndof()), K, x)
    assert rel(y, dense_y) < 1e-13
    y2 = m.spmv(np.ones(m.ndof()), K, x, alpha=2.0, beta=3.0)
    assert rel(y2, 3.0 + 2.0 * dense_y) < 1e-13
    bc = s.nodes_below(2, 1e-9)
    ref.set_bc(bc)
    ref.set_gravity(True)
    ref.setup()
    M = ref.mass()
    dt = 1e-3
    J = m.jacobian_combination(np.zeros(m.nnz), dt * dt, K, 1.0, M, bc)
    assert rel(J, ref.jacobian(K, dt)) < 1e-14
    # golden Dirichlet semantics on the GPU path
    Kb = m.apply_dirichlet_bc_csr(K.copy(), bc)
    Kr = O.dirichlet_csr(ro, ci, K, bc, 3)
    assert np.array_equal(Kb, Kr)


@pytest.mark.parametrize("variant", [8, 16, 32, 108, 116, 132])
def test_spmv_variants_agree(variant):
    # every SpMV traversal (also the ones inside CG) sums the same products
    e, m, mat, ref = embedded_setup(6)
    u = H.scenes.random_normal(1, m.ndof(), 0.01 * e.cell_size)
    K = ref.stiffness(u)
    x = H.scenes.random_normal(9, m.ndof(), 1.0)
    ro, ci = m.pattern()
    dense_y = np.array([np.dot(K[ro[r]:ro[r + 1]], x[ci[ro[r]:ro[r + 1]]]) for r in range(m.ndof())])
    m.set_spmv_variant(variant)
    assert rel(m.spmv(np.zeros(m.ndof()), K, x), dense_y) < 1e-13
    bc = e.nodes_below(2, 1e-9)
    ref.set_bc(bc)
    ref.setup()
    J = ref.jacobian(ref.stiffness(np.zeros(m.ndof())), 1e-3)  # SPD at rest
    P = H.DiagonalPreconditioner(m)
    P.update(J)
    b = H.scenes.random_normal(6, m.ndof(), 1.0)
    b[np.repeat(3 * bc, 3) + np.tile(np.arange(3), bc.size)] = 0.0
    xs = np.zeros(m.ndof())
    out = (H.ConjugateGradient(m).with_operator(J).with_preconditioner(P)
           .with_stopping_criterion(H.RelativeResidualCriterion(1e-8)).with_max_iter(5000).solve_with_guess(b, xs))
    st, xr, itr = ref.cg(J, b, 1e-8, 5000)
    assert st == 0 and abs(out.num_iterations - itr) <= 1
    assert rel(xs, xr) < 1e-6


def test_diagonal_preconditioner_and_cg():
    s, m, mat, ref = tet10_setup(6)
    u = H.scenes.random_normal(1, m.ndof(), 0.01 * s.cell_size)
    bc = s.nodes_below(2, 1e-9)
    ref.set_bc(bc)
    ref.setup()
    J = ref.jacobian(ref.stiffness(u), 1e-3)
    P = H.DiagonalPreconditioner(m)
    P.update(J)
    r = H.scenes.random_normal(4, m.ndof(), 1.0)
    ro, ci = m.pattern()
    diag = np.array([J[ro[i] + np.searchsorted(ci[ro[i]:ro[i + 1]], i)] for i in range(m.ndof())])
    assert rel(P.apply(r), r / diag) < 1e-15
    b = H.scenes.random_normal(6, m.ndof(), 1.0)
    b[np.repeat(3 * bc, 3) + np.tile(np.arange(3), bc.size)] = 0.0
    x = np.zeros(m.ndof())
    out = (H.ConjugateGradient(m).with_operator(J).with_preconditioner(P)
           .with_stopping_criterion(H.RelativeResidualCriterion(1e-10)).with_max_iter(2000).solve_with_guess(b, x))
    st, xr, itr = ref.cg(J, b, 1e-10, 2000)
    assert st == 0
    assert abs(out.num_iterations - itr) <= 1
    assert rel(x, xr) < 1e-8
    y = m.spmv(np.zeros(m.ndof()), J, x)
    assert np.linalg.norm(y - b) <= 1e-10 * np.linalg.norm(b) * 10


def test_cg_error_kinds():
    s, m, mat, ref = tet10_setup(3)
    ref.setup()
    J = ref.jacobian(ref.stiffness(np.zeros(m.ndof())), 1e-3)
    b = H.scenes.random_normal(6, m.ndof(), 1.0)
    with pytest.raises(H.SolveError) as ei:
        H.ConjugateGradient(m).with_operator(J).with_stopping_criterion(
            H.RelativeResidualCriterion(1e-14)).with_max_iter(2).solve_with_guess(b, np.zeros(m.ndof()))
    assert ei.value.kind == H.SolveErrorKind.MaxIterationsReached and ei.value.output.num_iterations == 2
    with pytest.raises(H.SolveError) as ei:
        H.ConjugateGradient(m).with_operator(-J).solve_with_guess(b, np.zeros(m.ndof()))
    assert ei.value.kind == H.SolveErrorKind.IndefiniteOperator and ei.value.output.num_iterations == 0
    x = np.ones(m.ndof())
    out = H.ConjugateGradient(m).with_operator(J).solve_with_guess(np.zeros(m.ndof()), x)
    assert out.num_iterations == 0 and not x.any()


def test_schwarz_preconditioner_values():
    e, m, mat, ref = embedded_setup(8)
    u = H.scenes.random_normal(3, m.ndof(), 0.01 * e.cell_size)
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(m, e.volume_fractions, 0.5)
    bc = e.nodes_below(2, 1e-9)
    ref.set_bc(bc)
    ref.set_schwarz(comp.schwarz_connectivity, comp.untreated_nodes)
    ref.setup()
    J = ref.jacobian(ref.stiffness(u), 1e-3)
    P = comp.build(m)
    ro, ci = P.pattern()
    ro2, ci2 = ref.schwarz_pattern()
    assert np.array_equal(ro, ro2) and np.array_equal(ci, ci2)
    P.update(J)
    pv = P.values()
    pr = ref.schwarz_update(J)
    assert rel(pv, pr) < RTOL
    r = H.scenes.random_normal(8, m.ndof(), 1.0)
    z = P.apply(r)
    zr = np.zeros(m.ndof())
    for i in range(m.ndof()):
        zr[i] = np.dot(pr[ro[i]:ro[i + 1]], r[ci[ro[i]:ro[i + 1]]])
    assert rel(z, zr) < 1e-12


def test_newton_step_tet10_matches_oracle():
    s, m, mat, ref = tet10_setup(4)
    bc = s.nodes_below(2, 1e-9)
    u0 = H.scenes.random_normal(1, m.ndof(), 0.01 * s.cell_size)
    v0 = np.zeros(m.ndof())
    integ = H.NewtonCgIntegrator3d(m, mat, 1000.0, bc)
    ref.set_bc(bc)
    ref.set_gravity(True)
    ref.set_solver(1e-5, 500, 100)
    ref.setup()
    assert rel(integ.mass(), ref.mass()) < RTOL
    u, v = u0.copy(), v0.copy()
    st = integ.step(u, v, 0.0, 1e-3)
    ur, vr, rs = ref.step(u0, v0, 0.0, 1e-3)
    assert rs["status"] == 0
    assert st["newton_iterations"] == rs["newton_iters"]
    assert abs(st["representative_force"] - ref.representative_force()) <= 1e-12 * ref.representative_force()
    assert rel(u, ur) < 1e-8 and rel(v, vr) < 1e-8


def test_newton_step_embedded_schwarz_matches_oracle():
    e, m, mat, ref = embedded_setup(6)
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
    assert abs(st["total_cg_iterations"] - sum(rs["cg_iters"])) <= max(2, 0.02 * sum(rs["cg_iters"]))
    assert rel(u, ur) < 1e-8 and rel(v, vr) < 1e-8


def test_schwarz_indefinite_blocks_take_the_eigen_path():
    # Negated system matrix: every block is negative definite, the Cholesky fast
    # path fails and the eigen-decomposition path applies the |lambda| rule.
    e, m, mat, ref = embedded_setup(6)
    u = H.scenes.random_normal(3, m.ndof(), 0.01 * e.cell_size)
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(m, e.volume_fractions, 0.5)
    ref.set_bc(e.nodes_below(2, 1e-9))
    ref.set_schwarz(comp.schwarz_connectivity, comp.untreated_nodes)
    ref.setup()
    J = -ref.jacobian(ref.stiffness(u), 1e-3)
    P = comp.build(m)
    P.update(J)
    assert rel(P.values(), ref.schwarz_update(J)) < RTOL


def test_schwarz_zero_diagonal_is_an_error():
    e, m, mat, ref = embedded_setup(6)
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(m, e.volume_fractions, 0.5)
    P = comp.build(m)
    with pytest.raises(H.HoefemError) as ei:
        P.update(np.zeros(m.nnz))
    assert ei.value.status in ("ZERO_DIAGONAL", "NONFINITE")
    D = H.DiagonalPreconditioner(m)
    with pytest.raises(H.HoefemError) as ei:
        D.update(np.zeros(m.nnz))
    assert ei.value.status == "ZERO_DIAGONAL"


@pytest.mark.parametrize("mixed", [False, True])
def test_schwarz_block_apply_matches_assembled_apply(mixed):
    # The CG's Schwarz apply as dense subdomain block products (default) and as
    # the SpMV over the assembled values: the same P r up to rounding, so the
    # Newton step agrees to the CG tolerance and the iteration counts match.
    e, m, mat, ref = embedded_setup(6)
    bc = e.nodes_below(2, 1e-9)
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(m, e.volume_fractions, 0.5)
    P = comp.build(m)
    integ = H.NewtonCgIntegrator3d(m, mat, 1000.0, bc, preconditioner=P)
    integ.set_precision(mixed, 0.1)
    u0 = H.scenes.random_normal(1, m.ndof(), 0.01 * e.cell_size)
    out = []
    for on in (True, False):
        P.set_block_apply(on)
        u, v = u0.copy(), np.zeros(m.ndof())
        st = integ.step(u, v, 0.0, 1e-3)
        out.append((u, v, st))
    (ub, vb, sb), (uc, vc, sc) = out
    assert sb["newton_iterations"] == sc["newton_iterations"]
    assert abs(sb["total_cg_iterations"] - sc["total_cg_iterations"]) <= 2
    assert rel(ub, uc) < 1e-8 and rel(vb, vc) < 1e-8
