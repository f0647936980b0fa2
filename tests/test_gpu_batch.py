"""Batched steps of independent scenes vs the FP64 oracle, scene by scene.

Every scene of a batch must end where the oracle's backward-Euler Newton-CG
step (diagonal preconditioner) takes it alone: displacement and velocity
within 1e-8 relative, the same number of Newton iterations.  The CG engines
of the batch (graphs, persistent launch, autotuned) give the same bits.
"""
import numpy as np
import pytest

import higher_order_embedded_fem_b200 as H
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


SCENES = [
    ("tet10", dict(unit=1.0, ux=1, uy=1, uz=1, cells_per_unit=3), 1e6, 0.40),
    ("hex27", dict(unit=0.5, ux=2, uy=1, uz=1, cells_per_unit=2), 3e5, 0.30),
    ("tet10", dict(unit=0.5, ux=2, uy=2, uz=1, cells_per_unit=2), 5e6, 0.45),
    ("cyl", dict(n=6, seed=4), 2e5, 0.35),
    ("hex27", dict(unit=1.0, ux=1, uy=1, uz=1, cells_per_unit=3), 1e7, 0.48),
    ("tet10", dict(unit=1.0, ux=1, uy=1, uz=2, cells_per_unit=2), 1e5, 0.33),
]


def make_scene(kind, args, young, nu):
    if kind == "tet10":
        s = H.scenes.tet10_box(**args)
    elif kind == "hex27":
        s = H.scenes.hex27_box(**args)
    else:
        s = H.scenes.embedded_cylinder(**args)
    mat = H.StableNeoHookeanMaterial(H.YoungPoisson(young, nu))
    if kind == "cyl":
        b0, b1 = s.blocks
        m = H.EmbeddedModel3d(s.vertices, b0.connectivity, b1.connectivity, (b0.weights, b0.points),
                              (b1.offsets, b1.weights, b1.points))
    else:
        b = s.blocks[0]
        m = H.NodalModel3d(s.vertices, b.connectivity, (b.weights, b.points), b.kind)
    ref = O.Scene(s.vertices)
    for b in s.blocks:
        ref.add_block(O.ELEM_TET10 if b.kind == H.ELEM_TET10 else O.ELEM_HEX27, b.connectivity, b.weights,
                      b.points, qoff=b.offsets)
    ref.finalize_pattern()
    ref.set_material(O.MAT_SNH, mat.lame.mu, mat.lame.lam, 1000.0)
    return s, m, mat, ref


@pytest.fixture(scope="module")
def batch_inputs():
    out = []
    for k, (kind, args, young, nu) in enumerate(SCENES):
        s, m, mat, ref = make_scene(kind, args, young, nu)
        bc = s.nodes_below(2, 1e-9)
        u0 = H.scenes.random_normal(100 + k, m.ndof(), 0.01 * s.cell_size)
        out.append((s, m, mat, ref, bc, u0))
    return out


def test_batch_step_matches_oracle_per_scene(batch_inputs):
    models = [x[1] for x in batch_inputs]
    mats = [x[2] for x in batch_inputs]
    bcs = [x[4] for x in batch_inputs]
    B = H.BatchedNewtonCgIntegrator3d(models, mats, 1000.0, bcs)
    assert B.num_scenes == len(SCENES)
    assert B.dof_offsets[-1] == sum(m.ndof() for m in models)
    u = np.concatenate([x[5] for x in batch_inputs])
    v = np.zeros_like(u)
    stats = B.step(u, v, 0.0, 1e-3)
    us, vs = B.split(u), B.split(v)
    for k, (s, m, mat, ref, bc, u0) in enumerate(batch_inputs):
        ref.set_bc(bc)
        ref.set_gravity(True)
        ref.set_solver(1e-5, 500, 100)
        ref.setup()
        ur, vr, rs = ref.step(u0, np.zeros_like(u0), 0.0, 1e-3)
        assert rs["status"] == 0 and stats[k]["status"] == 0
        assert stats[k]["newton_iterations"] == rs["newton_iters"], k
        assert abs(stats[k]["representative_force"] - ref.representative_force()) <= 1e-12 * ref.representative_force()
        assert abs(stats[k]["total_cg_iterations"] - sum(rs["cg_iters"])) <= max(2, 0.02 * sum(rs["cg_iters"])), k
        assert rel(us[k], ur) < 1e-8 and rel(vs[k], vr) < 1e-8, k


def test_batch_device_arrays_and_repeat(batch_inputs):
    torch = pytest.importorskip("torch")
    models = [x[1] for x in batch_inputs[:3]]
    mats = [x[2] for x in batch_inputs[:3]]
    bcs = [x[4] for x in batch_inputs[:3]]
    B = H.BatchedNewtonCgIntegrator3d(models, mats, 1000.0, bcs)
    u_h = np.concatenate([x[5] for x in batch_inputs[:3]])
    v_h = np.zeros_like(u_h)
    u_d = torch.tensor(u_h, device="cuda")
    v_d = torch.zeros_like(u_d)
    for _ in range(2):
        B.step(u_h, v_h, 0.0, 1e-3)
        B.step(u_d, v_d, 0.0, 1e-3)
    torch.cuda.synchronize()
    assert np.array_equal(u_d.cpu().numpy(), u_h) and np.array_equal(v_d.cpu().numpy(), v_h)


def test_batch_failure_is_per_scene(batch_inputs):
    # Without gravity a scene at rest is converged before any Newton iteration;
    # with newton_max_iter = 0 every other scene fails at every substep count.
    # (StVK: zero stress at rest, so the internal force of the rest state is zero)
    models = [x[1] for x in batch_inputs[:3]]
    mats = [H.StVKMaterial(H.YoungPoisson(*SCENES[k][2:])) for k in range(3)]
    bcs = [x[4] for x in batch_inputs[:3]]
    B = H.BatchedNewtonCgIntegrator3d(models, mats, 1000.0, bcs, gravity_enabled=False)
    B.set_tolerances(1e-5, 500, 0)
    parts = [np.zeros(models[0].ndof())] + [x[5].copy() for x in batch_inputs[1:3]]
    u = np.concatenate(parts)
    u0 = u.copy()
    v = np.zeros_like(u)
    with pytest.raises(H.HoefemError):
        B.step(u, v, 0.0, 1e-3)
    st = B.stats()
    assert st[0]["status"] == 0 and st[0]["newton_iterations"] == 0
    assert st[1]["status"] == 22 and st[2]["status"] == 22
    # failed scenes keep their state (Dirichlet values applied), the converged one stays at rest
    bc_mask = np.zeros(u.size, dtype=bool)
    for k, b in enumerate(bcs):
        for a in b:
            bc_mask[B.dof_offsets[k] + 3 * a:B.dof_offsets[k] + 3 * a + 3] = True
    assert np.array_equal(u[~bc_mask], u0[~bc_mask]) and np.all(u[bc_mask] == 0.0)
    assert np.all(v == 0.0)
    # the single-scene integrator reports the same failure
    integ = H.NewtonCgIntegrator3d(models[1], mats[1], 1000.0, bcs[1], gravity_enabled=False)
    integ.set_tolerances(1e-5, 500, 0)
    with pytest.raises(H.HoefemError):
        integ.step(parts[1].copy(), np.zeros_like(parts[1]), 0.0, 1e-3)


@pytest.mark.parametrize("cg_tol,cg_max", [(1e-5, 500), (1e-9, 60)])
def test_batch_cg_engines_give_the_same_bits(batch_inputs, cg_tol, cg_max):
    # The graph engine, the persistent launch at several grid sizes and the
    # autotuned choice run the same arithmetic: identical states and statistics
    # (also when the iteration cap ends solves early).
    models = [x[1] for x in batch_inputs]
    mats = [x[2] for x in batch_inputs]
    bcs = [x[4] for x in batch_inputs]
    u0 = np.concatenate([x[5] for x in batch_inputs])
    out = {}
    for key in [("chunked", 0), ("streamed", 0), ("streamed", 1), ("streamed", 2), ("auto", 0)]:
        B = H.BatchedNewtonCgIntegrator3d(models, mats, 1000.0, bcs)
        B.set_tolerances(cg_tol, cg_max, 100)
        B.set_cg_engine(*key)
        u, v = u0.copy(), np.zeros_like(u0)
        stats = []
        for _ in range(2):
            stats.append(B.step(u, v, 0.0, 1e-3, raise_on_failure=False))
        drop = ("ms_total",)
        stats = [[{k: x for k, x in d.items() if k not in drop} for d in st] for st in stats]
        out[key] = (u, v, stats, B.cg_choice())
    ua, va, sa, _ = out[("chunked", 0)]
    for key, (u, v, st, choice) in out.items():
        assert np.array_equal(u, ua) and np.array_equal(v, va), key
        assert st == sa, key
    eng, per, times = out[("auto", 0)][3]
    print("autotuner: %s, %d CTAs/SM, candidates (ms) %s" % (eng, per, ["%.2f" % t for t in times]))
    assert eng in ("chunked", "streamed") and len(times) >= 2
    assert out[("streamed", 1)][3][:2] == ("streamed", 1)
