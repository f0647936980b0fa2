"""Learned coarse correction: CUDA forward / backward vs the numpy oracle,
BF16 tensor-core inference vs FP32, Adam training on pairs from plain
Schwarz-CG solves, and the gain of the trained network on a held-out seed."""
import numpy as np
import pytest

import higher_order_embedded_fem_b200 as H
from oracle import mlp

from test_gpu_parity import embedded_setup

pytestmark = pytest.mark.gpu


def _model(n=8):
    e, m, mat, ref = embedded_setup(n)
    return e, m, mat


def test_mlp_forward_backward_match_oracle():
    e, m, mat = _model(6)
    L = H.LearnedCoarseCorrection(m, e.nodes_below(2, 1e-9), num_subdomains=16, seed=1)
    rng = np.random.default_rng(0)
    w = (rng.standard_normal(L.num_params) * 0.05).astype(np.float32)
    L.set_weights(w)
    X = rng.standard_normal((96, mlp.F)).astype(np.float32)
    T = rng.standard_normal((96, mlp.O)).astype(np.float32)
    loss, g, out = L.forward_backward(X, T)
    loss_r, g_r, out_r = mlp.loss_and_grads(w, X, T)
    assert abs(loss - loss_r) <= 1e-5 * abs(loss_r)
    assert np.abs(out - out_r).max() <= 1e-4 * np.abs(out_r).max()
    assert np.abs(g - g_r).max() <= 1e-4 * np.abs(g_r).max()


def test_bf16_tensor_core_inference_close_to_fp32():
    e, m, mat = _model(6)
    L = H.LearnedCoarseCorrection(m, e.nodes_below(2, 1e-9), num_subdomains=16, seed=2)
    rng = np.random.default_rng(1)
    L.set_weights((rng.standard_normal(L.num_params) * 0.05).astype(np.float32))
    X = rng.standard_normal((64, mlp.F)).astype(np.float32)
    y32 = L.infer(X, bf16=False)
    y16 = L.infer(X, bf16=True)
    _, _, yr = mlp.loss_and_grads(L.get_weights(), X, np.zeros((64, mlp.O)))
    assert np.abs(y32 - yr).max() <= 1e-4 * np.abs(yr).max()
    assert np.abs(y16 - y32).max() <= 3e-2 * np.abs(y32).max()


def _integrator(e, m, mat, comp, mixed=False):
    P = comp.build(m)
    it = H.NewtonCgIntegrator3d(m, mat, 1000.0, e.nodes_below(2, 1e-9), preconditioner=P)
    it.set_tolerances(1e-6, 500, 100)
    it.set_precision(mixed, 0.1)
    it._P = P
    return it


def _state(e, m, seed, amp=0.02):
    X = e.vertices
    u0 = np.zeros_like(X)
    u0[:, 0] = amp * X[:, 2] ** 2
    u0[:, 1] = 0.5 * amp * X[:, 2] ** 2
    return u0.reshape(-1) + H.scenes.random_normal(seed, m.ndof(), 0.001 * e.cell_size), np.zeros(m.ndof())


def test_training_on_cg_pairs_and_heldout_gain():
    e, m, mat = _model(8)
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(m, e.volume_fractions, 0.5)
    L = H.LearnedCoarseCorrection(m, e.nodes_below(2, 1e-9), num_subdomains=64, seed=3)
    it = _integrator(e, m, mat, comp)
    it.set_learned(L, 2)
    for seed in range(4):
        u, v = _state(e, m, 100 + seed, amp=0.01 + 0.01 * seed)
        it.step(u, v, 0.0, 1e-3)
    assert L.num_pairs() > 0
    hist = L.train(600, batch=256, lr=1e-3, seed=0)
    assert np.mean(hist[-50:]) < 0.5 * np.mean(hist[:10])
    # held-out seed: plain vs learned warm start
    u0, v0 = _state(e, m, 999, amp=0.025)
    it.set_learned(None)
    u, v = u0.copy(), v0.copy()
    plain = it.step(u, v, 0.0, 1e-3)
    it.set_learned(L, 1)
    ul, vl = u0.copy(), v0.copy()
    learned = it.step(ul, vl, 0.0, 1e-3)
    assert learned["learned_accepted"] + learned["learned_rejected"] == learned["num_cg_solves"]
    assert np.abs(ul - u).max() <= 1e-6 * np.abs(u).max()
    assert learned["total_cg_iterations"] <= 1.1 * plain["total_cg_iterations"] + 2
    print("plain CG iterations %d, learned %d (accepted %d, residual ratio %.3f)" % (
        plain["total_cg_iterations"], learned["total_cg_iterations"], learned["learned_accepted"],
        learned["learned_residual_ratio"]))


def test_two_level_learned_preconditioner_solves_the_step_at_dt_1e2():
    # dt = 1e-2: a stiffer Jacobian, where a coarse correction on this coarse
    # space could pay (the exact Galerkin one saves about a third of the
    # Schwarz-CG iterations, test_coarse_space_ceiling.py).  The network,
    # trained on (r_k, x* - x_k) pairs of plain Schwarz-CG solves of other
    # seeds, is applied beside Schwarz in every iteration (flexible CG).  The
    # step must reach the same solution; the iteration counts are reported:
    # the correction varies nonlinearly with r from one iteration to the next,
    # which costs the flexible recurrence its conjugacy, and it takes far more
    # iterations than plain Schwarz-CG.
    dt = 1e-2
    e, m, mat = _model(10)
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(m, e.volume_fractions, 0.5)
    L = H.LearnedCoarseCorrection(m, e.nodes_below(2, 1e-9), num_subdomains=32, seed=5)
    it = _integrator(e, m, mat, comp)
    it.set_tolerances(1e-6, 5000, 100)
    it.set_learned(L, 3)
    for seed in range(6):
        u, v = _state(e, m, 200 + seed, amp=0.01 + 0.004 * seed)
        it.step(u, v, 0.0, dt)
    assert L.num_pairs() > 0
    hist = L.train(1500, batch=256, lr=1e-3, seed=0)
    assert np.mean(hist[-50:]) < 0.5 * np.mean(hist[:10])
    u0, v0 = _state(e, m, 4242, amp=0.017)
    it.set_learned(None)
    u, v = u0.copy(), v0.copy()
    plain = it.step(u, v, 0.0, dt)
    it.set_learned(L, 4)
    ul, vl = u0.copy(), v0.copy()
    two = it.step(ul, vl, 0.0, dt)
    print("dt 1e-2: Schwarz-CG %d iterations (%d Newton), learned two-level %d (%d Newton; correction kept in %d "
          "of %d iterations)" % (plain["total_cg_iterations"], plain["newton_iterations"], two["total_cg_iterations"],
                                 two["newton_iterations"], two["learned_accepted"],
                                 two["learned_accepted"] + two["learned_rejected"]))
    assert two["learned_accepted"] > 0
    assert two["residual_norm"] <= dt * 1e-5 * two["representative_force"]
    assert np.abs(ul - u).max() <= 1e-5 * np.abs(u).max()
