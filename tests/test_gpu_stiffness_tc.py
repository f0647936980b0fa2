"""Tensor-core Tet10 stiffness (tcgen05 TF32 with a hi / lo split, element
blocks of all elements as one GEMM, then a gather into the CSR values)
against the FP64 oracle and the CUDA-core FP32 kernel.

Box sizes: 6 elements (one partial tile), 162 (a partial last tile, fewer
tiles than SMs), 3,072 (one or two tiles per CTA) and 6,000 (up to three
tiles per CTA, so both accumulators and both chunk buffers are reused).
Tolerance: 1e-5 relative to the largest entry, the FP32 element arithmetic
bound the CUDA-core kernel meets as well.  Also the staged node-pair path of
the CUDA-core kernels (one launch per block, then the same gather) in FP64
(1e-10 against the oracle) and FP32, Tet10 and embedded Hex27."""
import numpy as np
import pytest

import higher_order_embedded_fem_b200 as H
from oracle import oracle as O

from test_gpu_parity import rel, tet10_setup

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cpu", [1, 3, 8, 10])
@pytest.mark.parametrize("mat_kind", [O.MAT_SNH, O.MAT_STVK])
def test_tc_stiffness_matches_oracle_and_cuda_cores(cpu, mat_kind):
    s, m, mat, ref = tet10_setup(cpu, mat_kind)
    u = H.scenes.random_normal(7 + cpu, m.ndof(), 0.02 * s.cell_size)
    Kr = ref.stiffness(u)
    m.set_stiffness_path("auto")
    Ktc = m.assemble_stiffness_into_precision(np.zeros(m.nnz), u, mat, True)
    m.set_stiffness_path("cuda_cores")
    Kcc = m.assemble_stiffness_into_precision(np.zeros(m.nnz), u, mat, True)
    m.set_stiffness_path("auto")
    e_tc, e_cc, e_x = rel(Ktc, Kr), rel(Kcc, Kr), rel(Ktc, Kcc)
    print("Tet10 box cpu=%d (%d elements): tensor cores %.2e, CUDA cores %.2e, between %.2e"
          % (cpu, m.num_elements, e_tc, e_cc, e_x))
    assert e_tc < 1e-5 and e_x < 1e-5


def test_tc_stiffness_adds_into_values_and_repeats_bitwise():
    s, m, mat, ref = tet10_setup(4, O.MAT_SNH)
    u = H.scenes.random_normal(3, m.ndof(), 0.02 * s.cell_size)
    K1 = m.assemble_stiffness_into_precision(np.zeros(m.nnz), u, mat, True)
    K2 = m.assemble_stiffness_into_precision(np.zeros(m.nnz), u, mat, True)
    assert np.array_equal(K1, K2)
    init = H.scenes.random_normal(4, m.nnz, 1.0)
    K3 = m.assemble_stiffness_into_precision(init.copy(), u, mat, True)
    assert np.abs(K3 - (init + K1)).max() <= 1e-12 * np.abs(K1).max()


def test_tc_stiffness_collapsed_element_is_singular():
    s, m, mat, ref = tet10_setup(2, O.MAT_SNH)
    u = -np.asarray(s.vertices, dtype=np.float64).reshape(-1)  # F = 0 at every point
    with pytest.raises(H.HoefemError) as ei:
        m.assemble_stiffness_into_precision(np.zeros(m.nnz), u, mat, True)
    assert ei.value.status == "SINGULAR"
    # the model stays usable
    u = H.scenes.random_normal(5, m.ndof(), 0.01 * s.cell_size)
    K = m.assemble_stiffness_into_precision(np.zeros(m.nnz), u, mat, True)
    assert rel(K, ref.stiffness(u)) < 1e-5


def test_tc_mixed_newton_step_matches_cuda_core_step():
    s = H.scenes.tet10_box(1.0, 1, 1, 1, 6)
    b = s.blocks[0]
    bc = s.nodes_below(2, 1e-9)
    out = {}
    for path in ("auto", "cuda_cores"):
        m = H.NodalModel3d(s.vertices, b.connectivity, (b.weights, b.points))
        m.set_stiffness_path(path)
        mat = H.StableNeoHookeanMaterial(H.YoungPoisson(1e6, 0.4))
        integ = H.NewtonCgIntegrator3d(m, mat, 1000.0, bc)
        integ.set_tolerances(1e-6, 1000, 100)
        integ.set_precision(True, 0.1)
        X = s.vertices
        u0 = np.zeros_like(X)
        u0[:, 0] = 0.05 * X[:, 2] ** 2
        u, v = u0.reshape(-1).copy(), np.zeros(m.ndof())
        st = integ.step(u, v, 0.0, 1e-2)
        out[path] = (u, st)
    (ua, sa), (uc, sc) = out["auto"], out["cuda_cores"]
    assert sa["newton_iterations"] == sc["newton_iterations"]
    assert rel(ua, uc) < 1e-6


@pytest.mark.parametrize("scene", ["tet10", "embedded"])
@pytest.mark.parametrize("mat_kind", [O.MAT_SNH, O.MAT_STVK])
def test_staged_pair_stiffness_matches_oracle_and_colored(scene, mat_kind):
    # whole-block launches into node-pair blocks, then the gather (automatic
    # path for FP64 and for FP32 blocks the tensor cores do not take), against
    # the colored scatter and the oracle
    from test_gpu_parity import embedded_setup

    if scene == "tet10":
        s, m, mat, ref = tet10_setup(5, mat_kind)
        h = s.cell_size
    else:
        s, m, mat, ref = embedded_setup(8, mat_kind)
        h = s.cell_size
    u = H.scenes.random_normal(11, m.ndof(), 0.01 * h)
    Kr = ref.stiffness(u)
    out = {}
    for path in ("auto", "staged", "cuda_cores"):
        m.set_stiffness_path(path)
        out[path] = (m.assemble_stiffness_into_par(np.zeros(m.nnz), u, mat),
                     m.assemble_stiffness_into_precision(np.zeros(m.nnz), u, mat, True))
    m.set_stiffness_path("auto")
    (a64, a32), (s64, s32), (c64, c32) = out["auto"], out["staged"], out["cuda_cores"]
    assert rel(a64, Kr) < 1e-10 and rel(a64, c64) < 1e-12 and np.array_equal(a64, s64)
    assert rel(a32, Kr) < 1e-5 and rel(s32, Kr) < 1e-5 and rel(c32, Kr) < 1e-5
    # adds into the values
    init = H.scenes.random_normal(12, m.nnz, 1.0)
    K = m.assemble_stiffness_into_par(init.copy(), u, mat)
    assert np.abs(K - (init + a64)).max() <= 1e-12 * np.abs(a64).max()
