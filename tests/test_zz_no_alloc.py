"""hoefem_jacobian_combination_noalloc (scratch in a fixed library array) must
give exactly what hoefem_jacobian_combination gives, call after call: the
Dirichlet mask of one call must not leak into the next."""
import numpy as np
import pytest

import higher_order_embedded_fem_b200 as H
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_noalloc_jacobian_matches_allocating_entry_point():
    torch = pytest.importorskip("torch")
    s = H.scenes.tet10_box(1.0, 1, 1, 1, 4)
    b = s.blocks[0]
    m = H.NodalModel3d(s.vertices, b.connectivity, (b.weights, b.points))
    ref = O.Scene(s.vertices)
    ref.add_block(O.ELEM_TET10, b.connectivity, b.weights, b.points)
    ref.finalize_pattern()
    mat = H.StableNeoHookeanMaterial(H.YoungPoisson(1e6, 0.4))
    ref.set_material(O.MAT_SNH, mat.lame.mu, mat.lame.lam, 1000.0)
    u = H.scenes.random_normal(1, m.ndof(), 0.01 * s.cell_size)
    K = torch.tensor(ref.stiffness(u), device="cuda")
    M = torch.tensor(ref.mass_values(1000.0), device="cuda")
    bc_sets = [s.nodes_below(2, 1e-9), s.nodes_below(0, 0.26)]
    dt = 1e-3
    for bc in bc_sets:  # two calls in a row, different Dirichlet sets
        want = m.jacobian_combination(torch.zeros_like(K), dt * dt, K, 1.0, M, bc)
        got = m.jacobian_combination_noalloc(torch.zeros_like(K), dt * dt, K, 1.0, M, bc)
        torch.cuda.synchronize()
        assert torch.equal(got, want)
    # the point of the entry point: once its first call on the device has
    # looked up the scratch address, further calls allocate no device memory
    # (free device memory is unchanged; the check does see an allocation)
    def free_bytes():
        torch.cuda.synchronize()
        return torch.cuda.mem_get_info()[0]

    out = torch.zeros_like(K)
    torch.cuda.empty_cache()
    f0 = free_bytes()
    for bc in bc_sets * 3:
        m.jacobian_combination_noalloc(out, dt * dt, K, 1.0, M, bc)
    assert free_bytes() == f0
    probe = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    assert free_bytes() < f0
    del probe
    torch.cuda.empty_cache()
    # no Dirichlet nodes, mass only
    want = m.jacobian_combination(torch.zeros_like(K), 0.0, None, 1.0, M, ())
    got = m.jacobian_combination_noalloc(torch.zeros_like(K), 0.0, None, 1.0, M, ())
    assert torch.equal(got, want)
    # beyond the scratch's Dirichlet-node capacity: a clear error, nothing run
    too_many = np.zeros((1 << 18) + 1, dtype=np.int64)
    with pytest.raises(H.HoefemError, match="262,144"):
        m.jacobian_combination_noalloc(torch.zeros_like(K), dt * dt, K, 1.0, M, too_many)
