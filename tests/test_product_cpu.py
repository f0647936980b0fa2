"""Host-side logic of the product (no GPU): ABI exports, scenes, pattern,
coloring and Schwarz subdomain selection against the oracle."""
import ctypes
import json
import os
import re

import numpy as np
import pytest

import higher_order_embedded_fem_b200 as H
from higher_order_embedded_fem_b200 import _capi
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_vectors.json")))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "hoefem.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(hoefem_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_capi.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 40
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(_capi.SIGNATURES), set(syms) ^ set(_capi.SIGNATURES)
    assert _capi.lib().hoefem_abi_version() == 1


def test_lame_conversion_matches_reference():
    lame = H.LameParameters.from_young_poisson(H.YoungPoisson(1e6, 0.4))
    mu, lam = O.lame(1e6, 0.4)
    assert lame.mu == mu and lame.lam == lam


def test_quadrature_tables_match_reference_source():
    s = H.scenes.tet10_box(1.0, 1, 1, 1, 1)
    q = GOLD["quadrature"]["tet_quadrature_strength_5"]
    assert np.array_equal(s.blocks[0].weights, np.array(q["weights"]))
    assert np.array_equal(s.blocks[0].points, np.array(q["points"]))
    e = H.scenes.embedded_cylinder(4)
    q = GOLD["quadrature"]["hex_quadrature_strength_5"]
    assert np.array_equal(e.blocks[0].weights, np.array(q["weights"]))
    assert np.array_equal(e.blocks[0].points, np.array(q["points"]))


@pytest.mark.parametrize("cpu", [1, 2, 5, 8])
def test_tet10_scene_matches_reference_mesh_pipeline(cpu):
    s = H.scenes.tet10_box(1.0, 1, 1, 1, cpu)
    t = O.tets_from_hex(O.hex_box(1.0, 1, 1, 1, cpu), True)
    assert np.array_equal(s.vertices, t.vertices)
    assert np.array_equal(s.blocks[0].connectivity, t.cells)


def test_tet10_box_non_cubic_matches():
    s = H.scenes.tet10_box(0.25, 3, 2, 1, 2)
    t = O.tets_from_hex(O.hex_box(0.25, 3, 2, 1, 2), True)
    assert np.array_equal(s.vertices, t.vertices) and np.array_equal(s.blocks[0].connectivity, t.cells)


def test_hex27_box_matches_reference_refinement():
    s = H.scenes.hex27_box(0.5, 2, 1, 3, 2)
    t = O.hex27_from_hex(O.hex_box(0.5, 2, 1, 3, 2))
    assert np.array_equal(s.vertices, t.vertices) and np.array_equal(s.blocks[0].connectivity, t.cells)
    assert s.blocks[0].offsets is None and s.blocks[0].weights.size == 14


def test_pattern_and_coloring_bit_exact_hex27_box():
    s = H.scenes.hex27_box(1.0, 1, 1, 1, 3)
    b = s.blocks[0]
    with pytest.raises(ValueError):
        H.NodalModel3d(s.vertices, b.connectivity, (b.weights, b.points))  # Tet10 by default
    m = H.NodalModel3d(s.vertices, b.connectivity, (b.weights, b.points), H.ELEM_HEX27)
    _check_model_vs_oracle(s.blocks, s.vertices, m)


def test_embedded_cylinder_matches_reference_refinement_and_keep_cells():
    n = 6
    e = H.scenes.embedded_cylinder(n)
    h27 = O.hex27_from_hex(O.hex_box(1.0, 1, 1, 1, n))
    # reconstruct kept cell ids from the refined mesh: match cell centers
    full = h27.cells
    centers = h27.vertices[full[:, 26]]
    ids = []
    for b in e.blocks:
        cc = e.vertices[b.connectivity[:, 26]]
        for c in cc:
            ids.append(int(np.argmin(np.abs(centers - c).sum(axis=1))))
    kept = O.keep_cells(h27, np.array(ids))
    assert np.array_equal(kept.vertices, e.vertices)
    conn = np.vstack([b.connectivity for b in e.blocks])
    assert np.array_equal(kept.cells, conn)
    # interface weights: sum w = 8 phi, volume fractions in (0, 1)
    b = e.blocks[1]
    assert np.all(np.diff(b.offsets) >= 8) and np.all(np.diff(b.offsets) <= 27)
    vf = e.volume_fractions
    assert np.all(vf > 0) and np.all(vf < 1)


def _check_model_vs_oracle(blocks, vertices, model):
    conn_all = np.vstack([b.connectivity for b in blocks])
    ro, ci = model.pattern()
    ro2, ci2 = O.pattern(conn_all.tolist(), 3, vertices.shape[0])
    assert np.array_equal(ro, ro2) and np.array_equal(ci, ci2)
    for k, b in enumerate(blocks):
        cols = model.colors(k)
        cols2 = O.coloring(b.connectivity.tolist())
        assert len(cols) == len(cols2)
        for a, c in zip(cols, cols2):
            assert np.array_equal(a, np.array(c, dtype=np.int64))


def test_pattern_and_coloring_bit_exact_tet10():
    s = H.scenes.tet10_box(1.0, 1, 1, 1, 8)
    b = s.blocks[0]
    m = H.NodalModel3d(s.vertices, b.connectivity, (b.weights, b.points))
    assert m.nnz == 1141065 and m.ndof() == 14739
    _check_model_vs_oracle(s.blocks, s.vertices, m)


def test_pattern_and_coloring_bit_exact_embedded():
    e = H.scenes.embedded_cylinder(8)
    b0, b1 = e.blocks
    m = H.EmbeddedModel3d(e.vertices, b0.connectivity, b1.connectivity, (b0.weights, b0.points),
                          (b1.offsets, b1.weights, b1.points))
    _check_model_vs_oracle(e.blocks, e.vertices, m)


def test_large_tet10_sizes():
    # 40 x 40 x 21 hexes x 6 Tet10: 201,600 elements / 282,123 nodes / 70,917,201 nnz
    s = H.scenes.tet10_box(0.025, 40, 40, 21, 1)
    b = s.blocks[0]
    assert b.connectivity.shape == (201600, 10) and s.vertices.shape == (282123, 3)
    m = H.NodalModel3d(s.vertices, b.connectivity, (b.weights, b.points))
    assert m.nnz == 70917201


def test_schwarz_subdomain_selection():
    e = H.scenes.embedded_cylinder(8)
    b0, b1 = e.blocks
    m = H.EmbeddedModel3d(e.vertices, b0.connectivity, b1.connectivity, (b0.weights, b0.points),
                          (b1.offsets, b1.weights, b1.points))
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(m, e.volume_fractions, 0.5)
    sel = [i for i in range(b1.connectivity.shape[0]) if e.volume_fractions[i] <= 0.5]
    assert len(comp.schwarz_connectivity) == len(sel)
    treated = set(np.concatenate(comp.schwarz_connectivity).tolist())
    assert set(comp.untreated_nodes.tolist()) == set(range(e.vertices.shape[0])) - treated


def test_random_normal_is_seeded():
    a = H.scenes.random_normal(7, 1001, 2.0)
    b = H.scenes.random_normal(7, 1001, 2.0)
    assert np.array_equal(a, b)
    assert abs(a.mean()) < 0.2 and abs(a.std() - 2.0) < 0.2


def test_repeated_node_rejected():
    X = np.random.default_rng(0).random((30, 3))
    conn = np.arange(10, dtype=np.int64).reshape(1, 10)
    conn[0, 5] = conn[0, 4]
    s = H.scenes.tet10_box(1.0, 1, 1, 1, 1)
    with pytest.raises(H.HoefemError) as ei:
        H.NodalModel3d(X, conn, (s.blocks[0].weights, s.blocks[0].points))
    assert ei.value.status == "PATTERN"


def test_compute_without_device_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    s = H.scenes.tet10_box(1.0, 1, 1, 1, 1)
    b = s.blocks[0]
    m = H.NodalModel3d(s.vertices, b.connectivity, (b.weights, b.points))
    with pytest.raises(H.HoefemError) as ei:
        m.assemble_stiffness(np.zeros(m.ndof()), H.StVKMaterial(H.YoungPoisson(1e6, 0.3)))
    assert ei.value.status == "NO_DEVICE"


def test_batch_engine_entry_points_check_arguments():
    L = _capi.lib()
    invalid = [k for k, v in _capi.STATUS.items() if v == "INVALID_ARGUMENT"][0]
    e, c, n = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(0)
    assert L.hoefem_batch_set_cg_engine(None, 0, 0) == invalid
    assert L.hoefem_batch_cg_choice(None, ctypes.byref(e), ctypes.byref(c), None, ctypes.byref(n)) == invalid
    assert _capi.CG_ENGINE == {"auto": 0, "chunked": 1, "streamed": 2}


def test_header_is_plain_c():
    # the boundary is a C ABI: the header compiles as C99 and as C++11
    import shutil
    import subprocess

    hdr = os.path.join(ROOT, "include", "hoefem.h")
    for cc, lang, std in (("gcc", "c", "-std=c99"), ("g++", "c++", "-std=c++11")):
        exe = shutil.which(cc)
        if exe is None:
            pytest.skip("no host compiler")
        subprocess.check_call([exe, std, "-Wall", "-Werror", "-fsyntax-only", "-x", lang, hdr])
