"""VTK output (higher_order_embedded_fem_b200.io): legacy unstructured grids
as the reference writes them (fenris/src/geometry/vtk.rs).  The node orders
are checked against VTK's own cell definitions through the geometry: every
mid-edge node of a written cell must be the midpoint of the corner pair that
VTK assigns to that position.  Points and point data round-trip exactly."""
import numpy as np
import pytest

import higher_order_embedded_fem_b200 as H
from higher_order_embedded_fem_b200 import io as vtkio

# VTK edge tables (corner pairs of the mid-edge nodes, in VTK node order)
VTK_TETRA_EDGES = [(0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3)]
VTK_HEX_EDGES = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)]


def _check_midpoints(X, cells, edges):
    for c in cells:
        for k, (a, b) in enumerate(edges):
            assert np.allclose(X[c[len(c) - len(edges) + k]], 0.5 * (X[c[a]] + X[c[b]]), atol=1e-14)


def test_tet10_cells_follow_vtk_quadratic_tetra(tmp_path):
    s = H.scenes.tet10_box(1.0, 1, 1, 1, 2)
    u = H.scenes.random_normal(1, 3 * len(s.vertices), 0.01).reshape(-1, 3)
    p = tmp_path / vtkio.create_vtk_filename("box", "volume_mesh", 3)
    assert p.name == "box_volume_mesh_3.vtk"
    vtkio.write_fem_vtk(str(p), s.vertices, s.blocks, u)
    pts, cells, types, pdata = vtkio.read_vtk_unstructured(str(p))
    assert np.array_equal(pts, s.vertices + u)
    assert np.array_equal(pdata["displacement"], u)
    assert np.all(types == vtkio.VTK_QUADRATIC_TETRA) and len(cells) == len(s.blocks[0].connectivity)
    _check_midpoints(s.vertices, cells, VTK_TETRA_EDGES)


def test_hex27_cells_follow_vtk_quadratic_hexahedron(tmp_path):
    s = H.scenes.hex27_box(1.0, 2, 1, 1, 2)
    p = tmp_path / vtkio.create_vtk_filename("box", "volume_mesh")
    assert p.name == "box_volume_mesh.vtk"
    phi = np.arange(len(s.vertices), dtype=np.float64)
    vtkio.write_vtk_volume_mesh(str(p), s.vertices, s.blocks, {"node": phi})
    pts, cells, types, pdata = vtkio.read_vtk_unstructured(str(p))
    assert np.array_equal(pts, s.vertices) and np.array_equal(pdata["node"], phi)
    assert np.all(types == vtkio.VTK_QUADRATIC_HEXAHEDRON) and all(len(c) == 20 for c in cells)
    _check_midpoints(s.vertices, cells, VTK_HEX_EDGES)


def test_embedded_scene_two_blocks_and_bad_input(tmp_path):
    e = H.scenes.embedded_cylinder(4)
    p = tmp_path / "cyl.vtk"
    vtkio.write_vtk_volume_mesh(str(p), e.vertices, e.blocks)
    pts, cells, types, _ = vtkio.read_vtk_unstructured(str(p))
    assert len(cells) == sum(len(b.connectivity) for b in e.blocks)
    with pytest.raises(ValueError):
        vtkio.write_vtk_volume_mesh(str(p), e.vertices[:10], e.blocks)
    with pytest.raises(ValueError):
        vtkio.write_vtk_volume_mesh(str(p), e.vertices, e.blocks, {"x": np.zeros(7)})
    with pytest.raises(ValueError):
        vtkio.vtk_cells(H.ELEM_TET10, e.blocks[0].connectivity)
