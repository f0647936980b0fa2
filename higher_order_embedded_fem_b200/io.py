"""VTK output of volume meshes and finite element states (legacy VTK 4.1,
unstructured grid), as the reference writes them for ParaView.

Reference: fenris/src/geometry/vtk.rs (cell types and node orders of
Tet10 / Hex27, write_vtk with version 4.1), simulation_toolbox/src/io/vtk.rs
(create_vtk_filename, VtkVolumeMeshOutput / VtkFemOutput).

    write_vtk_volume_mesh("out/cylinder_volume_mesh_3.vtk", X + u.reshape(-1, 3), scene.blocks,
                          point_data={"displacement": u.reshape(-1, 3)})

Tet10 cells are written as VTK quadratic tetrahedra (the reference's node
order with nodes 8 and 9 swapped, as ParaView orders the last two edges);
Hex27 cells as VTK quadratic (20-node) hexahedra, since legacy VTK has no
tri-quadratic hexahedron: the 8 corners and the 12 edge midpoints, face and
centre nodes dropped.  The file is host output only; the arrays come from the
caller (device arrays must be copied to the host first).
"""
import os

import numpy as np

from ._capi import ELEM_HEX27, ELEM_TET10

VTK_QUADRATIC_TETRA = 24
VTK_QUADRATIC_HEXAHEDRON = 25

# node i of the VTK cell is node ORDER[i] of the element (gmsh order)
TET10_VTK_ORDER = np.array([0, 1, 2, 3, 4, 5, 6, 7, 9, 8])
HEX27_VTK_ORDER = np.array([0, 1, 2, 3, 4, 5, 6, 7, 8, 11, 13, 9, 16, 18, 19, 17, 10, 12, 14, 15])


def create_vtk_filename(object_name, tag, step_index=None):
    """`{object}_{tag}[_{step}].vtk` (simulation_toolbox/src/io/vtk.rs:118-127)."""
    return "%s_%s%s.vtk" % (object_name, tag, "" if step_index is None else "_%d" % step_index)


def vtk_cells(kind, connectivity):
    """(VTK cell type, connectivity in VTK node order) of a block."""
    conn = np.asarray(connectivity, dtype=np.int64)
    if kind == ELEM_TET10:
        if conn.shape[1] != 10:
            raise ValueError("Tet10 connectivity needs 10 nodes per element")
        return VTK_QUADRATIC_TETRA, conn[:, TET10_VTK_ORDER]
    if kind == ELEM_HEX27:
        if conn.shape[1] != 27:
            raise ValueError("Hex27 connectivity needs 27 nodes per element")
        return VTK_QUADRATIC_HEXAHEDRON, conn[:, HEX27_VTK_ORDER]
    raise ValueError("unknown element kind %r" % (kind,))


def write_vtk_volume_mesh(path, vertices, blocks, point_data=None, title="higher_order_embedded_fem"):
    """Writes the cells of `blocks` (objects with .kind and .connectivity, or
    (kind, connectivity) pairs) over `vertices` (nv x 3) as a legacy ASCII
    VTK unstructured grid; `point_data` maps names to per-vertex scalars
    (nv) or vectors (nv x 3)."""
    X = np.asarray(vertices, dtype=np.float64).reshape(-1, 3)
    nv = X.shape[0]
    types, cells = [], []
    for b in blocks:
        kind, conn = (b.kind, b.connectivity) if hasattr(b, "kind") else b
        t, c = vtk_cells(kind, conn)
        if c.size and (c.min() < 0 or c.max() >= nv):
            raise ValueError("connectivity refers to a vertex out of range")
        types.append(np.full(len(c), t, dtype=np.int64))
        cells.append(c)
    ncell = sum(len(c) for c in cells)
    size = sum(c.size + len(c) for c in cells)
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    with open(path, "w") as f:
        f.write("# vtk DataFile Version 4.1\n%s\nASCII\nDATASET UNSTRUCTURED_GRID\n" % title.replace("\n", " "))
        f.write("POINTS %d double\n" % nv)
        np.savetxt(f, X, fmt="%.17g")
        f.write("\nCELLS %d %d\n" % (ncell, size))
        for c in cells:
            np.savetxt(f, np.column_stack([np.full(len(c), c.shape[1]), c]), fmt="%d")
        f.write("\nCELL_TYPES %d\n" % ncell)
        for t in types:
            np.savetxt(f, t, fmt="%d")
        if point_data:
            f.write("\nPOINT_DATA %d\n" % nv)
            for name, arr in point_data.items():
                a = np.asarray(arr, dtype=np.float64)
                if a.ndim == 1 and a.size == nv:
                    f.write("SCALARS %s double 1\nLOOKUP_TABLE default\n" % name)
                    np.savetxt(f, a, fmt="%.17g")
                elif a.size == 3 * nv:
                    f.write("VECTORS %s double\n" % name)
                    np.savetxt(f, a.reshape(nv, 3), fmt="%.17g")
                else:
                    raise ValueError("point data %r has %d entries for %d vertices" % (name, a.size, nv))


def write_fem_vtk(path, reference_vertices, blocks, u, title="higher_order_embedded_fem"):
    """The deformed mesh X + u with the displacement u as point data."""
    X = np.asarray(reference_vertices, dtype=np.float64).reshape(-1, 3)
    U = np.asarray(u, dtype=np.float64).reshape(-1, 3)
    write_vtk_volume_mesh(path, X + U, blocks, {"displacement": U}, title)


def read_vtk_unstructured(path):
    """Reads back what write_vtk_volume_mesh writes: (points, cells as a list
    of node lists, cell types, point data dict)."""
    with open(path) as f:
        tok = f.read().split("\n")
    i = 4
    pts, cells, types, pdata = None, [], [], {}

    def numbers(start, count):
        vals, j = [], start
        while len(vals) < count:
            vals.extend(float(x) for x in tok[j].split())
            j += 1
        return vals, j

    nv = 0
    while i < len(tok):
        line = tok[i].split()
        if not line:
            i += 1
            continue
        if line[0] == "POINTS":
            nv = int(line[1])
            vals, i = numbers(i + 1, 3 * nv)
            pts = np.array(vals).reshape(nv, 3)
        elif line[0] == "CELLS":
            n = int(line[1])
            for k in range(n):
                row = [int(x) for x in tok[i + 1 + k].split()]
                cells.append(row[1:1 + row[0]])
            i += 1 + n
        elif line[0] == "CELL_TYPES":
            n = int(line[1])
            types = [int(tok[i + 1 + k]) for k in range(n)]
            i += 1 + n
        elif line[0] == "SCALARS":
            vals, i = numbers(i + 2, nv)
            pdata[line[1]] = np.array(vals)
        elif line[0] == "VECTORS":
            vals, i = numbers(i + 1, 3 * nv)
            pdata[line[1]] = np.array(vals).reshape(nv, 3)
        else:
            i += 1
    return pts, cells, np.array(types), pdata
