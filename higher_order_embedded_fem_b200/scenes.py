"""Synthetic scenes (input construction) built by libhoefem's host code.

tet10_box        : box of hexes, each split into 6 Tet10 (Max triangulation),
                   tet_quadrature_strength_5 (14 points)
hex27_box        : the same box as Hex27 cells, hex_quadrature_strength_5
embedded_cylinder: Hex27 background grid clipped to a hollow cylinder, interior
                   cells with hex_quadrature_strength_5, interface cells with
                   seeded synthetic quadrature (Q ~ U{q_min..q_max}, weights
                   summing to 8 * volume fraction in reference measure)
random_normal    : seeded N(0, sigma^2) samples (splitmix64 + Box-Muller)
"""
import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _capi
from ._capi import check, lib


@dataclass
class SceneBlock:
    kind: int
    connectivity: np.ndarray
    weights: np.ndarray
    points: np.ndarray
    offsets: np.ndarray = None  # None: uniform rule


@dataclass
class Scene:
    vertices: np.ndarray
    blocks: list
    cell_size: float
    volume_fractions: np.ndarray = field(default=None)

    def nodes_below(self, axis, value):
        return np.nonzero(self.vertices[:, axis] <= value)[0].astype(np.int64)


def _read(h):
    L = lib()
    info = _capi.SceneInfo()
    check(L.hoefem_scene_info_get(h, C.byref(info)))
    X = np.zeros((info.num_vertices, 3))
    check(L.hoefem_scene_vertices(h, X.ctypes.data))
    blocks = []
    for b in range(info.num_blocks):
        nn = 10 if info.block_kind[b] == _capi.ELEM_TET10 else 27
        ne = info.block_elements[b]
        conn = np.zeros((ne, nn), dtype=np.int64)
        nq = info.block_quad_points[b]
        w = np.zeros(nq)
        p = np.zeros((nq, 3))
        off = None if info.block_uniform[b] else np.zeros(ne + 1, dtype=np.int64)
        check(L.hoefem_scene_block(h, b, conn.ctypes.data if ne else None,
                                   None if off is None else off.ctypes.data, w.ctypes.data, p.ctypes.data))
        blocks.append(SceneBlock(info.block_kind[b], conn, w, p, off))
    vf = None
    if info.num_blocks == 2:
        vf = np.zeros(info.block_elements[1])
        if vf.size:
            check(L.hoefem_scene_volume_fractions(h, vf.ctypes.data))
    return Scene(X, blocks, info.cell_size, vf)


def tet10_box(unit=1.0, ux=1, uy=1, uz=1, cells_per_unit=8):
    h = C.c_void_p()
    check(lib().hoefem_scene_create_tet10_box(unit, ux, uy, uz, cells_per_unit, C.byref(h)))
    try:
        return _read(h)
    finally:
        lib().hoefem_scene_destroy(h)


def hex27_box(unit=1.0, ux=1, uy=1, uz=1, cells_per_unit=8):
    h = C.c_void_p()
    check(lib().hoefem_scene_create_hex27_box(unit, ux, uy, uz, cells_per_unit, C.byref(h)))
    try:
        return _read(h)
    finally:
        lib().hoefem_scene_destroy(h)


def embedded_cylinder(n=24, r_inner=0.3, r_outer=0.4, q_min=8, q_max=27, seed=2):
    h = C.c_void_p()
    check(lib().hoefem_scene_create_embedded_cylinder(n, r_inner, r_outer, q_min, q_max, seed, C.byref(h)))
    try:
        return _read(h)
    finally:
        lib().hoefem_scene_destroy(h)


def random_normal(seed, n, sigma):
    out = np.zeros(n)
    check(lib().hoefem_random_normal(seed, n, sigma, out.ctypes.data if n else None))
    return out


def hollow_cylinder_tets(r_inner=0.3, r_outer=0.4, height=1.0, n_r=2, n_theta=48, n_z=24, center=(0.5, 0.5)):
    """Tet4 mesh of a hollow cylinder (axis z, radii [r_inner, r_outer],
    z in [0, height]): a structured (r, theta, z) grid of n_r x n_theta x n_z
    cells, periodic in theta, each cell split into 6 tetrahedra around its
    main diagonal, every tetrahedron positively oriented.  Returns
    (vertices (nv x 3), tets (nt x 4))."""
    r = np.linspace(r_inner, r_outer, n_r + 1)
    th = 2.0 * np.pi * np.arange(n_theta) / n_theta
    z = np.linspace(0.0, height, n_z + 1)
    R, T, Z = np.meshgrid(r, th, z, indexing="ij")
    X = np.stack([center[0] + R * np.cos(T), center[1] + R * np.sin(T), Z], axis=-1).reshape(-1, 3)

    def vid(i, j, k):
        return (i * n_theta + (j % n_theta)) * (n_z + 1) + k

    # cube corners c[b] with b = bit0 (r) + 2 bit1 (theta) + 4 bit2 (z); the
    # 6 tetrahedra of the path decomposition of the diagonal 0 -> 7
    paths = [(1, 2, 4), (1, 4, 2), (2, 1, 4), (2, 4, 1), (4, 1, 2), (4, 2, 1)]
    tets = []
    for i in range(n_r):
        for j in range(n_theta):
            for k in range(n_z):
                c = [vid(i + (b & 1), j + ((b >> 1) & 1), k + ((b >> 2) & 1)) for b in range(8)]
                for p in paths:
                    a1 = p[0]
                    a2 = p[0] | p[1]
                    tets.append([c[0], c[a1], c[a2], c[7]])
    tets = np.array(tets, dtype=np.int64)
    a, b, cc, d = (X[tets[:, k]] for k in range(4))
    det = np.einsum("ij,ij->i", np.cross(b - a, cc - a), d - a)
    flip = det < 0
    tets[flip, 1], tets[flip, 2] = tets[flip, 2].copy(), tets[flip, 1].copy()
    return X, tets


def tet_mesh_volume_moments(vertices, tets):
    """Exact volume, first and second moments (int x_i, int x_i x_j) of a Tet4 mesh."""
    X = np.asarray(vertices, dtype=np.float64)
    P = X[np.asarray(tets)]
    a, b, c, d = P[:, 0], P[:, 1], P[:, 2], P[:, 3]
    V = np.abs(np.einsum("ij,ij->i", np.cross(b - a, c - a), d - a)) / 6.0
    s = P.sum(axis=1)
    m1 = (V[:, None] * s / 4.0).sum(axis=0)
    m2 = np.einsum("t,tij->ij", V / 20.0, np.einsum("tki,tkj->tij", P, P) + np.einsum("ti,tj->tij", s, s))
    return V.sum(), m1, m2


def embedded_cylinder_cut(n=8, r_inner=0.3, r_outer=0.4, n_r=2, n_theta=48, n_z=24, tet_strength=3,
                          simplify_strength=3, stabilization=None):
    """Hex27 background grid (n^3 cells on [0, 1]^3) with the hollow-cylinder
    Tet4 mesh embedded in it, as the reference's embedded scenes are built
    (armadillo_slingshot.rs:446-476): embed_mesh_3d classifies the cells,
    interior cells keep hex_quadrature_strength_5, interface cells get the
    cut-cell rule of tet_quadrature_strength_<tet_strength>, simplified to
    <simplify_strength> (None: not simplified); exterior cells are removed
    and the nodes renumbered in ascending order (keep_cells).  The embedding
    runs on the GPU.  Returns a Scene with two blocks (interior, interface)."""
    from . import embedding as E

    bg = hex27_box(1.0, 1, 1, 1, n)
    conn = bg.blocks[0].connectivity
    X, T = hollow_cylinder_tets(r_inner, r_outer, 1.0, n_r, n_theta, n_z)
    emb = E.embed_mesh_3d(bg.vertices, conn, X, T)
    hw, hp = bg.blocks[0].weights, bg.blocks[0].points
    quad = E.embed_quadrature_3d(emb, (hw, hp), E.tet_quadrature_strength(tet_strength), stabilization)
    if simplify_strength is not None:
        quad = quad.simplified(simplify_strength)
    interior, interface = emb.interior_cells, emb.interface_cells
    used = np.unique(np.concatenate([conn[interior].ravel(), conn[interface].ravel()]))
    remap = -np.ones(len(bg.vertices), dtype=np.int64)
    remap[used] = np.arange(len(used))
    blocks = [SceneBlock(_capi.ELEM_HEX27, remap[conn[interior]], hw.copy(), hp.copy()),
              SceneBlock(_capi.ELEM_HEX27, remap[conn[interface]], quad.weights, quad.points, quad.offsets)]
    h = 1.0 / n
    vf = np.array([quad.weights[quad.offsets[k]:quad.offsets[k + 1]].sum() / 8.0 for k in range(len(interface))])
    s = Scene(bg.vertices[used].copy(), blocks, h, vf)
    s.embedding = emb
    s.embedded_mesh = (X, T)
    return s
