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
