"""Embedded quadrature construction (fenris/src/embedding): the host mirror of
embed_mesh_3d / embed_quadrature_3d / EmbeddedQuadrature::simplified over
the CUDA implementation in libhoefem.so (csrc/embed.cu).

    emb = embed_mesh_3d(bg_vertices, bg_connectivity, tet_vertices, tets)
    quad = embed_quadrature_3d(emb, interior_quadrature, tet_quadrature_strength(3))
    quad = quad.simplified(3)

Background cells are hexahedra given by Hex8 or Hex27 connectivity (the first
8 nodes are the corners, faces planar); the embedded geometry is a Tet4 mesh.
Quadrature points are in the background element's reference coordinates
([-1, 1]^3), as the reference's EmbeddedQuadrature holds them.
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi
from ._capi import check, lib


def tet_quadrature_strength(strength):
    """tet_quadrature_strength_{1,2,3,5} (fenris/src/quadrature.rs:570-781)."""
    n = C.c_int64()
    check(lib().hoefem_tet_quadrature(int(strength), None, None, C.byref(n)))
    w = np.zeros(n.value)
    p = np.zeros((n.value, 3))
    check(lib().hoefem_tet_quadrature(int(strength), w.ctypes.data, p.ctypes.data, None))
    return w, p


@dataclass
class EmbedOptions:
    """EmbedOptions (embedding3d.rs:114-141)."""

    upper_volume_threshold: float = 0.999
    lower_volume_threshold: float = 1e-4


@dataclass
class StabilizationOptions:
    """StabilizationOptions (embedding3d.rs:207-218): `factor` times the
    uncut-cell rule `quadrature` = (weights, points) is appended to every
    interface rule."""

    stabilization_factor: float
    stabilization_quadrature: tuple


class Embedding:
    """Embedding (embedding3d.rs:24-36): exterior / interior / interface cells
    of the background mesh, and the intersection volume of every cell."""

    def __init__(self, handle, num_cells):
        self._h = handle
        self._lib = lib()  # kept for __del__ at interpreter exit
        cls = np.zeros(num_cells, dtype=np.int32)
        cut = np.zeros(num_cells)
        ne, ni, nf = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().hoefem_embedding_cells(handle, C.byref(ne), C.byref(ni), C.byref(nf), cls.ctypes.data,
                                           cut.ctypes.data))
        self.cell_class = cls
        self.cut_volume = cut
        self.exterior_cells = np.nonzero(cls == 0)[0]
        self.interior_cells = np.nonzero(cls == 1)[0]
        self.interface_cells = np.nonzero(cls == 2)[0]

    def __del__(self):
        if getattr(self, "_h", None) and getattr(self, "_lib", None) is not None:
            self._lib.hoefem_embedding_destroy(self._h)
            self._h = None


def embed_mesh_3d(bg_vertices, bg_connectivity, embedded_vertices, embedded_tets, opts=None):
    """embed_mesh_3d_with_opts (embedding3d.rs:152-196)."""
    opts = opts or EmbedOptions()
    bv = _capi.host_f64(bg_vertices).reshape(-1, 3)
    bc = _capi.host_i64(bg_connectivity)
    ev = _capi.host_f64(embedded_vertices).reshape(-1, 3)
    et = _capi.host_i64(embedded_tets).reshape(-1, 4)
    if bc.ndim != 2 or bc.shape[1] not in (8, 27):
        raise ValueError("background connectivity must be num_cells x 8 or x 27")
    h = C.c_void_p()
    check(lib().hoefem_embed_mesh_3d(bv.ctypes.data, bv.shape[0], bc.ctypes.data, bc.shape[0], bc.shape[1],
                                     ev.ctypes.data, ev.shape[0], et.ctypes.data, et.shape[0],
                                     float(opts.lower_volume_threshold), float(opts.upper_volume_threshold),
                                     C.byref(h)))
    return Embedding(h.value, bc.shape[0])


def compute_interface_quadrature_rules(embedding, tet_quadrature, stabilization=None):
    """compute_interface_quadrature_rules (embedding3d.rs:355-397): one rule
    per interface cell, as (offsets, weights, points)."""
    tw = _capi.host_f64(tet_quadrature[0])
    tp = _capi.host_f64(tet_quadrature[1]).reshape(-1, 3)
    if stabilization is not None:
        sw = _capi.host_f64(stabilization.stabilization_quadrature[0])
        sp = _capi.host_f64(stabilization.stabilization_quadrature[1]).reshape(-1, 3)
        fac, swp, spp, ns = float(stabilization.stabilization_factor), sw.ctypes.data, sp.ctypes.data, sw.shape[0]
    else:
        fac, swp, spp, ns = 0.0, None, None, 0
    total = C.c_int64()
    check(lib().hoefem_embedding_quadrature(embedding._h, tw.ctypes.data, tp.ctypes.data, tw.shape[0], fac, swp, spp,
                                            ns, C.byref(total)))
    off = np.zeros(len(embedding.interface_cells) + 1, dtype=np.int64)
    w = np.empty(total.value)
    p = np.empty((total.value, 3))
    check(lib().hoefem_embedding_copy_quadrature(embedding._h, off.ctypes.data, w.ctypes.data, p.ctypes.data))
    return off, w, p


def simplify_rules(offsets, weights, points, strength):
    """optimize_quadrature on every rule (quadrature_reduction.rs:107-190):
    (offsets, weights, points) with at most r points per rule."""
    off = _capi.host_i64(offsets)
    w = _capi.host_f64(weights)
    p = _capi.host_f64(points).reshape(-1, 3)
    oo = np.zeros_like(off)
    ow = np.empty_like(w)
    op = np.empty_like(p)
    check(lib().hoefem_quadrature_simplify(len(off) - 1, off.ctypes.data, w.ctypes.data, p.ctypes.data, int(strength),
                                           oo.ctypes.data, ow.ctypes.data, op.ctypes.data))
    n = int(oo[-1])
    return oo, ow[:n].copy(), op[:n].copy()


class EmbeddedQuadrature:
    """EmbeddedQuadrature (fenris/src/embedding/mod.rs:60-105): the interior
    rule and one rule per interface cell."""

    def __init__(self, interior_quadrature, offsets, weights, points):
        self.interior_quadrature = interior_quadrature
        self.offsets = offsets
        self.weights = weights
        self.points = points

    def interface_quadratures(self):
        o = self.offsets
        return [(self.weights[o[k]:o[k + 1]], self.points[o[k]:o[k + 1]]) for k in range(len(o) - 1)]

    def simplified(self, polynomial_strength):
        """EmbeddedQuadrature::simplified (quadrature_reduction.rs:214-229)."""
        o, w, p = simplify_rules(self.offsets, self.weights, self.points, polynomial_strength)
        return EmbeddedQuadrature(self.interior_quadrature, o, w, p)


def embed_quadrature_3d(embedding, interior_quadrature, tet_quadrature, stabilization=None):
    """embed_quadrature_3d_with_opts (embedding3d.rs:324-353)."""
    o, w, p = compute_interface_quadrature_rules(embedding, tet_quadrature, stabilization)
    return EmbeddedQuadrature(interior_quadrature, o, w, p)


def simplify_quadrature(polynomial_strength, quadrature):
    """simplify_quadrature (quadrature_reduction.rs:232-260)."""
    return quadrature.simplified(polynomial_strength)
