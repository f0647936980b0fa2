"""Elasticity models: NodalModel3d (fenris/src/model.rs:32-117) and
EmbeddedModel3d (fenris/src/embedding/mod.rs:39-59,243-283, 506-648).

Both expose the ElasticityModelParallel surface
(fenris/src/solid/mod.rs:124-172):

  assemble_elastic_pseudo_forces_into_par(f, u, material)  # f += f_int(u)
  assemble_stiffness_into_par(values, u, material)          # values += K(u)
  assemble_mass(density) -> values

Vectors and CSR value arrays are numpy float64 arrays (host memory, copied in
and out by the call) or contiguous CUDA torch float64 tensors (device memory,
used in place).  All arrays of one call must live in the same memory space.
"""
import ctypes as C

import numpy as np

from . import _capi
from ._capi import check, host_f64, host_i64, lib, ptr


def _same_space(*arrays):
    mems = {ptr(a)[1] for a in arrays if a is not None}
    if len(mems) > 1:
        raise ValueError("all arrays of one call must be host arrays or all device tensors")
    return mems.pop() if mems else _capi.MEM_HOST


class _Model:
    def __init__(self, vertices):
        X = host_f64(vertices).reshape(-1, 3)
        h = C.c_void_p()
        check(lib().hoefem_model_create(X.ctypes.data, X.shape[0], C.byref(h)))
        self._h = h
        self._lib = lib()  # kept for __del__ at interpreter exit
        self.num_vertices = X.shape[0]
        self.vertices = X
        self._blocks = []

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and getattr(self, "_lib", None) is not None:
            self._lib.hoefem_model_destroy(h)
            self._h = None

    def _add_block(self, kind, connectivity, weights, points, offsets=None):
        nn = 10 if kind == _capi.ELEM_TET10 else 27
        conn = host_i64(connectivity).reshape(-1, nn)
        if np.ndim(connectivity) == 2 and np.shape(connectivity)[1] != nn:
            raise ValueError("connectivity has %d nodes per element, element kind needs %d"
                             % (np.shape(connectivity)[1], nn))
        w = host_f64(weights)
        p = host_f64(points).reshape(-1, 3)
        off = None if offsets is None else host_i64(offsets)
        check(lib().hoefem_model_add_block(self._h, kind, conn.ctypes.data, conn.shape[0],
                                           None if off is None else off.ctypes.data, w.ctypes.data, p.ctypes.data,
                                           w.shape[0]))
        self._blocks.append((kind, conn.shape[0]))

    def _finalize(self):
        check(lib().hoefem_model_finalize(self._h))
        nd, nz, ne, nb = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().hoefem_model_sizes(self._h, C.byref(nd), C.byref(nz), C.byref(ne), C.byref(nb)))
        self._ndof, self.nnz, self.num_elements = nd.value, nz.value, ne.value

    def autotune(self):
        """Picks the fastest lanes-per-node SpMV variant for this pattern."""
        lanes = C.c_int32()
        check(lib().hoefem_model_autotune(self._h, C.byref(lanes)))
        return lanes.value

    def spmv_variants(self):
        """(FP64-value variant, FP32-value variant) in use."""
        a, b = C.c_int32(), C.c_int32()
        check(lib().hoefem_model_get_spmv_variants(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_spmv_variant(self, variant):
        """8 / 16 / 32 lanes per node, +100 for the column-streaming traversal."""
        check(lib().hoefem_model_set_spmv_variant(self._h, int(variant)))

    def set_stiffness_path(self, path="auto"):
        """Element stiffness / force implementation: "auto" (FP32 Tet10 blocks
        on the tensor cores where they qualify, the rest staged whole-block
        CUDA-core kernels), "staged" (no tensor cores) or "cuda_cores" (colored
        scatter) (hoefem_model_set_stiffness_path)."""
        check(lib().hoefem_model_set_stiffness_path(self._h, _capi.STIFFNESS_PATH[path]))

    def set_cg_engine(self, engine="auto", schwarz_fp16=False, phase_profile=False):
        """CG engine of ConjugateGradient solves on this model ("auto",
        "chunked", "streamed"; see hoefem_model_set_cg_engine)."""
        check(lib().hoefem_model_set_cg_engine(self._h, _capi.CG_ENGINE[engine],
                                                         (1 if schwarz_fp16 else 0) | (2 if phase_profile else 0)))

    def set_cg_l2_keep(self, nbytes=-1):
        """L2 residency budget (bytes) of the streamed CG; -1: the default (0)."""
        check(lib().hoefem_model_set_cg_l2_keep(self._h, int(nbytes)))

    def cg_engine_stats(self):
        """Streamed-CG counters of the last ConjugateGradient solve."""
        s = _capi.CgEngineStats()
        check(lib().hoefem_model_cg_engine_stats(self._h, C.byref(s)))
        out = {f: getattr(s, f) for f, _ in s._fields_}
        out["phase_us"] = list(out["phase_us"])
        for k in ("auto_us_per_iteration", "phase_us_max", "busy_us"):
            out[k] = list(out[k])
        return out

    def set_stream(self, stream):
        """Run this model's work on a CUDA stream handle (int), None: own stream."""
        check(lib().hoefem_model_set_stream(self._h, stream))

    # ---- ElasticityModel --------------------------------------------------------
    def ndof(self):
        return self._ndof

    def pattern(self):
        """(row_offsets, column_indices) of the shared CSR pattern (int64)."""
        ro = np.zeros(self._ndof + 1, dtype=np.int64)
        ci = np.zeros(max(self.nnz, 1), dtype=np.int64)
        check(lib().hoefem_model_pattern(self._h, ro.ctypes.data, ci.ctypes.data))
        return ro, ci[: self.nnz]

    def colors(self, block=0):
        """List of element-label arrays, one per color (DisjointSubsets labels)."""
        nc = C.c_int64()
        check(lib().hoefem_model_num_colors(self._h, block, C.byref(nc)))
        off = np.zeros(nc.value + 1, dtype=np.int64)
        lab = np.zeros(max(self._blocks[block][1], 1), dtype=np.int64)
        check(lib().hoefem_model_colors(self._h, block, off.ctypes.data, lab.ctypes.data))
        return [lab[off[c]:off[c + 1]].copy() for c in range(nc.value)]

    def assemble_elastic_pseudo_forces_into_par(self, f, u, material):
        mem = _same_space(f, u)
        check(lib().hoefem_assemble_elastic_pseudo_forces_into(self._h, C.byref(material.descriptor()), ptr(u)[0],
                                                               ptr(f)[0], mem))
        return f

    def assemble_elastic_pseudo_forces(self, u, material):
        f = np.zeros(self._ndof) if not _capi.is_device_array(u) else u.new_zeros(self._ndof)
        return self.assemble_elastic_pseudo_forces_into_par(f, u, material)

    def assemble_stiffness_into_par(self, values, u, material):
        mem = _same_space(values, u)
        check(lib().hoefem_assemble_stiffness_into(self._h, C.byref(material.descriptor()), ptr(u)[0],
                                                   ptr(values)[0], mem))
        return values

    def assemble_stiffness_into_precision(self, values, u, material, mixed):
        """Stiffness with FP32 element arithmetic when `mixed` (FP64 accumulation)."""
        mem = _same_space(values, u)
        check(lib().hoefem_assemble_stiffness_into_precision(self._h, C.byref(material.descriptor()), ptr(u)[0],
                                                             ptr(values)[0], 1 if mixed else 0, mem))
        return values

    def assemble_stiffness(self, u, material):
        v = np.zeros(self.nnz) if not _capi.is_device_array(u) else u.new_zeros(self.nnz)
        return self.assemble_stiffness_into_par(v, u, material)

    def assemble_mass_into(self, values, density):
        mem = _same_space(values)
        check(lib().hoefem_assemble_mass_into(self._h, float(density), ptr(values)[0], mem))
        return values

    def assemble_mass(self, density):
        return self.assemble_mass_into(np.zeros(self.nnz), density)

    def apply_dirichlet_bc_csr(self, values, nodes):
        """apply_homogeneous_dirichlet_bc_csr (assembly.rs:799-869), in place."""
        nodes = host_i64(nodes)
        mem = _same_space(values)
        check(lib().hoefem_apply_dirichlet_bc_csr(self._h, nodes.ctypes.data if nodes.size else None, nodes.size,
                                                  ptr(values)[0], mem))
        return values

    def assemble_projected_stiffness_into_par(self, values, u, material):
        """values += K(u) with every element matrix projected onto PSD
        (DefaultSemidefiniteProjection, assembly.rs:549-564)."""
        mem = _same_space(values, u)
        check(lib().hoefem_assemble_projected_stiffness_into(self._h, C.byref(material.descriptor()), ptr(u)[0],
                                                             ptr(values)[0], mem))
        return values

    def jacobian_combination_damped(self, out, c_stiffness, stiffness, c_damping, damping, c_mass, mass,
                                    bc_nodes=()):
        """out = c_k K + c_d D + c_m M (summed in that order), then Dirichlet."""
        bc = host_i64(bc_nodes)
        mem = _same_space(out, stiffness, damping, mass)
        check(lib().hoefem_jacobian_combination_damped(self._h, float(c_stiffness), ptr(stiffness)[0],
                                                       float(c_damping), ptr(damping)[0], float(c_mass),
                                                       ptr(mass)[0], bc.ctypes.data if bc.size else None, bc.size,
                                                       ptr(out)[0], mem))
        return out

    def jacobian_combination(self, out, c_stiffness, stiffness, c_mass, mass, bc_nodes=()):
        bc = host_i64(bc_nodes)
        mem = _same_space(out, stiffness, mass)
        check(lib().hoefem_jacobian_combination(self._h, float(c_stiffness), ptr(stiffness)[0], float(c_mass),
                                                ptr(mass)[0], bc.ctypes.data if bc.size else None, bc.size,
                                                ptr(out)[0], mem))
        return out

    def jacobian_combination_noalloc(self, out, c_stiffness, stiffness, c_mass, mass, bc_nodes=()):
        """jacobian_combination on device tensors with no device allocation
        (scratch preallocated in the library; see
        hoefem_jacobian_combination_noalloc for the limits)."""
        for a in (out, stiffness, mass):
            if a is not None and not _capi.is_device_array(a):
                raise ValueError("device tensors only")
        bc = host_i64(bc_nodes)
        check(lib().hoefem_jacobian_combination_noalloc(self._h, float(c_stiffness), ptr(stiffness)[0],
                                                        float(c_mass), ptr(mass)[0],
                                                        bc.ctypes.data if bc.size else None, bc.size,
                                                        ptr(out)[0]))
        return out

    def spmv(self, y, values, x, alpha=1.0, beta=0.0):
        """y = beta y + alpha A x (spmv_csr, sparse.rs:1164-1199)."""
        mem = _same_space(y, values, x)
        check(lib().hoefem_spmv(self._h, float(beta), ptr(y)[0], float(alpha), ptr(values)[0], ptr(x)[0], mem))
        return y


class NodalModel3d(_Model):
    """One Tet10 (or Hex27) block with a uniform quadrature rule."""

    def __init__(self, vertices, connectivity, quadrature, element_kind=_capi.ELEM_TET10):
        super().__init__(vertices)
        w, p = quadrature
        self._add_block(element_kind, connectivity, w, p)
        self._finalize()

    @staticmethod
    def from_mesh_and_quadrature(vertices, connectivity, quadrature, element_kind=_capi.ELEM_TET10):
        return NodalModel3d(vertices, connectivity, quadrature, element_kind)


class EmbeddedModel3d(_Model):
    """Interior block (uniform rule) followed by an interface block (one rule
    per element), each with its own coloring."""

    def __init__(self, vertices, interior_connectivity, interface_connectivity, interior_quadrature,
                 interface_quadrature, element_kind=_capi.ELEM_HEX27):
        super().__init__(vertices)
        w, p = interior_quadrature
        self._add_block(element_kind, interior_connectivity, w, p)
        off, wf, pf = interface_quadrature
        self._add_block(element_kind, interface_connectivity, wf, pf, offsets=off)
        self._finalize()
        self.num_interior = int(np.asarray(interior_connectivity).shape[0])
        self.interface_connectivity = host_i64(interface_connectivity)
