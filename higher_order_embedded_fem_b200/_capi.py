"""ctypes binding of libhoefem.so (the C ABI declared in include/hoefem.h).

The library is built in-tree (python -m higher_order_embedded_fem_b200.build).
There is no fallback: if the shared library is missing the import fails with
an error that says how to build it.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhoefem.so")

HOEFEM_OK = 0
STATUS = {
    0: "OK", 1: "INVALID_ARGUMENT", 2: "CUDA", 3: "OUT_OF_MEMORY", 4: "SINGULAR", 5: "NONFINITE", 6: "PATTERN",
    7: "ZERO_DIAGONAL", 8: "NOT_FINALIZED", 9: "DEVICE_TIMEOUT", 10: "CG_INDEFINITE_OPERATOR", 11: "CG_INDEFINITE_PRECONDITIONER",
    12: "CG_MAX_ITERATIONS", 20: "NEWTON_MAX_ITERATIONS", 21: "LINE_SEARCH_FAILED", 22: "SUBSTEPPING_FAILED",
    31: "NO_DEVICE",
}
MEM_HOST, MEM_DEVICE = 0, 1
ELEM_TET10, ELEM_HEX27 = 1, 3
MAT_STVK, MAT_SNH = 0, 1

vp = C.c_void_p
i64 = C.c_int64
dbl = C.c_double
pi64 = C.POINTER(C.c_int64)
pdbl = C.POINTER(C.c_double)


class HoefemError(RuntimeError):
    def __init__(self, code, message):
        super().__init__("%s (%d): %s" % (STATUS.get(code, "?"), code, message))
        self.code = code
        self.status = STATUS.get(code, "?")


class Material(C.Structure):
    _fields_ = [("kind", C.c_int32), ("mu", C.c_double), ("lam", C.c_double)]


class StepStats(C.Structure):
    _fields_ = [
        ("newton_iterations", C.c_int64), ("num_cg_solves", C.c_int64), ("total_cg_iterations", C.c_int64),
        ("max_cg_iterations", C.c_int64), ("substeps", C.c_int64), ("last_cg_status", C.c_int32),
        ("residual_norm", C.c_double), ("representative_force", C.c_double), ("ms_assemble_forces", C.c_double),
        ("ms_assemble_stiffness", C.c_double), ("ms_precond_update", C.c_double), ("ms_cg", C.c_double),
        ("ms_total", C.c_double), ("learned_accepted", C.c_int64), ("learned_rejected", C.c_int64),
        ("learned_residual_ratio", C.c_double), ("ms_learned", C.c_double), ("line_search_backtracks", C.c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class CgEngineStats(C.Structure):
    _fields_ = [("launches", C.c_int64), ("iterations", C.c_int64), ("device_ms", C.c_double),
                ("operator_bytes", C.c_int64), ("schwarz_bytes", C.c_int64), ("phase_us", C.c_double * 12),
                ("auto_us_per_iteration", C.c_double * 2), ("auto_choice", C.c_int32),
                ("phase_us_max", C.c_double * 12), ("busy_us", C.c_double * 2)]


CG_ENGINE = {"auto": 0, "chunked": 1, "streamed": 2}
STIFFNESS_PATH = {"auto": 0, "cuda_cores": 1, "staged": 2}


class SceneInfo(C.Structure):
    _fields_ = [("num_vertices", C.c_int64), ("num_blocks", C.c_int64), ("block_kind", C.c_int32 * 2),
                ("block_elements", C.c_int64 * 2), ("block_quad_points", C.c_int64 * 2),
                ("block_uniform", C.c_int32 * 2), ("cell_size", C.c_double)]


SIGNATURES = {
    "hoefem_last_error": (C.c_char_p, []),
    "hoefem_abi_version": (C.c_int, []),
    "hoefem_launch_count": (C.c_int, [pi64]),
    "hoefem_set_device": (C.c_int, [C.c_int]),
    "hoefem_lame_from_young_poisson": (C.c_int, [dbl, dbl, pdbl, pdbl]),
    "hoefem_model_create": (C.c_int, [vp, i64, C.POINTER(vp)]),
    "hoefem_model_add_block": (C.c_int, [vp, C.c_int, vp, i64, vp, vp, vp, i64]),
    "hoefem_model_finalize": (C.c_int, [vp]),
    "hoefem_model_destroy": (C.c_int, [vp]),
    "hoefem_model_set_stream": (C.c_int, [vp, vp]),
    "hoefem_model_autotune": (C.c_int, [vp, C.POINTER(C.c_int32)]),
    "hoefem_model_set_spmv_variant": (C.c_int, [vp, C.c_int32]),
    "hoefem_model_set_stiffness_path": (C.c_int, [vp, C.c_int]),
    "hoefem_model_sizes": (C.c_int, [vp, pi64, pi64, pi64, pi64]),
    "hoefem_model_pattern": (C.c_int, [vp, vp, vp]),
    "hoefem_model_num_colors": (C.c_int, [vp, C.c_int, pi64]),
    "hoefem_model_colors": (C.c_int, [vp, C.c_int, vp, vp]),
    "hoefem_assemble_elastic_pseudo_forces_into": (C.c_int, [vp, C.POINTER(Material), vp, vp, C.c_int]),
    "hoefem_assemble_stiffness_into": (C.c_int, [vp, C.POINTER(Material), vp, vp, C.c_int]),
    "hoefem_assemble_stiffness_into_precision": (C.c_int, [vp, C.POINTER(Material), vp, vp, C.c_int, C.c_int]),
    "hoefem_assemble_projected_stiffness_into": (C.c_int, [vp, C.POINTER(Material), vp, vp, C.c_int]),
    "hoefem_jacobian_combination_damped": (C.c_int, [vp, dbl, vp, dbl, vp, dbl, vp, vp, i64, vp, C.c_int]),
    "hoefem_integrator_set_damping": (C.c_int, [vp, C.c_int, dbl, C.c_int, dbl]),
    "hoefem_assemble_mass_into": (C.c_int, [vp, dbl, vp, C.c_int]),
    "hoefem_apply_dirichlet_bc_csr": (C.c_int, [vp, vp, i64, vp, C.c_int]),
    "hoefem_jacobian_combination": (C.c_int, [vp, dbl, vp, dbl, vp, vp, i64, vp, C.c_int]),
    "hoefem_jacobian_combination_noalloc": (C.c_int, [vp, dbl, vp, dbl, vp, vp, i64, vp]),
    "hoefem_spmv": (C.c_int, [vp, dbl, vp, dbl, vp, vp, C.c_int]),
    "hoefem_precond_create_diagonal": (C.c_int, [vp, C.POINTER(vp)]),
    "hoefem_precond_create_schwarz": (C.c_int, [vp, vp, vp, i64, vp, i64, C.POINTER(vp)]),
    "hoefem_precond_update": (C.c_int, [vp, vp, C.c_int]),
    "hoefem_precond_apply": (C.c_int, [vp, vp, vp, C.c_int]),
    "hoefem_precond_set_spmv_variant": (C.c_int, [vp, C.c_int32]),
    "hoefem_precond_get_spmv_variants": (C.c_int, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "hoefem_model_get_spmv_variants": (C.c_int, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "hoefem_precond_nnz": (C.c_int, [vp, pi64]),
    "hoefem_precond_pattern": (C.c_int, [vp, vp, vp]),
    "hoefem_precond_values": (C.c_int, [vp, vp]),
    "hoefem_precond_destroy": (C.c_int, [vp]),
    "hoefem_cg_solve": (C.c_int, [vp, vp, vp, vp, vp, dbl, i64, pi64, C.c_int]),
    "hoefem_cg_solve_mixed": (C.c_int, [vp, vp, vp, vp, vp, dbl, i64, dbl, pi64, C.c_int]),
    "hoefem_integrator_create": (C.c_int, [vp, C.POINTER(Material), dbl, vp, i64, C.c_int, dbl, vp, C.POINTER(vp)]),
    "hoefem_integrator_set_tolerances": (C.c_int, [vp, dbl, i64, i64]),
    "hoefem_integrator_set_precision": (C.c_int, [vp, C.c_int, dbl]),
    "hoefem_integrator_set_cg_engine": (C.c_int, [vp, C.c_int, C.c_int]),
    "hoefem_model_set_cg_engine": (C.c_int, [vp, C.c_int, C.c_int]),
    "hoefem_integrator_cg_engine_stats": (C.c_int, [vp, vp]),
    "hoefem_model_cg_engine_stats": (C.c_int, [vp, vp]),
    "hoefem_integrator_set_cg_l2_keep": (C.c_int, [vp, i64]),
    "hoefem_model_set_cg_l2_keep": (C.c_int, [vp, i64]),
    "hoefem_integrator_step": (C.c_int, [vp, vp, vp, dbl, dbl, C.c_int]),
    "hoefem_integrator_stats": (C.c_int, [vp, C.POINTER(StepStats)]),
    "hoefem_integrator_mass": (C.c_int, [vp, vp]),
    "hoefem_integrator_eval_f": (C.c_int, [vp, vp, vp, vp, C.c_int]),
    "hoefem_integrator_destroy": (C.c_int, [vp]),
    "hoefem_learned_create": (C.c_int, [vp, vp, i64, C.c_int, C.c_uint64, C.POINTER(vp)]),
    "hoefem_learned_destroy": (C.c_int, [vp]),
    "hoefem_learned_num_pairs": (C.c_int, [vp, pi64]),
    "hoefem_learned_num_params": (C.c_int, [vp, pi64]),
    "hoefem_learned_add_pair": (C.c_int, [vp, vp, vp, C.c_int]),
    "hoefem_learned_train": (C.c_int, [vp, i64, C.c_int32, C.c_float, C.c_uint64, vp]),
    "hoefem_learned_forward_backward": (C.c_int, [vp, vp, vp, C.c_int32, C.POINTER(C.c_float), vp, vp]),
    "hoefem_learned_infer": (C.c_int, [vp, vp, C.c_int32, C.c_int32, vp]),
    "hoefem_learned_get_weights": (C.c_int, [vp, vp]),
    "hoefem_learned_set_weights": (C.c_int, [vp, vp]),
    "hoefem_learned_predict": (C.c_int, [vp, vp, vp, C.c_int]),
    "hoefem_integrator_set_learned": (C.c_int, [vp, vp, C.c_int]),
    "hoefem_scene_create_tet10_box": (C.c_int, [dbl, i64, i64, i64, i64, C.POINTER(vp)]),
    "hoefem_scene_create_hex27_box": (C.c_int, [dbl, i64, i64, i64, i64, C.POINTER(vp)]),
    "hoefem_batch_create": (C.c_int, [vp, C.c_int32, vp, dbl, vp, vp, C.c_int, dbl, C.POINTER(vp)]),
    "hoefem_batch_destroy": (C.c_int, [vp]),
    "hoefem_batch_set_stream": (C.c_int, [vp, vp]),
    "hoefem_batch_set_tolerances": (C.c_int, [vp, dbl, i64, i64]),
    "hoefem_batch_set_cg_engine": (C.c_int, [vp, C.c_int32, C.c_int32]),
    "hoefem_batch_cg_choice": (C.c_int, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), vp,
                                         C.POINTER(C.c_int32)]),
    "hoefem_batch_sizes": (C.c_int, [vp, pi64, pi64, pi64, vp]),
    "hoefem_batch_step": (C.c_int, [vp, vp, vp, dbl, dbl, C.c_int]),
    "hoefem_batch_scene_stats": (C.c_int, [vp, C.c_int32, C.POINTER(StepStats), C.POINTER(C.c_int32)]),
    "hoefem_scene_create_embedded_cylinder": (C.c_int, [i64, dbl, dbl, C.c_int, C.c_int, C.c_uint64, C.POINTER(vp)]),
    "hoefem_scene_info_get": (C.c_int, [vp, C.POINTER(SceneInfo)]),
    "hoefem_scene_vertices": (C.c_int, [vp, vp]),
    "hoefem_scene_block": (C.c_int, [vp, C.c_int, vp, vp, vp, vp]),
    "hoefem_scene_volume_fractions": (C.c_int, [vp, vp]),
    "hoefem_scene_nodes_below": (C.c_int, [vp, C.c_int, dbl, vp, pi64]),
    "hoefem_scene_destroy": (C.c_int, [vp]),
    "hoefem_random_normal": (C.c_int, [C.c_uint64, i64, dbl, vp]),
    "hoefem_tet_quadrature": (C.c_int, [C.c_int, vp, vp, vp]),
    "hoefem_precond_set_block_apply": (C.c_int, [vp, C.c_int32]),
    "hoefem_embed_mesh_3d": (C.c_int, [vp, i64, vp, i64, C.c_int, vp, i64, vp, i64, dbl, dbl, vp]),
    "hoefem_embedding_cells": (C.c_int, [vp, vp, vp, vp, vp, vp]),
    "hoefem_embedding_quadrature": (C.c_int, [vp, vp, vp, i64, dbl, vp, vp, i64, vp]),
    "hoefem_embedding_copy_quadrature": (C.c_int, [vp, vp, vp, vp]),
    "hoefem_embedding_destroy": (C.c_int, [vp]),
    "hoefem_quadrature_simplify": (C.c_int, [i64, vp, vp, vp, C.c_int, vp, vp, vp]),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libhoefem.so is not built; run `python -m higher_order_embedded_fem_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def launch_count():
    n = C.c_int64()
    check(lib().hoefem_launch_count(C.byref(n)))
    return n.value


def check(status):
    if status != HOEFEM_OK:
        raise HoefemError(status, lib().hoefem_last_error().decode())
    return status


def is_device_array(a):
    mod = type(a).__module__
    return mod.startswith("torch") and getattr(a, "is_cuda", False)


def ptr(a):
    """(pointer, mem) of a numpy array (host) or a CUDA torch tensor (device)."""
    if a is None:
        return None, MEM_HOST
    if is_device_array(a):
        assert a.is_contiguous(), "device arrays must be contiguous"
        return a.data_ptr(), MEM_DEVICE
    assert isinstance(a, np.ndarray) and a.flags.c_contiguous, "host arrays must be C-contiguous numpy arrays"
    return a.ctypes.data, MEM_HOST


def host_f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def host_i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)
