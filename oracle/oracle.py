"""ctypes wrapper of liboracle.so — TEST INFRASTRUCTURE ONLY.

The FP64 CPU restatement of the reference path (hoefem_oracle.cpp).  The
CUDA library's results are compared with it, and it is the timed CPU
baseline; the product package never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")

MAT_STVK, MAT_SNH, MAT_LINEAR = 0, 1, 2
ELEM_TET4, ELEM_TET10, ELEM_HEX8, ELEM_HEX27 = 0, 1, 2, 3
NODES = {ELEM_TET4: 4, ELEM_TET10: 10, ELEM_HEX8: 8, ELEM_HEX27: 27}


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp = C.c_void_p
        sig = {
            "oracle_last_error": (C.c_char_p, []),
            "oracle_num_threads": (C.c_int, []),
            "oracle_set_num_threads": (None, [C.c_int]),
            "oracle_lame_from_young_poisson": (None, [C.c_double, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
            "oracle_material_stress": (C.c_int, [C.c_int, C.c_double, C.c_double, f64p, f64p]),
            "oracle_material_energy": (C.c_double, [C.c_int, C.c_double, C.c_double, f64p]),
            "oracle_material_contract": (C.c_int, [C.c_int, C.c_double, C.c_double, f64p, f64p, f64p, f64p]),
            "oracle_material_contract_multiple": (C.c_int, [C.c_int, C.c_double, C.c_double, f64p, f64p, C.c_int, f64p]),
            "oracle_snh_dp_df": (C.c_int, [C.c_double, C.c_double, f64p, f64p]),
            "oracle_element_basis": (None, [C.c_int, f64p, f64p]),
            "oracle_element_gradients": (None, [C.c_int, f64p, f64p]),
            "oracle_element_force": (C.c_int, [C.c_int, f64p, f64p, f64p, f64p, C.c_int, C.c_int, C.c_double, C.c_double, f64p]),
            "oracle_element_stiffness": (C.c_int, [C.c_int, f64p, f64p, f64p, f64p, C.c_int, C.c_int, C.c_double, C.c_double, f64p]),
            "oracle_element_mass": (None, [C.c_int, f64p, f64p, f64p, C.c_int, C.c_double, f64p]),
            "oracle_pattern_create": (vp, [i64p, i64p, C.c_int64, C.c_int, C.c_int64]),
            "oracle_pattern_nnz": (C.c_int64, [vp]),
            "oracle_pattern_nrows": (C.c_int64, [vp]),
            "oracle_pattern_copy": (None, [vp, i64p, i64p]),
            "oracle_pattern_destroy": (None, [vp]),
            "oracle_greedy_coloring": (C.c_int64, [i64p, i64p, C.c_int64, i64p, i64p]),
            "oracle_dirichlet_csr": (None, [C.c_int64, i64p, i64p, f64p, i64p, C.c_int64, C.c_int]),
            "oracle_cg_dense": (C.c_int, [C.c_int64, f64p, vp, f64p, f64p, C.c_double, C.c_int64, C.POINTER(C.c_int64)]),
            "oracle_invert_block": (None, [C.c_int, f64p, f64p]),
            "oracle_mesh_hex_box": (vp, [C.c_double, C.c_int64, C.c_int64, C.c_int64, C.c_int64]),
            "oracle_mesh_tets_from_hex": (vp, [vp, C.c_int]),
            "oracle_mesh_hex27_from_hex": (vp, [vp]),
            "oracle_mesh_keep_cells": (vp, [vp, i64p, C.c_int64]),
            "oracle_mesh_num_vertices": (C.c_int64, [vp]),
            "oracle_mesh_num_cells": (C.c_int64, [vp]),
            "oracle_mesh_cell_size": (C.c_int, [vp]),
            "oracle_mesh_copy": (None, [vp, f64p, i64p]),
            "oracle_mesh_destroy": (None, [vp]),
            "oracle_scene_create": (vp, [f64p, C.c_int64]),
            "oracle_scene_add_block": (C.c_int, [vp, C.c_int, i64p, C.c_int64, vp, f64p, f64p, C.c_int64]),
            "oracle_scene_block_colors": (C.c_int64, [vp, C.c_int, vp, vp]),
            "oracle_scene_finalize_pattern": (C.c_int, [vp]),
            "oracle_scene_nnz": (C.c_int64, [vp]),
            "oracle_scene_pattern": (None, [vp, i64p, i64p]),
            "oracle_scene_set_material": (None, [vp, C.c_int, C.c_double, C.c_double, C.c_double]),
            "oracle_scene_assemble_forces": (C.c_int, [vp, f64p, f64p]),
            "oracle_scene_assemble_stiffness": (C.c_int, [vp, f64p, f64p]),
            "oracle_scene_assemble_mass": (None, [vp, C.c_double, f64p]),
            "oracle_scene_set_bc": (None, [vp, i64p, C.c_int64]),
            "oracle_scene_set_gravity": (None, [vp, C.c_int, C.c_double]),
            "oracle_scene_set_solver": (None, [vp, C.c_double, C.c_int64, C.c_int64]),
            "oracle_scene_set_damping": (None, [vp, C.c_int, C.c_double, C.c_int, C.c_double]),
            "oracle_scene_damping": (C.c_int, [vp, f64p, f64p]),
            "oracle_scene_assemble_stiffness_projected": (C.c_int, [vp, f64p, f64p]),
            "oracle_scene_set_schwarz": (None, [vp, i64p, i64p, C.c_int64, i64p, C.c_int64]),
            "oracle_scene_setup": (C.c_int, [vp]),
            "oracle_scene_mass": (None, [vp, f64p]),
            "oracle_scene_representative_force": (C.c_double, [vp]),
            "oracle_scene_schwarz_nnz": (C.c_int64, [vp]),
            "oracle_scene_schwarz_pattern": (None, [vp, i64p, i64p]),
            "oracle_scene_schwarz_update": (C.c_int, [vp, f64p, f64p]),
            "oracle_scene_jacobian": (None, [vp, f64p, C.c_double, f64p]),
            "oracle_scene_cg": (C.c_int, [vp, f64p, f64p, f64p, C.c_double, C.c_int64, C.POINTER(C.c_int64)]),
            "oracle_scene_eval_f": (C.c_int, [vp, f64p, f64p, f64p]),
            "oracle_scene_step": (C.c_int, [vp, f64p, f64p, C.c_double, C.c_double]),
            "oracle_scene_last_newton_iters": (C.c_int64, [vp]),
            "oracle_scene_last_num_cg": (C.c_int64, [vp]),
            "oracle_scene_last_cg": (None, [vp, i64p, i32p]),
            "oracle_scene_last_substeps": (C.c_int64, [vp]),
            "oracle_scene_last_ls_backtracks": (C.c_int64, [vp]),
            "oracle_scene_last_residual": (C.c_double, [vp]),
            "oracle_scene_destroy": (None, [vp]),
            "oracle_embed_last_error": (C.c_char_p, []),
            "oracle_embed_create": (vp, [f64p, C.c_int64, i64p, C.c_int64, C.c_int, f64p, C.c_int64, i64p, C.c_int64,
                                         C.c_double, C.c_double]),
            "oracle_embed_destroy": (None, [vp]),
            "oracle_embed_cells": (None, [vp, i32p, vp]),
            "oracle_embed_quadrature": (C.c_int64, [vp, f64p, f64p, C.c_int, C.c_double, vp, vp, C.c_int]),
            "oracle_embed_copy_quadrature": (None, [vp, i64p, f64p, f64p]),
            "oracle_quadrature_simplify": (C.c_int, [C.c_int64, i64p, f64p, f64p, C.c_int, i64p, f64p, f64p]),
            "oracle_moment_matrix": (C.c_int, [f64p, C.c_int, C.c_int, vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def set_num_threads(n):
    lib().oracle_set_num_threads(int(n))


def num_threads():
    return lib().oracle_num_threads()


def lame(young, poisson):
    mu, lam = C.c_double(), C.c_double()
    lib().oracle_lame_from_young_poisson(young, poisson, C.byref(mu), C.byref(lam))
    return mu.value, lam.value


def stress(kind, mu, lam, F):
    P = np.zeros(9)
    if lib().oracle_material_stress(kind, mu, lam, f64(F).reshape(9), P):
        raise ArithmeticError("singular deformation gradient")
    return P.reshape(3, 3)


def energy(kind, mu, lam, F):
    return lib().oracle_material_energy(kind, mu, lam, f64(F).reshape(9))


def contract(kind, mu, lam, F, a, b):
    out = np.zeros(9)
    if lib().oracle_material_contract(kind, mu, lam, f64(F).reshape(9), f64(a), f64(b), out):
        raise ArithmeticError("singular deformation gradient")
    return out.reshape(3, 3)


def contract_multiple(kind, mu, lam, F, a, out):
    """a: 3 x n; out (3n x 3n) is added into (in place)."""
    a = f64(a)
    assert out.flags.c_contiguous and out.dtype == np.float64
    if lib().oracle_material_contract_multiple(kind, mu, lam, f64(F).reshape(9), a, a.shape[1], out):
        raise ArithmeticError("singular deformation gradient")
    return out


def snh_dp_df(mu, lam, F):
    Cm = np.zeros(81)
    lib().oracle_snh_dp_df(mu, lam, f64(F).reshape(9), Cm)
    return Cm.reshape(9, 9)


def basis(kind, xi):
    N = np.zeros(NODES[kind])
    lib().oracle_element_basis(kind, f64(xi), N)
    return N


def gradients(kind, xi):
    g = np.zeros(3 * NODES[kind])
    lib().oracle_element_gradients(kind, f64(xi), g)
    return g.reshape(3, NODES[kind])


def element_force(kind, X, ue, qw, qp, mat_kind, mu, lam):
    n = NODES[kind]
    fe = np.zeros(3 * n)
    if lib().oracle_element_force(kind, f64(X).reshape(-1), f64(ue).reshape(-1), f64(qw), f64(qp).reshape(-1),
                                  len(qw), mat_kind, mu, lam, fe):
        raise ArithmeticError("element force failed")
    return fe.reshape(3, n)


def element_stiffness(kind, X, ue, qw, qp, mat_kind, mu, lam):
    n = NODES[kind]
    Ke = np.zeros(9 * n * n)
    if lib().oracle_element_stiffness(kind, f64(X).reshape(-1), f64(ue).reshape(-1), f64(qw), f64(qp).reshape(-1),
                                      len(qw), mat_kind, mu, lam, Ke):
        raise ArithmeticError("element stiffness failed")
    return Ke.reshape(3 * n, 3 * n)


def element_mass(kind, X, qw, qp, density):
    n = NODES[kind]
    Me = np.zeros(9 * n * n)
    lib().oracle_element_mass(kind, f64(X).reshape(-1), f64(qw), f64(qp).reshape(-1), len(qw), density, Me)
    return Me.reshape(3 * n, 3 * n)


def _ragged(elems):
    offs = np.zeros(len(elems) + 1, dtype=np.int64)
    for i, e in enumerate(elems):
        offs[i + 1] = offs[i] + len(e)
    flat = np.array([x for e in elems for x in e], dtype=np.int64)
    if flat.size == 0:
        flat = np.zeros(1, dtype=np.int64)
    return offs, flat


def pattern(elems, sdim, num_nodes):
    offs, flat = _ragged(elems)
    L = lib()
    p = L.oracle_pattern_create(offs, flat, len(elems), sdim, num_nodes)
    if not p:
        raise ValueError(L.oracle_last_error().decode())
    nnz, nrows = L.oracle_pattern_nnz(p), L.oracle_pattern_nrows(p)
    ro = np.zeros(nrows + 1, dtype=np.int64)
    ci = np.zeros(max(nnz, 1), dtype=np.int64)
    L.oracle_pattern_copy(p, ro, ci)
    L.oracle_pattern_destroy(p)
    return ro, ci[:nnz]


def coloring(elems):
    offs, flat = _ragged(elems)
    co = np.zeros(len(elems) + 2, dtype=np.int64)
    lab = np.zeros(max(len(elems), 1), dtype=np.int64)
    nc = lib().oracle_greedy_coloring(offs, flat, len(elems), co, lab)
    return [lab[co[c]:co[c + 1]].tolist() for c in range(nc)]


def dirichlet_csr(row_offsets, cols, values, nodes, dim):
    values = f64(values).copy()
    nodes = i64(nodes)
    lib().oracle_dirichlet_csr(len(row_offsets) - 1, i64(row_offsets), i64(cols), values, nodes, len(nodes), dim)
    return values


def cg_dense(A, b, x0, tol, max_iter=-1, P=None):
    A = f64(A)
    n = A.shape[0]
    x = f64(x0).copy()
    it = C.c_int64()
    Pp = f64(P) if P is not None else None
    st = lib().oracle_cg_dense(n, A.reshape(-1), Pp.ctypes.data if Pp is not None else None, f64(b), x, tol,
                               max_iter, C.byref(it))
    return st, x, it.value


def invert_block(A):
    A = f64(A)
    out = np.zeros_like(A)
    lib().oracle_invert_block(A.shape[0], A.reshape(-1), out.reshape(-1))
    return out


class Mesh:
    def __init__(self, handle):
        L = lib()
        self._h = handle
        nv, nc, cs = L.oracle_mesh_num_vertices(handle), L.oracle_mesh_num_cells(handle), L.oracle_mesh_cell_size(handle)
        self.vertices = np.zeros((nv, 3))
        self.cells = np.zeros((nc, cs), dtype=np.int64)
        L.oracle_mesh_copy(handle, self.vertices.reshape(-1), self.cells.reshape(-1) if nc else np.zeros(1, np.int64))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_mesh_destroy(self._h)
            self._h = None


def hex_box(unit, ux, uy, uz, cells_per_unit):
    return Mesh(lib().oracle_mesh_hex_box(unit, ux, uy, uz, cells_per_unit))


def tets_from_hex(hexmesh, tet10=True):
    h = lib().oracle_mesh_tets_from_hex(hexmesh._h, 1 if tet10 else 0)
    if not h:
        raise ValueError(lib().oracle_last_error().decode())
    return Mesh(h)


def hex27_from_hex(hexmesh):
    return Mesh(lib().oracle_mesh_hex27_from_hex(hexmesh._h))


def keep_cells(mesh, cells):
    return Mesh(lib().oracle_mesh_keep_cells(mesh._h, i64(cells), len(cells)))


class Scene:
    """Model + material + integrator state: the NewtonCgIntegrator3d path."""

    def __init__(self, vertices):
        X = f64(vertices).reshape(-1)
        self.num_nodes = X.size // 3
        self.ndof = 3 * self.num_nodes
        self._h = lib().oracle_scene_create(X, self.num_nodes)
        self.blocks = []

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_scene_destroy(self._h)
            self._h = None

    def add_block(self, kind, conn, qw, qp, qoff=None):
        conn = i64(conn)
        qw, qp = f64(qw), f64(qp).reshape(-1)
        qo = i64(qoff) if qoff is not None else None
        self._keep = getattr(self, "_keep", []) + [qo]
        lib().oracle_scene_add_block(self._h, kind, conn.reshape(-1) if conn.size else np.zeros(1, np.int64),
                                     conn.shape[0], qo.ctypes.data if qo is not None else None, qw, qp, qw.size)
        self.blocks.append(kind)

    def colors(self, bi):
        L = lib()
        nc = L.oracle_scene_block_colors(self._h, bi, None, None)
        co = np.zeros(nc + 1, dtype=np.int64)
        tot = 1 << 26
        lab = np.zeros(tot, dtype=np.int64)
        L.oracle_scene_block_colors(self._h, bi, co.ctypes.data, lab.ctypes.data)
        return co, lab[: co[-1]].copy()

    def finalize_pattern(self):
        L = lib()
        if L.oracle_scene_finalize_pattern(self._h):
            raise ValueError(L.oracle_last_error().decode())
        self.nnz = L.oracle_scene_nnz(self._h)

    def pattern(self):
        ro = np.zeros(self.ndof + 1, dtype=np.int64)
        ci = np.zeros(self.nnz, dtype=np.int64)
        lib().oracle_scene_pattern(self._h, ro, ci)
        return ro, ci

    def set_material(self, kind, mu, lam, density=1000.0):
        lib().oracle_scene_set_material(self._h, kind, mu, lam, density)

    def forces(self, u, f=None):
        f = np.zeros(self.ndof) if f is None else f64(f).copy()
        if lib().oracle_scene_assemble_forces(self._h, f64(u), f):
            raise ArithmeticError("force assembly failed")
        return f

    def stiffness(self, u):
        v = np.zeros(self.nnz)
        r = lib().oracle_scene_assemble_stiffness(self._h, f64(u), v)
        if r:
            raise ArithmeticError("stiffness assembly failed")
        return v

    def mass_values(self, density):
        v = np.zeros(self.nnz)
        lib().oracle_scene_assemble_mass(self._h, density, v)
        return v

    def set_bc(self, nodes):
        nodes = i64(nodes)
        lib().oracle_scene_set_bc(self._h, nodes if nodes.size else np.zeros(1, np.int64), nodes.size)

    def set_gravity(self, enabled, g=-9.81):
        lib().oracle_scene_set_gravity(self._h, 1 if enabled else 0, g)

    def set_solver(self, cg_tol, cg_max_iter=500, newton_max_iter=100):
        lib().oracle_scene_set_solver(self._h, cg_tol, cg_max_iter, newton_max_iter)

    def set_schwarz(self, subdomains, untreated):
        offs, flat = _ragged(subdomains)
        un = i64(untreated)
        lib().oracle_scene_set_schwarz(self._h, offs, flat, len(subdomains), un if un.size else np.zeros(1, np.int64),
                                       un.size)

    def setup(self):
        L = lib()
        if L.oracle_scene_setup(self._h):
            raise ValueError(L.oracle_last_error().decode())

    def mass(self):
        v = np.zeros(self.nnz)
        lib().oracle_scene_mass(self._h, v)
        return v

    def representative_force(self):
        return lib().oracle_scene_representative_force(self._h)

    def schwarz_pattern(self):
        nnz = lib().oracle_scene_schwarz_nnz(self._h)
        ro = np.zeros(self.ndof + 1, dtype=np.int64)
        ci = np.zeros(nnz, dtype=np.int64)
        lib().oracle_scene_schwarz_pattern(self._h, ro, ci)
        return ro, ci

    def schwarz_update(self, jv):
        nnz = lib().oracle_scene_schwarz_nnz(self._h)
        pv = np.zeros(nnz)
        if lib().oracle_scene_schwarz_update(self._h, f64(jv), pv):
            raise ArithmeticError("schwarz update failed")
        return pv

    def stiffness_projected(self, u):
        """Stiffness with every element matrix projected onto PSD (eigenvalues
        clamped at zero) before the scatter."""
        v = np.zeros(self.nnz)
        if lib().oracle_scene_assemble_stiffness_projected(self._h, f64(u), v):
            raise ArithmeticError("stiffness assembly failed")
        return v

    def set_damping(self, mass=None, stiffness=None):
        """D = mass * M + stiffness * K_proj(u) at the start of every (sub)step;
        None = term absent (Option::None in the reference)."""
        lib().oracle_scene_set_damping(self._h, 0 if mass is None else 1, 0.0 if mass is None else float(mass),
                                       0 if stiffness is None else 1, 0.0 if stiffness is None else float(stiffness))

    def damping(self, u):
        d = np.zeros(self.nnz)
        if lib().oracle_scene_damping(self._h, f64(u), d):
            raise ArithmeticError("damping assembly failed")
        return d

    def jacobian(self, K, dt):
        J = np.zeros(self.nnz)
        lib().oracle_scene_jacobian(self._h, f64(K), dt, J)
        return J

    def cg(self, J, b, tol, max_iter=500):
        x = np.zeros(self.ndof)
        it = C.c_int64()
        st = lib().oracle_scene_cg(self._h, f64(J), f64(b), x, tol, max_iter, C.byref(it))
        return st, x, it.value

    def eval_f(self, u, v):
        f = np.zeros(self.ndof)
        if lib().oracle_scene_eval_f(self._h, f64(u), f64(v), f):
            raise ArithmeticError("eval_f failed")
        return f

    def step(self, u, v, t, dt):
        u, v = f64(u).copy(), f64(v).copy()
        L = lib()
        st = L.oracle_scene_step(self._h, u, v, t, dt)
        ncg = L.oracle_scene_last_num_cg(self._h)
        its = np.zeros(max(ncg, 1), dtype=np.int64)
        sts = np.zeros(max(ncg, 1), dtype=np.int32)
        L.oracle_scene_last_cg(self._h, its, sts)
        stats = dict(status=st, newton_iters=L.oracle_scene_last_newton_iters(self._h),
                     cg_iters=its[:ncg].tolist(), cg_status=sts[:ncg].tolist(),
                     substeps=L.oracle_scene_last_substeps(self._h), residual=L.oracle_scene_last_residual(self._h),
                     ls_backtracks=L.oracle_scene_last_ls_backtracks(self._h))
        return u, v, stats


# ---- embedded quadrature construction (embed_oracle.cpp) --------------------
class Embedding:
    """embed_mesh_3d + embed_quadrature_3d restated on the CPU
    (fenris/src/embedding/embedding3d.rs:57-289).  Background cells: Hex8 or
    Hex27 connectivity (the first 8 nodes are the corners); embedded mesh:
    Tet4."""

    def __init__(self, bg_vertices, bg_connectivity, emb_vertices, emb_tets, lower=1e-4, upper=0.999):
        L = lib()
        self._bgv = f64(bg_vertices)
        self._conn = i64(bg_connectivity)
        self._ev = f64(emb_vertices)
        self._et = i64(emb_tets)
        nbc, npc = self._conn.shape
        h = L.oracle_embed_create(self._bgv, self._bgv.shape[0], self._conn, nbc, npc, self._ev,
                                  self._ev.shape[0], self._et, self._et.shape[0], lower, upper)
        if not h:
            raise RuntimeError(L.oracle_embed_last_error().decode())
        self._h = h
        self.num_cells = nbc
        cls = np.zeros(nbc, dtype=np.int32)
        vol = np.zeros(nbc)
        L.oracle_embed_cells(h, cls, vol.ctypes.data)
        self.cell_class = cls
        self.cut_volume = vol
        self.exterior_cells = np.nonzero(cls == 0)[0]
        self.interior_cells = np.nonzero(cls == 1)[0]
        self.interface_cells = np.nonzero(cls == 2)[0]

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_embed_destroy(self._h)
            self._h = None

    def interface_quadratures(self, tet_weights, tet_points, stabilization=None):
        """(offsets, weights, points) of the interface cells' rules, in
        interface-cell order; stabilization = (factor, weights, points)."""
        L = lib()
        tw, tp = f64(tet_weights), f64(tet_points)
        if stabilization is None:
            fac, sw, sp, ns = 0.0, None, None, 0
        else:
            fac = float(stabilization[0])
            sw, sp = f64(stabilization[1]), f64(stabilization[2])
            ns = sw.shape[0]
        total = L.oracle_embed_quadrature(self._h, tw, tp, tw.shape[0], fac,
                                          sw.ctypes.data if ns else None, sp.ctypes.data if ns else None, ns)
        if total < 0:
            raise RuntimeError(L.oracle_embed_last_error().decode())
        off = np.zeros(len(self.interface_cells) + 1, dtype=np.int64)
        w = np.zeros(total)
        p = np.zeros((total, 3))
        L.oracle_embed_copy_quadrature(self._h, off, w, p)
        return off, w, p


def simplify_quadratures(offsets, weights, points, strength):
    """Moment-preserving reduction of every rule (Caratheodory elimination
    standing in for the reference's LP basic feasible point)."""
    off, w, p = i64(offsets), f64(weights), f64(points)
    oo = np.zeros_like(off)
    ow = np.zeros_like(w)
    op = np.zeros_like(p)
    lib().oracle_quadrature_simplify(len(off) - 1, off, w, p, int(strength), oo, ow, op)
    n = int(oo[-1])
    return oo, ow[:n].copy(), op[:n].copy()


def moment_matrix(points, strength):
    p = f64(points)
    r = lib().oracle_moment_matrix(p, p.shape[0], int(strength), None)
    P = np.zeros((r, p.shape[0]))
    lib().oracle_moment_matrix(p, p.shape[0], int(strength), P.ctypes.data)
    return P
