"""Preconditioners, conjugate gradient and the Newton-CG backward Euler
integrator, mirroring:

  SystemPreconditioner, DiagonalPreconditioner, SchwarzPreconditioner
      simulation_toolbox/src/fem/newton_cg.rs:297-411,534-593
  SchwarzPreconditionerComponent::from_embedded_model
      simulation_toolbox/src/fem/schwarz_precond.rs:65-127
  ConjugateGradient, RelativeResidualCriterion, SolveError(Kind), CgOutput
      fenris/src/cg.rs:62-124,195-482
  NewtonCgIntegrator3d
      simulation_toolbox/src/fem/newton_cg.rs:43-295
"""
import ctypes as C
import enum

import numpy as np

from . import _capi
from ._capi import HoefemError, check, host_f64, host_i64, lib, ptr
from .model import _same_space


class DiagonalPreconditioner:
    """z = r / diag(A); update() fails with ZERO_DIAGONAL like the reference."""

    def __init__(self, model):
        self.model = model
        h = C.c_void_p()
        check(lib().hoefem_precond_create_diagonal(model._h, C.byref(h)))
        self._h = h
        self._lib = lib()  # kept for __del__ at interpreter exit

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and getattr(self, "_lib", None) is not None:
            self._lib.hoefem_precond_destroy(h)
            self._h = None

    def update(self, system_values):
        check(lib().hoefem_precond_update(self._h, ptr(system_values)[0], _same_space(system_values)))

    def apply(self, r, z=None):
        if z is None:
            z = np.zeros_like(r) if not _capi.is_device_array(r) else r.new_zeros(r.shape)
        check(lib().hoefem_precond_apply(self._h, ptr(r)[0], ptr(z)[0], _same_space(r, z)))
        return z

    def values(self):
        nnz = C.c_int64()
        check(lib().hoefem_precond_nnz(self._h, C.byref(nnz)))
        v = np.zeros(nnz.value)
        check(lib().hoefem_precond_values(self._h, v.ctypes.data))
        return v


class SchwarzPreconditioner(DiagonalPreconditioner):
    """Element-wise additive Schwarz on `subdomains` (node lists), scalar
    Jacobi on `untreated_nodes` (build_schwarz_preconditioner_into)."""

    def __init__(self, model, subdomains, untreated_nodes):
        self.model = model
        subs = [np.asarray(s, dtype=np.int64) for s in subdomains]
        off = np.zeros(len(subs) + 1, dtype=np.int64)
        for i, s in enumerate(subs):
            off[i + 1] = off[i] + s.size
        flat = np.concatenate(subs) if subs else np.zeros(0, dtype=np.int64)
        un = host_i64(untreated_nodes)
        h = C.c_void_p()
        check(lib().hoefem_precond_create_schwarz(model._h, off.ctypes.data, flat.ctypes.data if flat.size else None,
                                                  len(subs), un.ctypes.data if un.size else None, un.size,
                                                  C.byref(h)))
        self._h = h
        self._lib = lib()  # kept for __del__ at interpreter exit
        self.num_subdomains = len(subs)

    def set_spmv_variant(self, variant):
        """8 / 16 / 32 lanes per node, +100 for the column-streaming traversal."""
        check(lib().hoefem_precond_set_spmv_variant(self._h, int(variant)))

    def set_block_apply(self, on):
        """CG applies the subdomain blocks as dense products (True, default) or
        the assembled CSR matrix (False); both are P r up to rounding."""
        check(lib().hoefem_precond_set_block_apply(self._h, 1 if on else 0))

    def spmv_variants(self):
        """(FP64-value variant, FP32-value variant) in use."""
        a, b = C.c_int32(), C.c_int32()
        check(lib().hoefem_precond_get_spmv_variants(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def pattern(self):
        nnz = C.c_int64()
        check(lib().hoefem_precond_nnz(self._h, C.byref(nnz)))
        ro = np.zeros(self.model.ndof() + 1, dtype=np.int64)
        ci = np.zeros(max(nnz.value, 1), dtype=np.int64)
        check(lib().hoefem_precond_pattern(self._h, ro.ctypes.data, ci.ctypes.data))
        return ro, ci[: nnz.value]


class SchwarzPreconditionerComponent:
    """Subdomain selection of the reference: interface elements whose embedded
    volume fraction is <= threshold become subdomains, every node outside them
    is untreated (schwarz_precond.rs:65-127)."""

    def __init__(self, subdomains, untreated_nodes):
        self.schwarz_connectivity = subdomains
        self.untreated_nodes = untreated_nodes

    @staticmethod
    def from_embedded_model(model, volume_fractions, volume_fraction_threshold):
        conn = model.interface_connectivity
        sel = [conn[i] for i in range(conn.shape[0]) if volume_fractions[i] <= volume_fraction_threshold]
        is_iface = np.zeros(model.num_vertices, dtype=bool)
        for s in sel:
            is_iface[s] = True
        untreated = np.nonzero(~is_iface)[0].astype(np.int64)
        return SchwarzPreconditionerComponent(sel, untreated)

    def build(self, model):
        return SchwarzPreconditioner(model, self.schwarz_connectivity, self.untreated_nodes)


class RelativeResidualCriterion:
    """||r|| <= tol ||b|| on the CG recurrence residual (cg.rs:77-124)."""

    def __init__(self, tol=1e-8):
        self.tol = float(tol)


class SolveErrorKind(enum.Enum):
    IndefiniteOperator = _capi.STATUS[10]
    IndefinitePreconditioner = _capi.STATUS[11]
    MaxIterationsReached = _capi.STATUS[12]


class CgOutput:
    def __init__(self, num_iterations):
        self.num_iterations = num_iterations


class SolveError(Exception):
    def __init__(self, kind, output):
        super().__init__("CG solve failed after %d iterations: %s" % (output.num_iterations, kind.name))
        self.kind = kind
        self.output = output


_CG_KIND = {10: SolveErrorKind.IndefiniteOperator, 11: SolveErrorKind.IndefinitePreconditioner,
            12: SolveErrorKind.MaxIterationsReached}


class ConjugateGradient:
    """Builder as in cg.rs:195-275: with_operator / with_preconditioner /
    with_stopping_criterion / with_max_iter, then solve_with_guess(b, x)."""

    def __init__(self, model):
        self.model = model
        self.values = None
        self.preconditioner = None
        self.criterion = RelativeResidualCriterion()
        self.max_iter = -1

    def with_operator(self, values):
        self.values = values
        return self

    def with_preconditioner(self, p):
        self.preconditioner = p
        return self

    def with_stopping_criterion(self, c):
        self.criterion = c
        return self

    def with_max_iter(self, n):
        self.max_iter = int(n)
        return self

    def solve_with_guess_mixed(self, b, x, delta=0.1):
        """PCG with FP32 operator / preconditioner values and FP64 vectors;
        the residual is replaced by the true FP64 residual whenever it has
        dropped by `delta` (reliable updates) and before stopping."""
        it = C.c_int64()
        mem = _same_space(self.values, b, x)
        st = lib().hoefem_cg_solve_mixed(self.model._h, ptr(self.values)[0],
                                         self.preconditioner._h if self.preconditioner is not None else None,
                                         ptr(b)[0], ptr(x)[0], self.criterion.tol, self.max_iter, float(delta),
                                         C.byref(it), mem)
        if st in _CG_KIND:
            raise SolveError(_CG_KIND[st], CgOutput(it.value))
        check(st)
        return CgOutput(it.value)

    def solve_with_guess(self, b, x):
        it = C.c_int64()
        mem = _same_space(self.values, b, x)
        st = lib().hoefem_cg_solve(self.model._h, ptr(self.values)[0],
                                   self.preconditioner._h if self.preconditioner is not None else None, ptr(b)[0],
                                   ptr(x)[0], self.criterion.tol, self.max_iter, C.byref(it), mem)
        if st in _CG_KIND:
            raise SolveError(_CG_KIND[st], CgOutput(it.value))
        check(st)
        return CgOutput(it.value)


class NewtonCgIntegrator3d:
    """One backward-Euler step per call, solved by Newton with backtracking line
    search and preconditioned CG (homogeneous Dirichlet nodes, scalar gravity
    on z, no damping).  `preconditioner` is a SchwarzPreconditioner of the same
    model or None (diagonal, the reference's fallback)."""

    def __init__(self, model, material, density, dirichlet_nodes=(), gravity=-9.81, gravity_enabled=True,
                 preconditioner=None):
        self.model = model
        self.material = material
        self.preconditioner = preconditioner
        bc = host_i64(dirichlet_nodes)
        self._bc = bc
        h = C.c_void_p()
        check(lib().hoefem_integrator_create(model._h, C.byref(material.descriptor()), float(density),
                                             bc.ctypes.data if bc.size else None, bc.size,
                                             1 if gravity_enabled else 0, float(gravity),
                                             preconditioner._h if preconditioner is not None else None, C.byref(h)))
        self._h = h
        self._lib = lib()  # kept for __del__ at interpreter exit

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and getattr(self, "_lib", None) is not None:
            self._lib.hoefem_integrator_destroy(h)
            self._h = None

    def set_tolerances(self, cg_tol=1e-5, cg_max_iter=500, newton_max_iter=100):
        check(lib().hoefem_integrator_set_tolerances(self._h, cg_tol, cg_max_iter, newton_max_iter))

    def set_damping(self, mass=None, stiffness=None):
        """Rayleigh damping D = mass M + stiffness K_proj(u) per (sub)step;
        None = no such term (the reference's Option::None)."""
        check(lib().hoefem_integrator_set_damping(self._h, 0 if mass is None else 1, 0.0 if mass is None else mass,
                                                  0 if stiffness is None else 1,
                                                  0.0 if stiffness is None else stiffness))

    def set_learned(self, learned, mode=1):
        """mode 1: guarded learned warm start; 2: collect (b, x*) training pairs
        from this integrator's plain FP64 CG solves; 3: as 2 plus the CG
        iterates (r_k, x* - x_k); 4: two-level preconditioner (the network's
        coarse correction beside Schwarz in every CG iteration, flexible CG);
        0 / learned=None: off."""
        self._learned = learned
        check(lib().hoefem_integrator_set_learned(self._h, learned._h if learned is not None else None,
                                                  int(mode) if learned is not None else 0))

    def set_precision(self, mixed, delta=1e-3):
        """mixed=True: FP32 element stiffness, FP32 operator / Schwarz apply in
        a reliable-update PCG with FP64 vectors, the recurrence residual
        replaced by the FP64 one after every drop by `delta` (see
        hoefem_integrator_set_precision)."""
        check(lib().hoefem_integrator_set_precision(self._h, 1 if mixed else 0, float(delta)))

    def set_cg_engine(self, engine="auto", schwarz_fp16=False, phase_profile=False):
        """CG engine of the Jacobian solves: "auto" (the faster engine, timed
        on the first solves), "chunked" (CUDA graphs of kernel chunks) or
        "streamed" (persistent streamed CG; error if it cannot run);
        schwarz_fp16 keeps the Schwarz blocks of the mixed form in scaled FP16;
        phase_profile records per-phase times (hoefem_integrator_set_cg_engine)."""
        check(lib().hoefem_integrator_set_cg_engine(self._h, _capi.CG_ENGINE[engine],
                                                         (1 if schwarz_fp16 else 0) | (2 if phase_profile else 0)))

    def set_cg_l2_keep(self, nbytes=-1):
        """L2 residency budget (bytes) of the streamed CG; -1: the default (0)."""
        check(lib().hoefem_integrator_set_cg_l2_keep(self._h, int(nbytes)))

    def cg_engine_stats(self):
        """Streamed-CG counters of the last step: launches, iterations, device
        ms and the bytes one iteration streams."""
        s = _capi.CgEngineStats()
        check(lib().hoefem_integrator_cg_engine_stats(self._h, C.byref(s)))
        out = {f: getattr(s, f) for f, _ in s._fields_}
        out["phase_us"] = list(out["phase_us"])
        for k in ("auto_us_per_iteration", "phase_us_max", "busy_us"):
            out[k] = list(out[k])
        return out

    def step(self, u, v, t, dt):
        """Advances (u, v) in place by dt; returns the step statistics."""
        mem = _same_space(u, v)
        check(lib().hoefem_integrator_step(self._h, ptr(u)[0], ptr(v)[0], float(t), float(dt), mem))
        return self.stats()

    def stats(self):
        s = _capi.StepStats()
        check(lib().hoefem_integrator_stats(self._h, C.byref(s)))
        return s.as_dict()

    def mass(self):
        v = np.zeros(self.model.nnz)
        check(lib().hoefem_integrator_mass(self._h, v.ctypes.data))
        return v

    def eval_f(self, u, v, f=None):
        if f is None:
            f = np.zeros(self.model.ndof()) if not _capi.is_device_array(u) else u.new_zeros(self.model.ndof())
        check(lib().hoefem_integrator_eval_f(self._h, ptr(u)[0], ptr(v)[0], ptr(f)[0], _same_space(u, v, f)))
        return f


class BatchedNewtonCgIntegrator3d:
    """Many independent scenes advanced together: each scene takes the path of
    NewtonCgIntegrator3d.step with the diagonal preconditioner (its own
    Dirichlet scale, tolerances, line search and substepping), while all
    scenes share every kernel launch (see hoefem_batch_create).  `models`:
    NodalModel3d / EmbeddedModel3d objects; `materials`: one per scene, all of
    one kind; `dirichlet_nodes`: one node list per scene.  Not in the
    reference, which steps one model at a time."""

    def __init__(self, models, materials, density, dirichlet_nodes=None, gravity=-9.81, gravity_enabled=True):
        ns = len(models)
        if len(materials) != ns:
            raise ValueError("one material per scene")
        self.models = list(models)
        handles = (C.c_void_p * ns)(*[m._h.value if hasattr(m._h, "value") else m._h for m in self.models])
        descs = (_capi.Material * ns)(*[mat.descriptor() for mat in materials])
        bc_lists = dirichlet_nodes if dirichlet_nodes is not None else [()] * ns
        if len(bc_lists) != ns:
            raise ValueError("one Dirichlet node list per scene")
        off = np.zeros(ns + 1, dtype=np.int64)
        flat = []
        for k, b in enumerate(bc_lists):
            b = host_i64(b)
            off[k + 1] = off[k] + b.size
            flat.append(b)
        flat = np.concatenate(flat) if off[-1] else np.zeros(1, dtype=np.int64)
        self._bc = (off, flat)
        h = C.c_void_p()
        check(lib().hoefem_batch_create(handles, ns, descs, float(density), off.ctypes.data, flat.ctypes.data,
                                        1 if gravity_enabled else 0, float(gravity), C.byref(h)))
        self._h = h
        self._lib = lib()  # kept for __del__ at interpreter exit
        self.num_scenes = ns
        ndof = C.c_int64()
        nnz = C.c_int64()
        self.dof_offsets = np.zeros(ns + 1, dtype=np.int64)
        check(lib().hoefem_batch_sizes(h, None, C.byref(ndof), C.byref(nnz), self.dof_offsets.ctypes.data))
        self.ndof = ndof.value
        self.nnz = nnz.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and getattr(self, "_lib", None) is not None:
            self._lib.hoefem_batch_destroy(h)
            self._h = None

    def set_stream(self, stream):
        check(lib().hoefem_batch_set_stream(self._h, C.c_void_p(int(stream)) if stream else None))

    def set_tolerances(self, cg_tol=1e-5, cg_max_iter=500, newton_max_iter=100):
        check(lib().hoefem_batch_set_tolerances(self._h, cg_tol, cg_max_iter, newton_max_iter))

    def set_cg_engine(self, engine="auto", ctas_per_sm=0):
        """'chunked': CUDA graphs of per-phase kernels; 'streamed': one
        persistent launch per solve (ctas_per_sm CTAs per multiprocessor, 0 =
        as many as fit); 'auto': the autotuner times both on the first solve
        (see hoefem_batch_set_cg_engine).  Results do not depend on it."""
        check(lib().hoefem_batch_set_cg_engine(self._h, _capi.CG_ENGINE[engine], int(ctas_per_sm)))

    def cg_choice(self):
        """(engine name, CTAs per multiprocessor, autotuner ms per candidate)."""
        e, c, n = C.c_int32(), C.c_int32(), C.c_int32(16)
        t = (C.c_float * 16)()
        check(lib().hoefem_batch_cg_choice(self._h, C.byref(e), C.byref(c), C.cast(t, C.c_void_p), C.byref(n)))
        names = {v: k for k, v in _capi.CG_ENGINE.items()}
        return names[e.value], c.value, [t[k] for k in range(min(n.value, 16))]

    def split(self, x):
        """Per-scene views of a concatenated DOF vector."""
        o = self.dof_offsets
        return [x[o[k]:o[k + 1]] for k in range(self.num_scenes)]

    def step(self, u, v, t, dt, raise_on_failure=True):
        """Advances the concatenated (u, v) in place; returns one statistics
        dict per scene (with its 'status')."""
        mem = _same_space(u, v)
        st = lib().hoefem_batch_step(self._h, ptr(u)[0], ptr(v)[0], float(t), float(dt), mem)
        if st not in (0, 20, 21, 22) and st not in _CG_KIND:
            check(st)
        stats = self.stats()
        if raise_on_failure and st != 0:
            check(st)
        return stats

    def stats(self):
        out = []
        for k in range(self.num_scenes):
            s = _capi.StepStats()
            code = C.c_int32()
            check(lib().hoefem_batch_scene_stats(self._h, k, C.byref(s), C.byref(code)))
            d = s.as_dict()
            d["status"] = code.value
            out.append(d)
        return out
