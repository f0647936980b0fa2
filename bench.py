#!/usr/bin/env python
"""Newton-step benchmark of the embedded Hex27 hollow-cylinder scene.

Workload (one "step" = one backward-Euler Newton-CG time step from the same
initial state): unit-box Hex27 background grid n^3 = 24^3 (13,824 cells)
clipped to the hollow cylinder r in [0.3, 0.4] (4,608 kept cells: 1,536
interior with the 14-point rule, 3,072 cut cells with seeded Q ~ U{8..27}
points and Dirichlet weights summing to the volume fraction), StVK
E = 5e5 nu = 0.45 rho = 1000, gravity -9.81 on z, nodes with z <= 1e-9 fixed,
u0 = smooth sway (0.02 z^2, 0.01 z^2, 0) + N(0, (0.001 h)^2), v0 = 0, dt = 1e-3, additive-Schwarz-preconditioned CG
to 1e-6 relative residual (reference subdomain rule: cut cells with volume
fraction <= 0.5, Jacobi elsewhere), FP64.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl hoefem|reference]

Prints one JSON line (rank 0).  `value` is the device-timed Newton-step time
(max over ranks), `e2e` the same step through the public API with host
buffers (H2D / D2H inside the timed region).  `--impl reference` times the
reference path's CPU restatement (the oracle; the Rust reference cannot be
built here) on the host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Newton-step ms & CG iters at 1e-6 rel res: learned/FP32 vs plain FP64 on 1 GPU"
DT = 1e-3
# arithmetic of each variant (the line's `dtype` is the headline variant's)
DTYPES = {
    "plain": "f64",
    "mixed": "mixed: f32 element stiffness arithmetic, f32 operator and Schwarz values in CG, f64 vectors, dot "
             "products, residual replacement and CSR accumulation",
    "learned": "mixed (as the mixed variant) + bf16 MLP inference with f32 accumulation",
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="hoefem", choices=["hoefem", "reference"])
    ap.add_argument("--n", type=int, default=24, help="background cells per axis")
    ap.add_argument("--cg-tol", type=float, default=1e-6)
    ap.add_argument("--cg-max-iter", type=int, default=500)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--roofline-reps", type=int, default=20)
    ap.add_argument("--delta", type=float, default=1e-3,
                    help="mixed variant: reliable-update threshold (residual drop between FP64 replacements)")
    ap.add_argument("--cg-engine", default="auto", choices=["auto", "chunked", "streamed"],
                    help="CG engine of the Jacobian solves (hoefem_integrator_set_cg_engine)")
    ap.add_argument("--schwarz-fp16", action="store_true", help="mixed variants: FP16 Schwarz blocks in the streamed CG")
    ap.add_argument("--cg-phase-profile", action="store_true",
                    help="streamed CG: per-phase times (mean and largest over CTAs) in each variant's cg_engine")
    ap.add_argument("--variants", default="plain,mixed,learned", help="comma list: plain, mixed, learned")
    ap.add_argument("--train-states", type=int, default=16, help="learned: training initial states (seeded)")
    ap.add_argument("--train-steps", type=int, default=2000, help="learned: Adam steps")
    ap.add_argument("--coarse-subdomains", type=int, default=256, help="learned: coarse subdomains")
    ap.add_argument("--workload", default="cylinder", choices=["cylinder", "batched", "tet10", "embed"],
                    help="cylinder: embedded Hex27 cylinder Newton step; batched: 64 independent scenes in one "
                         "batch; tet10: 201,600-element Tet10 box, plain vs mixed precision; embed: embedded "
                         "quadrature construction (classification, cut-cell rules, simplification)")
    ap.add_argument("--scenes", type=int, default=64, help="batched: number of scenes")
    ap.add_argument("--tet10-grid", default="40,40,21",
                    help="tet10: hex cells per axis (6 Tet10 each); the benchmark box is 40,40,21")
    ap.add_argument("--min-elements", type=float, default=1e3, help="batched: smallest scene (elements)")
    ap.add_argument("--max-elements", type=float, default=5e4, help="batched: largest scene (elements)")
    ap.add_argument("--no-sequential", action="store_true", help="batched: skip the one-scene-at-a-time comparison")
    ap.add_argument("--batch-cg-engine", default="auto", choices=["auto", "chunked", "streamed"],
                    help="batched: CG engine (graphs, persistent launch, or the autotuner's choice)")
    ap.add_argument("--roofline-only", action="store_true",
                    help="cylinder: autotune the SpMV, then only the roofline launches (for a DRAM-traffic capture)")
    return ap.parse_args()


def sway_state(H, e, ndof, amp_x, amp_y, noise_seed):
    """u = (amp_x z^2, amp_y z^2, 0) + N(0, (0.001 h)^2), v = 0."""
    X = e.vertices
    u0 = np.zeros_like(X)
    u0[:, 0] = amp_x * X[:, 2] ** 2
    u0[:, 1] = amp_y * X[:, 2] ** 2
    return u0.reshape(-1) + H.scenes.random_normal(noise_seed, ndof, 0.001 * e.cell_size), np.zeros(ndof)


def workload(H, n, seed):
    e = H.scenes.embedded_cylinder(n, 0.3, 0.4, 8, 27, seed)
    b0, b1 = e.blocks
    model = H.EmbeddedModel3d(e.vertices, b0.connectivity, b1.connectivity, (b0.weights, b0.points),
                              (b1.offsets, b1.weights, b1.points))
    mat = H.StVKMaterial(H.YoungPoisson(5e5, 0.45))
    bc = e.nodes_below(2, 1e-9)
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(model, e.volume_fractions, 0.5)
    # initial state: smooth sway u = (0.02 z^2, 0.01 z^2, 0) plus seeded noise N(0, (0.001 h)^2), at rest
    u0, v0 = sway_state(H, e, model.ndof(), 0.02, 0.01, 1000 + seed)
    return e, model, mat, bc, comp, u0, v0


def train_learned(H, e, model, integ, bc, args, dev):
    """Learned coarse correction trained on (b, x*) pairs of plain FP64
    Schwarz-CG Jacobian solves from seeded training states (sway amplitudes
    and noise seeds disjoint from the timed state)."""
    import torch

    L = H.LearnedCoarseCorrection(model, bc, num_subdomains=args.coarse_subdomains, seed=7)
    integ.set_precision(False, args.delta)
    integ.set_learned(L, 2)
    rng = np.random.default_rng(12345)
    t0 = time.perf_counter()
    for k in range(args.train_states):
        ax, ay = rng.uniform(-0.03, 0.03, size=2)
        u, v = sway_state(H, e, model.ndof(), ax, ay, 50000 + k)
        ud, vd = torch.from_numpy(u).to(dev), torch.from_numpy(v).to(dev)
        integ.step(ud, vd, 0.0, DT)
    t_collect = time.perf_counter() - t0
    t0 = time.perf_counter()
    hist = L.train(args.train_steps, batch=512, lr=1e-3, seed=0)
    t_train = time.perf_counter() - t0
    integ.set_learned(None)
    info = {"rows": int(L.num_pairs()), "coarse_subdomains": args.coarse_subdomains,
            "train_states": args.train_states, "adam_steps": args.train_steps,
            "loss_first10": float(np.mean(hist[:10])), "loss_last50": float(np.mean(hist[-50:])),
            "collect_s": t_collect, "train_s": t_train}
    return L, info


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        rows = [r.split(", ") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows if len(r) >= 9 for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(x, world, device=None):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def workload_name(n, cg_tol):
    """The workload string both arms report (identical by construction)."""
    return ("embedded Hex27 hollow cylinder %d^3 (r 0.3-0.4), StVK E=5e5 nu=0.45, one backward-Euler Newton step "
            "dt=1e-3, Schwarz-CG to %g" % (n, cg_tol))


def oracle_step_sample(n, seed, cg_tol, threads):
    """The reference path's CPU restatement (the oracle) on the benchmark scene,
    built entirely on the oracle side (oracle/scenes.py, checked bit for bit
    against the product's scene): returns (ref, u0, v0) ready for ref.step."""
    from oracle import oracle as O
    from oracle import scenes as OS

    if threads:
        O.set_num_threads(threads)
    sc = OS.embedded_cylinder(n, 0.3, 0.4, 8, 27, seed)
    u0, v0 = OS.sway_state(sc, 0.02, 0.01, 1000 + seed)
    ref = OS.cylinder_reference_scene(sc, cg_tol=cg_tol)
    return ref, u0, v0


def timed_oracle_steps(ref, u0, v0, warmup, steps):
    """Whole backward-Euler steps of the oracle from the same initial state:
    per-step wall ms, CG iterations and Newton iterations of the last step."""
    for _ in range(warmup):
        ref.step(u0, v0, 0.0, DT)
    times, st = [], None
    for _ in range(steps):
        t0 = time.perf_counter()
        _, _, st = ref.step(u0, v0, 0.0, DT)
        times.append((time.perf_counter() - t0) * 1e3)
    return times, st


def run_reference(args):
    """`--impl reference`: the reference path's CPU restatement (the Rust
    reference cannot be built here) on all host cores, whole Newton steps, no
    product code on the path."""
    world, rank, local = dist_setup(args.gpus)
    if rank != 0:
        return
    from oracle import oracle as O

    ref, u0, v0 = oracle_step_sample(args.n, args.seed, args.cg_tol, os.cpu_count() or 1)
    # a whole oracle step takes tens of seconds on the host cores: at most one
    # warm-up and three timed steps keep the run within a few minutes
    warmup, steps = min(args.warmup, 1), max(1, min(args.steps, 3))
    times, st = timed_oracle_steps(ref, u0, v0, warmup, steps)
    ms = float(np.mean(times))
    line = {
        "metric": METRIC, "value": ms, "unit": "ms", "impl": "reference", "n_gpus": args.gpus, "steps": steps,
        "warmup": warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded scene, built by the oracle)",
        "config": {"workload": workload_name(args.n, args.cg_tol), "ndof": int(u0.size), "nnz": int(ref.nnz)},
        "cg_iterations": int(sum(st["cg_iters"])), "newton_iterations": int(st["newton_iters"]),
        "cpu_baseline": {"value": ms, "unit": "ms", "cores": O.num_threads(), "kind": "port",
                         "sample": "whole backward-Euler Newton steps of the oracle (C++ FP64 restatement of the "
                                   "reference path, OpenMP over the host cores), %d timed after %d warm-up"
                                   % (steps, warmup)},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "step_ms": times,
    }
    print(json.dumps(line), flush=True)


def run_hoefem(args):
    import torch

    world, rank, local = dist_setup(args.gpus)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import higher_order_embedded_fem_b200 as H

    H._capi.check(H._capi.lib().hoefem_set_device(local))
    # replicas: each rank integrates its own scene (different seed)
    e, model, mat, bc, comp, u0, v0 = workload(H, args.n, args.seed + rank)
    stream = torch.cuda.current_stream(dev)
    model.set_stream(stream.cuda_stream)
    P = comp.build(model)
    integ = H.NewtonCgIntegrator3d(model, mat, 1000.0, bc, preconditioner=P)
    integ.set_tolerances(args.cg_tol, args.cg_max_iter, 100)
    integ.set_cg_engine(args.cg_engine, args.schwarz_fp16, phase_profile=args.cg_phase_profile)

    u0d = torch.from_numpy(u0).to(dev)
    v0d = torch.from_numpy(v0).to(dev)
    ud, vd = u0d.clone(), v0d.clone()

    def step():
        ud.copy_(u0d)
        vd.copy_(v0d)
        return integ.step(ud, vd, 0.0, DT)

    variants = {}
    learned, learned_info = None, None
    for vname in [v.strip() for v in args.variants.split(",") if v.strip()]:
        if vname == "learned" and learned is None:
            learned, learned_info = train_learned(H, e, model, integ, bc, args, dev)
        integ.set_precision(vname in ("mixed", "learned"), args.delta)
        integ.set_learned(learned if vname == "learned" else None, 1)
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        clocks = Clocks(local)
        clocks.start()
        n0 = H._capi.launch_count()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        per = []
        for _ in range(args.steps):
            per.append(step())
        ev1.record(stream)
        torch.cuda.synchronize()
        launches = H._capi.launch_count() - n0
        if world > 1:
            torch.distributed.barrier()
        ck = clocks.stop()
        ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, world, dev)
        s_ = per[-1]
        eng = integ.cg_engine_stats()
        variants[vname] = {
            "ms_per_step": ms, "cg_iterations": int(s_["total_cg_iterations"]),
            "newton_iterations": int(s_["newton_iterations"]), "residual_norm": s_["residual_norm"],
            "phase_ms": {"forces": s_["ms_assemble_forces"], "stiffness": s_["ms_assemble_stiffness"],
                         "precond_update": s_["ms_precond_update"], "cg": s_["ms_cg"], "total": s_["ms_total"]},
            "gpu_launches": int(launches), "clocks": ck, "u": ud.cpu().numpy(),
            "cg_engine": eng,
        }
        if vname == "learned":
            variants[vname].update({"learned_accepted": int(s_["learned_accepted"]),
                                    "learned_rejected": int(s_["learned_rejected"]),
                                    "learned_residual_ratio": s_["learned_residual_ratio"],
                                    "ms_learned": s_["ms_learned"], "training": learned_info})
    op64, op32 = model.spmv_variants()
    pr64, pr32 = P.spmv_variants()
    spmv_variants = {"operator_fp64": op64, "operator_fp32": op32, "schwarz_fp64": pr64, "schwarz_fp32": pr32}
    head = "learned" if "learned" in variants else ("mixed" if "mixed" in variants else list(variants)[0])
    ms = variants[head]["ms_per_step"]
    launches = variants[head]["gpu_launches"]
    ck = variants[head]["clocks"]
    integ.set_precision(head in ("mixed", "learned"), args.delta)
    integ.set_learned(learned if head == "learned" else None, 1)
    for vn in ("mixed", "learned"):
        if vn in variants and "plain" in variants:
            up, um = variants["plain"]["u"], variants[vn]["u"]
            variants[vn]["rel_diff_u_vs_plain"] = float(np.abs(um - up).max() / np.abs(up).max())
    for vn_, v in variants.items():
        v.pop("u")
        v["cg_roofline"] = cg_roofline(v, vn_, args.schwarz_fp16)

    # end to end through the public API with pinned host buffers
    uh = torch.empty(model.ndof(), dtype=torch.float64, pin_memory=True).numpy()
    vh = torch.empty(model.ndof(), dtype=torch.float64, pin_memory=True).numpy()
    model.set_stream(None)
    uh[:] = u0
    vh[:] = v0
    integ.step(uh, vh, 0.0, DT)  # warm the host path
    t0 = time.perf_counter()
    for _ in range(args.steps):
        uh[:] = u0
        vh[:] = v0
        integ.step(uh, vh, 0.0, DT)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    e2e_ms = max_over_ranks(e2e_ms, world, dev)
    model.set_stream(stream.cuda_stream)

    # roofline of the dominant kernel: the persistent streamed CG of the headline
    # variant (its CUDA-event device time over the step's iterations)
    roof = cg_roofline(variants[head], head, args.schwarz_fp16)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O

        ref, ru0, rv0 = oracle_step_sample(args.n, args.seed, args.cg_tol, os.cpu_count())
        times, rst = timed_oracle_steps(ref, ru0, rv0, 0, 1)
        cpu = {"value": times[0], "unit": "ms", "cores": O.num_threads(), "kind": "port",
               "sample": "one whole backward-Euler Newton step of the oracle on the same scene (OpenMP over the "
                         "host cores)", "cg_iterations": int(sum(rst["cg_iters"])),
               "newton_iterations": int(rst["newton_iters"])}

    if rank == 0:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
            os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
        line = {
            "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPES[head], "data": "synthetic (seeded scene, replicas per rank)",
            "variant": {"mixed": "mixed_fp32", "plain": "plain_fp64", "learned": "learned_mixed"}[head],
            "variants": variants,
            "config": {"workload": workload_name(args.n, args.cg_tol),
                       "ndof": model.ndof(), "nnz": model.nnz, "elements": model.num_elements,
                       "schwarz_subdomains": len(comp.schwarz_connectivity),
                       "l2": "inputs larger than L2 (CSR values %d MB)" % (model.nnz * 8 // 2 ** 20),
                       "parallelism": "replicas" if world > 1 else "single"},
            "cg_iterations": variants[head]["cg_iterations"], "newton_iterations": variants[head]["newton_iterations"],
            "speedup_vs_plain_fp64": (variants["plain"]["ms_per_step"] / ms) if "plain" in variants else None,
            "roofline": roof,
            "spmv_variants": spmv_variants,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": 2 * 8 * model.ndof(),
                    "d2h_bytes_per_step": 2 * 8 * model.ndof()},
            "gpu_launches": int(launches),
            "clocks": ck,
            "peaks": {"hbm_gbs": peaks.get("hbm_gbs"), "source": "MEASURED_PEAKS.json" if peaks else "fallback"},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def cg_roofline(var, head, fp16=False):
    """Streamed CG of one variant: algorithmic bytes per iteration = operator
    tiles (values + neighbour lists + tile headers) + Schwarz block chunks, the
    data an iteration must read from HBM (vectors, 1 MB each, stay in L2);
    achieved = bytes x iterations / summed device time of the persistent
    launches (CUDA events on the launch stream)."""
    eng = var.get("cg_engine") or {}
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = json.load(open(peaks_path))["hbm_gbs"] if os.path.exists(peaks_path) else 6650.0
    if not eng.get("launches") or not eng.get("iterations") or not eng.get("device_ms"):
        return None
    per_it = eng["operator_bytes"] + eng["schwarz_bytes"]
    ms_it = eng["device_ms"] / eng["iterations"]
    gbs = per_it / (ms_it * 1e-3) / 1e9
    kern = {"plain": "k_cg_stream<double,double,2>", "mixed": "k_cg_stream<float,float,2>",
            "learned": "k_cg_stream<float,float,2>"}[head]
    if fp16 and head != "plain":
        kern = kern.replace("float,float", "float,__half")
    # DRAM bytes per iteration of the same kernel on this workload, from an ncu
    # capture of all its launches in a bench run (dram__bytes_read.sum +
    # dram__bytes_write.sum summed over the launches / the iterations they ran)
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "k_cg_stream_traffic_embedded_cylinder_n24.json")
    if os.path.exists(tpath):
        t = json.load(open(tpath)).get("kernels", {}).get(kern)
        # the same stream up to item headers (segment cuts shift by a few bytes)
        if t and abs(t.get("bytes_per_iteration_algorithmic", 0) - per_it) <= 1e-3 * per_it:
            traffic = t["dram_bytes_per_iteration"]
    return {"kernel": kern + " (persistent streamed Schwarz-PCG)", "bound": "hbm", "achieved": gbs, "peak": peak,
            "unit": "GB/s", "frac": gbs / peak, "traffic": traffic, "traffic_unit": "DRAM bytes per CG iteration",
            "bytes_per_iteration": per_it,
            "us_per_iteration": ms_it * 1e3, "iterations": eng["iterations"], "launches": eng["launches"],
            "peak_source": "measured" if os.path.exists(peaks_path) else "fallback"}


def spmv_roofline(H, model, integ, mat, ud, stream, reps):
    """Node-row SpMV (the CG operator A p) timed alone with CUDA events on the
    model's stream; algorithmic bytes = values 8 B/nnz + adjacency 4 B per
    neighbour + base/offset 12 B per node + x read + y write (8 B per dof each)."""
    import torch

    K = torch.zeros(model.nnz, dtype=torch.float64, device=ud.device)
    model.assemble_stiffness_into_par(K, ud, mat)
    x = torch.randn(model.ndof(), dtype=torch.float64, device=ud.device)
    y = torch.zeros_like(x)
    for _ in range(3):
        model.spmv(y, K, x)
    # flush L2 between launches with a 256 MB write
    flush = torch.empty(32 * 2 ** 20, dtype=torch.float64, device=ud.device)
    tot = 0.0
    for _ in range(reps):
        flush.fill_(1.0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        model.spmv(y, K, x)
        b.record(stream)
        torch.cuda.synchronize()
        tot += a.elapsed_time(b)
    ms = tot / reps
    nv = model.num_vertices
    nbr = model.nnz // 9
    bytes_alg = model.nnz * 8 + nbr * 4 + nv * 12 + 2 * model.ndof() * 8
    gbs = bytes_alg / (ms * 1e-3) / 1e9
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = json.load(open(peaks_path))["hbm_gbs"] if os.path.exists(peaks_path) else 6650.0
    # DRAM bytes of one launch from an ncu capture of the same command (`--roofline-only`)
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(tpath):
        t = json.load(open(tpath))
        if t.get("nnz") == model.nnz:
            traffic = t.get("dram_bytes_per_launch")
    return {"kernel": "k_spmv (node-row SpMV, CG operator)", "bound": "hbm", "achieved": gbs, "peak": peak,
            "unit": "GB/s", "frac": gbs / peak, "traffic": traffic, "ms_per_launch": ms,
            "algorithmic_bytes": bytes_alg, "peak_source": "measured" if os.path.exists(peaks_path) else "fallback"}


def run_roofline_only(args):
    """The workload's model, the SpMV autotuner (6 variants x 4 launches), then
    3 warm-up and --roofline-reps timed roofline launches; prints the roofline."""
    import torch

    dev = torch.device("cuda", 0)
    import higher_order_embedded_fem_b200 as H

    e, model, mat, bc, comp, u0, v0 = workload(H, args.n, args.seed)
    stream = torch.cuda.current_stream(dev)
    model.set_stream(stream.cuda_stream)
    lanes = model.autotune()
    ud = torch.from_numpy(u0).to(dev)
    roof = spmv_roofline(H, model, None, mat, ud, stream, args.roofline_reps)
    roof["spmv_variant"] = lanes
    print(json.dumps({"roofline": roof, "nnz": model.nnz}), flush=True)


def batched_scenes(H, args):
    """Seeded scene list: element counts log-uniform in [min, max], Tet10 box
    grids (6 tets per cell) and Hex27 box grids alternating, SNH with E
    log-uniform in [1e5, 1e7] and nu uniform in [0.3, 0.48], bottom nodes
    clamped, u0 = small sway + N(0, (0.001 h)^2), v0 = 0."""
    rng = np.random.default_rng(args.seed)
    out = []
    for k in range(args.scenes):
        target = float(np.exp(rng.uniform(np.log(args.min_elements), np.log(args.max_elements))))
        tet = (k % 2 == 0)
        cells = max(1.0, target / 6.0 if tet else target)
        n = max(1, int(round(cells ** (1.0 / 3.0))))
        nz = max(1, int(round(cells / (n * n))))
        h = 1.0 / max(n, nz)
        young = float(np.exp(rng.uniform(np.log(1e5), np.log(1e7))))
        nu = float(rng.uniform(0.3, 0.48))
        if tet:
            s = H.scenes.tet10_box(h, n, n, nz, 1)
        else:
            s = H.scenes.hex27_box(h, n, n, nz, 1)
        b = s.blocks[0]
        m = H.NodalModel3d(s.vertices, b.connectivity, (b.weights, b.points), b.kind)
        mat = H.StableNeoHookeanMaterial(H.YoungPoisson(young, nu))
        bc = s.nodes_below(2, 1e-9)
        u0, v0 = sway_state(H, s, m.ndof(), 0.01 * rng.uniform(-1, 1), 0.01 * rng.uniform(-1, 1), 7000 + k)
        out.append({"scene": s, "model": m, "mat": mat, "bc": bc, "u0": u0, "v0": v0, "kind": "tet10" if tet else "hex27",
                    "elements": int(m.num_elements), "young": young, "nu": nu})
    return out


def run_batched(args):
    """Batched solves: all scenes advanced by one backward-Euler Newton-CG step
    (diagonal preconditioner) in one batch, against the same scenes stepped
    one at a time by NewtonCgIntegrator3d."""
    import torch

    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import higher_order_embedded_fem_b200 as H

    H._capi.check(H._capi.lib().hoefem_set_device(local))
    t0 = time.perf_counter()
    sc = batched_scenes(H, args)
    B = H.BatchedNewtonCgIntegrator3d([x["model"] for x in sc], [x["mat"] for x in sc], 1000.0,
                                      [x["bc"] for x in sc])
    setup_s = time.perf_counter() - t0
    B.set_tolerances(args.cg_tol, args.cg_max_iter, 100)
    B.set_cg_engine(args.batch_cg_engine)
    stream = torch.cuda.current_stream(dev)
    B.set_stream(stream.cuda_stream)
    u0 = torch.from_numpy(np.concatenate([x["u0"] for x in sc])).to(dev)
    v0 = torch.from_numpy(np.concatenate([x["v0"] for x in sc])).to(dev)
    ud, vd = u0.clone(), v0.clone()

    def step():
        ud.copy_(u0)
        vd.copy_(v0)
        return B.step(ud, vd, 0.0, DT)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    n0 = H._capi.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        stats = step()
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = H._capi.launch_count() - n0
    ck = clocks.stop()
    ms = ev0.elapsed_time(ev1) / args.steps
    # end to end with pinned host buffers
    uh = torch.empty(B.ndof, dtype=torch.float64, pin_memory=True).numpy()
    vh = torch.empty(B.ndof, dtype=torch.float64, pin_memory=True).numpy()
    B.set_stream(None)
    uh[:] = u0.cpu().numpy()
    vh[:] = v0.cpu().numpy()
    B.step(uh, vh, 0.0, DT)
    t1 = time.perf_counter()
    for _ in range(args.steps):
        uh[:] = u0.cpu().numpy()
        vh[:] = v0.cpu().numpy()
        B.step(uh, vh, 0.0, DT)
    e2e_ms = (time.perf_counter() - t1) * 1e3 / args.steps
    seq_ms = None
    if not args.no_sequential:
        # the same scenes one at a time (one integrator alive at a time): the
        # sum of the per-scene device times of one step each, after a warm-up
        B.set_stream(stream.cuda_stream)
        seq_ms = 0.0
        for x in sc:
            it = H.NewtonCgIntegrator3d(x["model"], x["mat"], 1000.0, x["bc"])
            it.set_tolerances(args.cg_tol, args.cg_max_iter, 100)
            # the CUDA-graph engine: the faster one for every scene size here
            # (all 64 one at a time: 2.1 s against 3.1 s streamed), and an
            # integrator that lives for two steps cannot amortise the
            # automatic choice's sampling of both engines
            it.set_cg_engine("chunked")
            x["model"].set_stream(stream.cuda_stream)
            a = torch.from_numpy(x["u0"]).to(dev)
            b = torch.from_numpy(x["v0"]).to(dev)
            it.step(a.clone(), b.clone(), 0.0, DT)
            ua, vb = a.clone(), b.clone()
            torch.cuda.synchronize()
            ev0.record(stream)
            it.step(ua, vb, 0.0, DT)
            ev1.record(stream)
            torch.cuda.synchronize()
            seq_ms += ev0.elapsed_time(ev1)
            del it
    newton = [s["newton_iterations"] for s in stats]
    cgit = [s["total_cg_iterations"] for s in stats]
    eng, per, tune_ms = B.cg_choice()
    line = {
        "metric": "batched Newton step ms (all scenes) on 1 GPU", "value": ms, "unit": "ms", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded scenes)",
        "config": {"workload": "%d scenes, elements log-uniform [%g, %g], Tet10/Hex27 boxes alternating, SNH E "
                               "log-uniform [1e5, 1e7], nu U[0.3, 0.48], one BE Newton step dt=1e-3, diagonal PCG "
                               "to %g" % (args.scenes, args.min_elements, args.max_elements, args.cg_tol),
                   "elements": int(sum(x["elements"] for x in sc)), "ndof": int(B.ndof), "nnz": int(B.nnz),
                   "l2": "inputs larger than L2 (CSR values %d MB)" % (B.nnz * 8 // 2 ** 20)},
        "sequential_ms": seq_ms, "speedup_vs_sequential": (seq_ms / ms) if seq_ms else None,
        "newton_iterations": {"min": int(min(newton)), "max": int(max(newton)), "sum": int(sum(newton))},
        "cg_iterations": {"min": int(min(cgit)), "max": int(max(cgit)), "sum": int(sum(cgit))},
        "statuses": sorted({int(s["status"]) for s in stats}),
        "cg_engine": {"requested": args.batch_cg_engine, "used": eng, "ctas_per_sm": per,
                      "autotuner_first_solve_ms": [round(t, 3) for t in tune_ms],
                      "candidates": "chunked graphs, then persistent at 1, 2, 4, ... CTAs/SM"},
        "setup_s": setup_s,
        "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": 16 * int(B.ndof),
                "d2h_bytes_per_step": 16 * int(B.ndof)},
        "gpu_launches": int(launches), "clocks": ck,
    }
    print(json.dumps(line), flush=True)


def run_tet10(args):
    """Mixed precision at scale: Tet10 box 40 x 40 x 21 cells of h = 0.025
    (201,600 elements, 6 Tet10 per hex), SNH E = 1e6 nu = 0.4, bottom
    clamped, u0 ~ N(0, (0.02 h)^2), v0 = 0; one backward-Euler Newton step
    (diagonal PCG, the reference's choice without a Schwarz component) in
    FP64 and in the mixed form; element stiffness / force errors against the
    FP64 oracle at u0."""
    import torch

    dev = torch.device("cuda", 0)
    import higher_order_embedded_fem_b200 as H

    nx, ny, nz = (int(v) for v in args.tet10_grid.split(","))
    s = H.scenes.tet10_box(0.025, nx, ny, nz, 1)
    b = s.blocks[0]
    model = H.NodalModel3d(s.vertices, b.connectivity, (b.weights, b.points))
    mat = H.StableNeoHookeanMaterial(H.YoungPoisson(1e6, 0.4))
    bc = s.nodes_below(2, 1e-9)
    u0 = H.scenes.random_normal(args.seed, model.ndof(), 0.02 * 0.025)
    v0 = np.zeros(model.ndof())
    stream = torch.cuda.current_stream(dev)
    model.set_stream(stream.cuda_stream)
    integ = H.NewtonCgIntegrator3d(model, mat, 1000.0, bc)
    integ.set_tolerances(args.cg_tol, args.cg_max_iter, 100)
    integ.set_cg_engine(args.cg_engine, False, phase_profile=args.cg_phase_profile)
    u0d, v0d = torch.from_numpy(u0).to(dev), torch.from_numpy(v0).to(dev)
    out = {}
    names = [v for v in ("plain", "mixed") if v in [x.strip() for x in args.variants.split(",")]] or ["plain", "mixed"]
    for vname in names:
        integ.set_precision(vname == "mixed", args.delta)
        for _ in range(args.warmup):
            integ.step(u0d.clone(), v0d.clone(), 0.0, DT)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            ud, vd = u0d.clone(), v0d.clone()
            st = integ.step(ud, vd, 0.0, DT)
        ev1.record(stream)
        torch.cuda.synchronize()
        out[vname] = {"ms_per_step": ev0.elapsed_time(ev1) / args.steps, "cg_iterations": int(st["total_cg_iterations"]),
                      "newton_iterations": int(st["newton_iterations"]),
                      "phase_ms": {"forces": st["ms_assemble_forces"], "stiffness": st["ms_assemble_stiffness"],
                                   "cg": st["ms_cg"], "total": st["ms_total"]},
                      "cg_engine": integ.cg_engine_stats(), "u": ud.cpu().numpy()}
    if "plain" in out and "mixed" in out:
        up, um = out["plain"].pop("u"), out["mixed"].pop("u")
        out["mixed"]["rel_diff_u_vs_plain"] = float(np.abs(um - up).max() / np.abs(up).max())
    for v in out.values():
        v.pop("u", None)
    # the element stiffness alone (device arrays; adds into K); CUDA events on
    # the model's stream
    stiff = {}
    Kd = torch.zeros(model.nnz, dtype=torch.float64, device=dev)
    reps = max(3, args.steps)
    # auto: FP32 on the tensor cores, FP64 on the CUDA cores with staged
    # node-pair blocks and the gather; cuda_cores: the colored scatter kernels
    for name, path, f32 in (("fp32_tensor_cores", "auto", True), ("fp32_staged_pairs", "staged", True),
                            ("fp32_colored", "cuda_cores", True), ("fp64_staged_pairs", "auto", False),
                            ("fp64_colored", "cuda_cores", False)):
        model.set_stiffness_path(path)
        for _ in range(3):
            model.assemble_stiffness_into_precision(Kd, u0d, mat, f32)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(reps):
            model.assemble_stiffness_into_precision(Kd, u0d, mat, f32)
        ev1.record(stream)
        torch.cuda.synchronize()
        stiff[name] = ev0.elapsed_time(ev1) / reps
    model.set_stiffness_path("auto")
    del Kd
    ntiles = -(-model.num_elements // 14)
    # tensor work the kernel issues: per 14-element tile 2 K chunks x 8 K steps
    # x 3 products of M 128, N 64, K 8 (TF32)
    tflop = 3 * 2 * 128 * 64 * 128 * ntiles / 1e12
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    bf16 = json.load(open(peaks_path))["bf16_tflops"] if os.path.exists(peaks_path) else 1590.0
    stiff["tensor_roofline"] = {
        "kernel": "k_stiffness_tc + k_stiffness_gather", "bound": "tensor", "unit": "TFLOP/s",
        "achieved": tflop / (stiff["fp32_tensor_cores"] * 1e-3), "peak": bf16 / 2,
        "frac": tflop / (stiff["fp32_tensor_cores"] * 1e-3) / (bf16 / 2),
        "peak_source": "measured bf16 dense / 2 (TF32 rate)" if os.path.exists(peaks_path) else "fallback / 2",
        "tflop_per_launch": tflop, "traffic": None}
    # element arithmetic errors at u0 against the FP64 oracle (host arrays)
    K64 = model.assemble_stiffness_into_par(np.zeros(model.nnz), u0, mat)
    K32 = model.assemble_stiffness_into_precision(np.zeros(model.nnz), u0, mat, True)
    f64 = model.assemble_elastic_pseudo_forces_into_par(np.zeros(model.ndof()), u0, mat)
    errs = {"stiffness_fp32_vs_fp64_gpu": float(np.abs(K32 - K64).max() / np.abs(K64).max())}
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        ref = O.Scene(s.vertices)
        ref.add_block(O.ELEM_TET10, b.connectivity, b.weights, b.points)
        ref.finalize_pattern()
        ref.set_material(O.MAT_SNH, mat.lame.mu, mat.lame.lam, 1000.0)
        Kr = ref.stiffness(u0)
        fr = ref.forces(u0)
        errs.update({"stiffness_fp64_vs_oracle": float(np.abs(K64 - Kr).max() / np.abs(Kr).max()),
                     "stiffness_fp32_vs_oracle": float(np.abs(K32 - Kr).max() / np.abs(Kr).max()),
                     "forces_fp64_vs_oracle": float(np.abs(f64 - fr).max() / np.abs(fr).max())})
    line = {"metric": "Newton-step ms, plain FP64 vs mixed, Tet10 box %d elements, 1 GPU" % model.num_elements,
            "value": out[names[-1]]["ms_per_step"], "unit": "ms", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": False, "dtype": "f64/f32", "data": "synthetic (seeded)",
            "config": {"workload": "Tet10 box %dx%dx%d cells h=0.025 x6 tets, SNH E=1e6 nu=0.4, u0 ~ N(0,(0.02h)^2), "
                                   "one BE Newton step dt=1e-3, diagonal PCG to %g" % (nx, ny, nz, args.cg_tol),
                       "elements": int(model.num_elements), "ndof": int(model.ndof()), "nnz": int(model.nnz)},
            "variants": out, "speedup_mixed_vs_plain": (out["plain"]["ms_per_step"] / out["mixed"]["ms_per_step"]
                                                        if len(out) == 2 else None),
            "stiffness_ms": stiff, "errors": errs}
    print(json.dumps(line), flush=True)


def run_embed(args):
    """Embedded quadrature construction for the benchmark's background grid:
    Hex27 24^3 on [0, 1]^3, hollow-cylinder Tet4 mesh (r 0.3-0.4, 3 x 144 x 72
    cells x 6 = 186,624 tets); embed_mesh_3d, the cut-cell rules of
    tet_quadrature_strength_3, simplified to strength 3.  Each stage timed
    through the public API with host arrays (device work + copies), the
    oracle on all host cores on the same input."""
    import higher_order_embedded_fem_b200 as H

    bg = H.scenes.hex27_box(1.0, 1, 1, 1, 24)
    V, conn = bg.vertices, bg.blocks[0].connectivity
    X, T = H.scenes.hollow_cylinder_tets(0.3, 0.4, 1.0, 3, 144, 72)
    tq = H.tet_quadrature_strength(3)
    H.embed_mesh_3d(V, conn, X[T[0]], np.array([[0, 1, 2, 3]]))  # context / module load outside the timing
    runs = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        emb = H.embed_mesh_3d(V, conn, X, T)
        t1 = time.perf_counter()
        o, w, p = H.embedding.compute_interface_quadrature_rules(emb, tq)
        t2 = time.perf_counter()
        oo, ow, op = H.embedding.simplify_rules(o, w, p, 3)
        t3 = time.perf_counter()
        if it >= args.warmup:
            runs.append((t1 - t0, t2 - t1, t3 - t2))
    g = np.median(np.array(runs), axis=0) * 1e3
    line = {"metric": "embedded quadrature construction ms (classify + cut-cell rules + simplify), 1 GPU",
            "value": float(g.sum()), "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": False, "dtype": "f64", "data": "synthetic (procedural hollow cylinder)",
            "config": {"workload": "Hex27 24^3 background, hollow-cylinder Tet4 mesh 186,624 tets, tet rule strength 3, "
                                   "simplified to strength 3", "background_cells": int(len(conn)), "tets": int(len(T)),
                       "interface_cells": int(len(emb.interface_cells)), "interior_cells": int(len(emb.interior_cells)),
                       "cut_points": int(len(w)), "simplified_points": int(len(ow))},
            "stages_ms": {"embed_mesh_3d": float(g[0]), "interface_quadrature": float(g[1]), "simplify": float(g[2])},
            "e2e": {"value": float(g.sum()), "unit": "ms", "h2d_bytes_per_step": int(V.nbytes + conn.nbytes + X.nbytes +
                                                                                 T.nbytes + w.nbytes + p.nbytes),
                    "d2h_bytes_per_step": int(w.nbytes + p.nbytes + ow.nbytes + op.nbytes)}}
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        t0 = time.perf_counter()
        ref = O.Embedding(V, conn, X, T)
        t1 = time.perf_counter()
        ro, rw, rp = ref.interface_quadratures(*tq)
        t2 = time.perf_counter()
        O.simplify_quadratures(ro, rw, rp, 3)
        t3 = time.perf_counter()
        line["cpu_baseline"] = {"value": (t3 - t0) * 1e3, "unit": "ms", "cores": O.num_threads(), "kind": "port",
                                "sample": "the full workload once",
                                "stages_ms": {"embed_mesh_3d": (t1 - t0) * 1e3, "interface_quadrature": (t2 - t1) * 1e3,
                                              "simplify": (t3 - t2) * 1e3}}
        line["classification_equal"] = bool(np.array_equal(ref.cell_class, emb.cell_class))
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "tet10":
        run_tet10(args)
    elif args.workload == "embed":
        run_embed(args)
    elif args.roofline_only:
        run_roofline_only(args)
    else:
        run_hoefem(args)


if __name__ == "__main__":
    main()
