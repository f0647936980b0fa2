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
    ap.add_argument("--inner-tol", type=float, default=1e-2, help="mixed variant: inner FP32 PCG tolerance")
    ap.add_argument("--variants", default="plain,mixed", help="comma list: plain, mixed")
    return ap.parse_args()


def workload(H, n, seed):
    e = H.scenes.embedded_cylinder(n, 0.3, 0.4, 8, 27, seed)
    b0, b1 = e.blocks
    model = H.EmbeddedModel3d(e.vertices, b0.connectivity, b1.connectivity, (b0.weights, b0.points),
                              (b1.offsets, b1.weights, b1.points))
    mat = H.StVKMaterial(H.YoungPoisson(5e5, 0.45))
    bc = e.nodes_below(2, 1e-9)
    comp = H.SchwarzPreconditionerComponent.from_embedded_model(model, e.volume_fractions, 0.5)
    # initial state: smooth sway u = (0.02 z^2, 0.01 z^2, 0) plus seeded noise N(0, (0.001 h)^2), at rest
    X = e.vertices
    u0 = np.zeros_like(X)
    u0[:, 0] = 0.02 * X[:, 2] ** 2
    u0[:, 1] = 0.01 * X[:, 2] ** 2
    u0 = u0.reshape(-1) + H.scenes.random_normal(1000 + seed, model.ndof(), 0.001 * e.cell_size)
    v0 = np.zeros(model.ndof())
    return e, model, mat, bc, comp, u0, v0


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


def cpu_reference_step(e, model, mat, bc, comp, u0, v0, cg_tol, threads):
    """The oracle (FP64 CPU restatement of the reference path) on the same scene."""
    from oracle import oracle as O

    if threads:
        O.set_num_threads(threads)
    b0, b1 = e.blocks
    ref = O.Scene(e.vertices)
    ref.add_block(O.ELEM_HEX27, b0.connectivity, b0.weights, b0.points)
    ref.add_block(O.ELEM_HEX27, b1.connectivity, b1.weights, b1.points, qoff=b1.offsets)
    ref.finalize_pattern()
    ref.set_material(O.MAT_STVK, mat.lame.mu, mat.lame.lam, 1000.0)
    ref.set_bc(bc)
    ref.set_gravity(True)
    ref.set_schwarz(comp.schwarz_connectivity, comp.untreated_nodes)
    ref.set_solver(cg_tol, 500, 100)
    ref.setup()
    return ref


def run_reference(args):
    world, rank, local = dist_setup(args.gpus)
    if rank != 0:
        return
    import higher_order_embedded_fem_b200 as H
    from oracle import oracle as O

    e, model, mat, bc, comp, u0, v0 = workload(H, args.n, args.seed)
    threads = os.cpu_count() or 1
    ref = cpu_reference_step(e, model, mat, bc, comp, u0, v0, args.cg_tol, threads)
    stats = None
    for _ in range(args.warmup):
        ref.step(u0, v0, 0.0, DT)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, _, stats = ref.step(u0, v0, 0.0, DT)
        times.append((time.perf_counter() - t0) * 1e3)
    ms = float(np.mean(times))
    line = {
        "metric": METRIC, "value": ms, "unit": "ms", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": "embedded Hex27 hollow cylinder %d^3, StVK, one BE Newton step, Schwarz-CG 1e-6"
                   % args.n, "ndof": model.ndof(), "nnz": model.nnz},
        "cg_iterations": int(sum(stats["cg_iters"])), "newton_iterations": int(stats["newton_iters"]),
        "cpu_baseline": {"value": ms, "unit": "ms", "cores": O.num_threads(), "kind": "port",
                         "sample": "full Newton step of the workload, OpenMP per color"},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_hoefem(args):
    import torch

    world, rank, local = dist_setup(args.gpus)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
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

    u0d = torch.from_numpy(u0).to(dev)
    v0d = torch.from_numpy(v0).to(dev)
    ud, vd = u0d.clone(), v0d.clone()

    def step():
        ud.copy_(u0d)
        vd.copy_(v0d)
        return integ.step(ud, vd, 0.0, DT)

    variants = {}
    for vname in [v.strip() for v in args.variants.split(",") if v.strip()]:
        integ.set_precision(vname == "mixed", args.inner_tol)
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
        variants[vname] = {
            "ms_per_step": ms, "cg_iterations": int(s_["total_cg_iterations"]),
            "newton_iterations": int(s_["newton_iterations"]), "residual_norm": s_["residual_norm"],
            "phase_ms": {"forces": s_["ms_assemble_forces"], "stiffness": s_["ms_assemble_stiffness"],
                         "precond_update": s_["ms_precond_update"], "cg": s_["ms_cg"], "total": s_["ms_total"]},
            "gpu_launches": int(launches), "clocks": ck, "u": ud.cpu().numpy(),
        }
    head = "mixed" if "mixed" in variants else list(variants)[0]
    ms = variants[head]["ms_per_step"]
    launches = variants[head]["gpu_launches"]
    ck = variants[head]["clocks"]
    integ.set_precision(head == "mixed", args.inner_tol)
    if "mixed" in variants and "plain" in variants:
        up, um = variants["plain"]["u"], variants["mixed"]["u"]
        variants["mixed"]["rel_diff_u_vs_plain"] = float(np.abs(um - up).max() / np.abs(up).max())
    for v in variants.values():
        v.pop("u")

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

    # roofline of the dominant kernel class: node-row SpMV of the CG operator
    roof = spmv_roofline(H, model, integ, mat, ud, stream, args.roofline_reps)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref = cpu_reference_step(e, model, mat, bc, comp, u0, v0, args.cg_tol, os.cpu_count())
        from oracle import oracle as O

        t0 = time.perf_counter()
        _, _, rst = ref.step(u0, v0, 0.0, DT)
        cms = (time.perf_counter() - t0) * 1e3
        cpu = {"value": cms, "unit": "ms", "cores": O.num_threads(), "kind": "port",
               "sample": "one full Newton step of the workload (oracle, OpenMP per color)",
               "cg_iterations": int(sum(rst["cg_iters"]))}

    if rank == 0:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
            os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
        line = {
            "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded scene, replicas per rank)",
            "variant": {"mixed": "mixed_fp32", "plain": "plain_fp64"}[head],
            "variants": variants,
            "config": {"workload": "embedded Hex27 hollow cylinder %d^3 (r 0.3-0.4), StVK E=5e5 nu=0.45, one "
                                   "backward-Euler Newton step dt=1e-3, Schwarz-CG to %g" % (args.n, args.cg_tol),
                       "ndof": model.ndof(), "nnz": model.nnz, "elements": model.num_elements,
                       "schwarz_subdomains": len(comp.schwarz_connectivity),
                       "l2": "inputs larger than L2 (CSR values %d MB)" % (model.nnz * 8 // 2 ** 20),
                       "parallelism": "replicas" if world > 1 else "single"},
            "cg_iterations": variants[head]["cg_iterations"], "newton_iterations": variants[head]["newton_iterations"],
            "speedup_vs_plain_fp64": (variants["plain"]["ms_per_step"] / ms) if "plain" in variants else None,
            "roofline": roof,
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
    return {"kernel": "k_spmv (node-row SpMV, CG operator)", "bound": "hbm", "achieved": gbs, "peak": peak,
            "unit": "GB/s", "frac": gbs / peak, "traffic": None, "ms_per_launch": ms,
            "algorithmic_bytes": bytes_alg, "peak_source": "measured" if os.path.exists(peaks_path) else "fallback"}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_hoefem(args)


if __name__ == "__main__":
    main()
