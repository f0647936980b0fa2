"""bench.py's multi-rank path (replicas, one process per GPU) with two gloo
ranks on the CPU: the rank / world discovery from the torchrun environment,
the max-over-ranks timing reduction, the per-rank scene seeds (each replica
integrates its own scene, no data-path collective), and the reference arm
running on rank 0 only.  The GPU part of a rank needs a device and is covered
by the single-GPU tests.
"""
import json
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = textwrap.dedent("""
    import contextlib, datetime, io, json, os, sys
    sys.path.insert(0, {root!r})
    sys.argv = ["bench.py"]
    import numpy as np
    import torch.distributed as dist
    import bench
    import higher_order_embedded_fem_b200 as H

    world, rank, local = bench.dist_setup(2)
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    out = {{"world": world, "rank": rank, "local": local}}
    # time-like metric: the job's step time is the slowest rank's
    out["max"] = bench.max_over_ranks(1.5 + rank, world)
    # replicas: rank r integrates the scene of seed + r
    e, model, mat, bc, comp, u0, v0 = bench.workload(H, 4, 2 + rank)
    gathered = [None, None]
    dist.all_gather_object(gathered, (model.ndof(), u0.tolist()))
    out["ndof"] = [g[0] for g in gathered]
    out["u0_differ"] = bool(np.abs(np.array(gathered[0][1]) - np.array(gathered[1][1])).max() > 0)
    # the reference arm: ranks other than 0 exit without work or output
    if rank == 1:
        args = bench.parse()
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            r = bench.run_reference(args)
        out["ref_rank1_output"] = buf.getvalue()
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join({tmp!r}, "rank%d.json" % rank), "w") as f:
        json.dump(out, f)
""")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(root=ROOT, tmp=str(tmp_path)))
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(script)]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    res = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-3000:]
    outs = [json.load(open(tmp_path / ("rank%d.json" % r))) for r in range(2)]
    for r, o in enumerate(outs):
        assert o["world"] == 2 and o["rank"] == r and o["local"] == r
        assert o["max"] == 2.5
        assert o["ndof"][0] == o["ndof"][1]
        assert o["u0_differ"]
    assert outs[1]["ref_rank1_output"] == ""
