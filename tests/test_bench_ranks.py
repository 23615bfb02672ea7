"""The N>1 path of bench.py on CPU: two ranks over gloo (world size 2), the
plumbing that `torchrun --nproc-per-node N bench.py` uses.  Each rank runs
bench.py's own helpers:

* dist_setup() picks gloo when no GPU is present and reports (world, rank,
  local rank);
* max_over_ranks() returns the largest per-rank time, which is what the step
  time of a replica run is;
* barrier() completes on both ranks;
* the reference arm returns on rank 1 without any work or output.

No GPU is touched; a rank that fails reports its exception through its
result file.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import contextlib, io, json, os, sys, traceback
sys.path.insert(0, os.environ["MCG_ROOT"])
out = {"rank": int(os.environ["RANK"])}
try:
    import bench
    world, rank, local = bench.dist_setup()
    import torch.distributed as dist
    out["setup"] = [world, rank, local, dist.get_backend()]
    out["max"] = bench.max_over_ranks(world, 10.0 + 5.0 * rank)
    bench.barrier(world)
    class Args:
        case = "jet_128x256x128"
        steps = 1
        warmup = 0
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        if rank != 0:
            bench.run_reference(Args, world, rank)
    out["reference_output"] = buf.getvalue()
    bench.barrier(world)
    dist.destroy_process_group()
except Exception:
    out["error"] = traceback.format_exc()
with open(os.environ["MCG_RESULT"], "w") as fh:
    json.dump(out, fh)
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_over_gloo(tmp_path):
    port = str(_free_port())
    procs = []
    for rank in (0, 1):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=port, MCG_ROOT=ROOT, MCG_RESULT=str(tmp_path / f"rank{rank}.json"),
                   CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT))
    logs = []
    for p in procs:
        try:
            logs.append(p.communicate(timeout=240)[0].decode(errors="replace"))
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            pytest.fail("a rank did not finish within 240 s")
    for rank, p in enumerate(procs):
        assert p.returncode == 0, logs[rank][-2000:]
        res = json.loads((tmp_path / f"rank{rank}.json").read_text())
        assert "error" not in res, res.get("error")
        assert res["setup"] == [2, rank, rank, "gloo"]
        assert res["max"] == 15.0  # the slower rank's time, on both ranks
        assert res["reference_output"] == ""
