"""The multi-GPU form of bench.py is N independent replicas (the path has no
exchange step on one rank's system): the only collectives are a barrier and
the MAX of the ranks' timings, and the reference arm runs on rank 0 alone.
Checked here with two gloo ranks on the CPU (127.0.0.1)."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import REPO

WORKER = r"""
import os, sys, datetime
sys.path.insert(0, os.environ["OWTK_REPO"])
import torch.distributed as dist
import bench
rank, world, local = bench.dist_env()
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
dist.barrier()
got = bench._max_over_ranks(10.0 + 5.0 * rank, world, local)
dist.barrier()
dist.destroy_process_group()
print("RESULT", rank, world, got, flush=True)
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_max_over_ranks_gloo_world2(tmp_path):
    port = _free_port()
    script = tmp_path / "worker.py"
    script.write_text(WORKER)
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), OWTK_REPO=REPO)
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = [p.communicate(timeout=180)[0] for p in procs]
    assert all(p.returncode == 0 for p in procs), outs
    results = sorted(line.split()[1:] for o in outs for line in o.splitlines() if line.startswith("RESULT"))
    assert results == [["0", "2", "15.0"], ["1", "2", "15.0"]], outs


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
