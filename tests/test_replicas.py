"""Multi-GPU form of bench.py: independent replicas, one rank per GPU, no data-path
collective.  The rank logic (rendezvous, barrier, max-over-ranks device time, whole-job
aggregation, reference arm printing on rank 0 only) runs here as gloo ranks on CPU."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    r, local, w, dist = bench.dist_setup(world)
    bench.barrier(dist)
    ms = bench.reduce_max(dist, 10.0 * (rank + 1))  # rank 1 is the slow one
    q.put((r, w, ms, bench.replica_value(1000, 20, w, ms)))
    bench.barrier(dist)
    dist.destroy_process_group()


def test_replica_ranks_take_max_device_time_and_aggregate():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert all(o[2] == 20.0 for o in out)               # both ranks see the slowest rank's time
    assert all(abs(o[3] - 1000 * 20 * 2 / 20e-3 / 1e6) < 1e-9 for o in out)


def test_reference_arm_prints_once_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--workload", "c0", "--steps", "1", "--warmup", "3",
           "--fdtd-steps", "2"]
    env = dict(os.environ, OMP_NUM_THREADS="2", CUDA_VISIBLE_DEVICES="")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(ROOT), env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] in ("reference", "port")
