"""The multi-GPU path is replicas only: every rank scans its own input and
the job reports all ranks' elements over the slowest rank's time.  Its host
logic runs here as world-size-2 `gloo` process groups on CPU: the max over
ranks, the whole-job throughput, and the launcher contract of the reference
arm under torchrun (rank 0 alone prints its JSON line, other ranks exit 0)."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist

    sys.path.insert(0, REPO)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        ms = [3.5, 7.25][rank]
        mx = bench.max_over_ranks(ms, world, "cpu")
        q.put((rank, mx, bench.replica_throughput(world, 1 << 28, 10, mx)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_throughput_gloo():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [7.25, 7.25]  # both ranks see the slowest time
    assert res[0][2] == pytest.approx(2 * (1 << 28) * 10 / 7.25e-3)


def test_single_rank_is_identity():
    sys.path.insert(0, REPO)
    import bench

    assert bench.max_over_ranks(4.0, 1, "cpu") == 4.0
    assert bench.replica_throughput(1, 100, 2, 1.0) == pytest.approx(2e5)


def test_reference_arm_under_torchrun_prints_once():
    from oracle import build_ref

    if build_ref.built_module_path() is None:
        pytest.skip("reference CPU scan not built")
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(REPO, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] in ("reference", "port")
