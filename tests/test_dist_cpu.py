"""Host logic of the sharded scan (tcuscan_b200.dist.scan_sharded) as
world-size-2 and -3 `gloo` process groups on CPU: the all_gather of the local
totals, the exclusive prefix per rank (int32 wrap for int8 input), and that the
pieces concatenate to the scan of the whole array.  The two device steps (the
local total and the chained tensor-core scan) are replaced by torch CPU forms
here; tests/test_dist_gpu.py runs the real ones."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "pytorch-tcuscan_b200")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _cpu_total(x):
    if x.dtype == torch.int8:
        return x.to(torch.int64).sum().reshape(1)
    return x.to(torch.float64).sum().reshape(1)


def _cpu_scan(x, S, prefix):
    if x.dtype == torch.int8:
        z = torch.cumsum(x.to(torch.int64), 0) + int(prefix.item())
        return ((z + 2 ** 31) % 2 ** 32 - 2 ** 31).to(torch.int32)
    return (torch.cumsum(x.to(torch.float64), 0) + float(prefix.item())).to(torch.float32)


def _worker(rank, world, port, dtype_name, lengths, q):
    import torch.distributed as dist

    for p in (REPO, PKG):
        sys.path.insert(0, p)
    from tcuscan_b200 import dist as tdist

    tdist._local_total = _cpu_total
    tdist._local_scan = _cpu_scan
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        g = torch.Generator().manual_seed(rank)
        n = lengths[rank]
        if dtype_name == "int8":
            x = torch.randint(100, 127, (n,), generator=g, dtype=torch.int64).to(torch.int8)  # large: wraps int32
        else:
            x = torch.rand(n, generator=g)
        z = tdist.scan_sharded(x)
        q.put((rank, x.numpy(), z.numpy()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dtype_name,lengths", [("int8", (9_000_000, 12_000_000, 7)), ("float32", (1000, 0, 4097))])
def test_scan_sharded_host_logic_gloo(dtype_name, lengths):
    world = len(lengths)
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, dtype_name, lengths, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    x = np.concatenate([r[1] for r in res])
    z = np.concatenate([r[2] for r in res])
    if dtype_name == "int8":
        ref = np.cumsum(x.astype(np.int64))
        ref = ((ref + 2 ** 31) % 2 ** 32 - 2 ** 31).astype(np.int32)
        assert z.dtype == np.int32 and np.array_equal(z, ref)
        assert ref.max() > 2 ** 31 - 2 ** 27 or ref.min() < -2 ** 30  # the case wraps int32
    else:
        ref = np.cumsum(x.astype(np.float64))
        assert np.max(np.abs(z - ref) / np.maximum(np.abs(ref), 1.0)) <= 1e-6


def test_exclusive_prefix_wide_totals():
    """Totals travel as int64 (int8 pieces) / float64 (float pieces): the
    prefix of the ranks before does not wrap or round to fp32; the int32 wrap
    happens only in the chained scan's output, as in the unsharded scan."""
    sys.path.insert(0, PKG)
    from tcuscan_b200 import dist as tdist

    assert tdist.total_dtype(torch.int8) == torch.int64
    assert tdist.total_dtype(torch.float16) == torch.float64 == tdist.total_dtype(torch.float32)
    t = [torch.tensor([2 ** 31 - 1], dtype=torch.int64), torch.tensor([5], dtype=torch.int64),
         torch.tensor([1], dtype=torch.int64)]
    assert int(tdist.exclusive_prefix(t, 0).item()) == 0
    assert int(tdist.exclusive_prefix(t, 1).item()) == 2 ** 31 - 1
    assert int(tdist.exclusive_prefix(t, 2).item()) == 2 ** 31 + 4
    f = [torch.tensor([1.0 + 2 ** -40], dtype=torch.float64), torch.tensor([2 ** -40], dtype=torch.float64),
         torch.tensor([0.5], dtype=torch.float64)]
    assert float(tdist.exclusive_prefix(f, 2).item()) == 1.0 + 2 ** -39  # below fp32 resolution
