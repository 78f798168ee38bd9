"""The sharded scan on the GPU with a one-rank NCCL group: the result equals
the single-array scan (bit-exact for int8), through the real local total
(tcu_total: int64 / FP64) and the chained scan reading its int64 / FP64 start
value from device memory (tcu_scan_chained_typed).  Several ranks are covered
on CPU (tests/test_dist_cpu.py); one GPU is available to these tests."""
import os
import socket

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.fixture(scope="module")
def group():
    import torch.distributed as dist

    if not dist.is_initialized():
        with socket.socket() as s:
            s.bind(("127.0.0.1", 0))
            port = s.getsockname()[1]
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ["MASTER_PORT"] = str(port)
        torch.cuda.set_device(0)
        import datetime

        dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    yield None
    dist.destroy_process_group()


@pytest.mark.parametrize("dtype", [torch.int8, torch.float16, torch.float32])
@pytest.mark.parametrize("n", [1, 4097, 3_000_001])
def test_scan_sharded_one_rank(group, dtype, n):
    import tcuscan_ops
    from tcuscan_b200 import dist as tdist

    g = torch.Generator().manual_seed(n)
    if dtype == torch.int8:
        x = torch.randint(-8, 9, (n,), generator=g, dtype=torch.int64).to(dtype)
    else:
        x = (torch.rand(n, generator=g) * 2 - 1).to(dtype)
    z = tdist.scan_sharded(x.to(DEV)).cpu().numpy()
    if dtype == torch.int8:
        assert np.array_equal(z, oracle.scan(x.numpy()))
    else:
        ref = oracle.scan_f64(x.float().numpy())
        assert np.max(np.abs(z - ref) / np.maximum(np.abs(ref), 1.0)) <= 1e-4


def test_local_total_and_chained_start(group):
    from tcuscan_b200 import dist as tdist

    x = torch.randint(-8, 9, (1 << 20,), dtype=torch.int64).to(torch.int8).to(DEV)
    tot = tdist._local_total(x)
    assert tot.dtype == torch.int64 and int(tot.item()) == int(x.long().sum().item())
    for start in (torch.tensor([123456], dtype=torch.int32, device=DEV),
                  torch.tensor([2 ** 32 + 123456], dtype=torch.int64, device=DEV)):  # wraps like the int32 output
        z = tdist._local_scan(x, None, start)
        assert torch.equal(z, (torch.cumsum(x.long(), 0) + 123456).int())
    # float pieces: an FP64 total in a fixed order (same bits twice), and an
    # FP64 start below fp32 resolution of the prefix is kept by the carry chain
    for n in (1, 17, 4097, 3_000_001):
        xf = torch.randn(n, device=DEV)
        t1, t2 = tdist._local_total(xf), tdist._local_total(xf)
        assert t1.dtype == torch.float64 and torch.equal(t1, t2)
        ref = xf.double().sum().item()
        assert abs(t1.item() - ref) <= 1e-12 * max(1.0, xf.double().abs().sum().item())
        xh = xf.half()
        assert abs(tdist._local_total(xh).item() - xh.double().sum().item()) <= 1e-12 * max(1.0, n)
    # the FP64 start is read as FP64 (within one fp32 ulp of the exact sum)
    xs = torch.ones(1000, device=DEV)
    z = tdist._local_scan(xs, None, torch.tensor([2.0 ** 25 + 0.25], dtype=torch.float64, device=DEV))
    ref = torch.arange(1, 1001, device=DEV, dtype=torch.float64) + 2.0 ** 25 + 0.25
    assert (z.double() - ref).abs().max().item() <= 4.0  # one ulp at 2^25
