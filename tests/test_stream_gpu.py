"""Scans of host-resident data with overlapped copies (tcuscan_b200.stream):
chained chunks must give exactly the scan of the whole input (int8 bit-exact
with int32 wrap, fp16 within 1e-3 of FP64 relative to max(|ref|, 1)), with a
starting value, ragged last chunks and reuse of the same scanner."""
import ctypes

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def test_chained_halves_equal_full_scan():
    import tcuscan_ops
    from tcuscan_ops import _lib as L

    n = 3_000_017
    x = torch.randint(-8, 9, (n,), dtype=torch.int8, device=DEV)
    z = torch.empty(n, dtype=torch.int32, device=DEV)
    ws, wsb = L.workspace(torch.device(DEV), L.lib.tcu_workspace_bytes(n, 128))
    sp = ctypes.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)
    h = 1_234_560  # a multiple of 16: the second half stays 16-byte aligned
    assert L.lib.tcu_scan_chained(x.data_ptr(), L.TCU_INT8, h, 128, 5.0, None, z.data_ptr(), ws, wsb, sp) == 0
    assert L.lib.tcu_scan_chained(x.data_ptr() + h, L.TCU_INT8, n - h, 128, 0.0, z.data_ptr() + (h - 1) * 4,
                                  z.data_ptr() + h * 4, ws, wsb, sp) == 0
    ref = (torch.cumsum(x.long(), 0) + 5).int()
    assert torch.equal(z, ref)
    tcuscan_ops.raise_device_error(DEV)


@pytest.mark.parametrize("dtype", [torch.int8, torch.float16, torch.float32])
def test_scan_host_matches_oracle(dtype):
    from tcuscan_b200 import stream

    n = (1 << 22) + 12_345
    g = torch.Generator().manual_seed(n)
    if dtype == torch.int8:
        x = torch.randint(-8, 9, (n,), dtype=torch.int8, generator=g)
    else:
        x = (torch.rand(n, generator=g) * 2 - 1).to(dtype)
    xh = x.pin_memory()
    sc = stream.HostScanner(n, dtype, DEV, chunk=1 << 20)
    out = torch.empty(n, dtype=sc.out_dtype, pin_memory=True)
    for start in (0.0, 3.0):  # the scanner is reused
        sc.scan(xh, out, None, start)
        torch.cuda.synchronize()
        if dtype == torch.int8:
            assert torch.equal(out, (torch.cumsum(x.long(), 0) + int(start)).int())
        else:
            ref = oracle.scan_f64(x.numpy().astype(np.float64), start)
            assert oracle.max_rel_err(out.numpy(), ref) <= 1e-3


def test_scan_host_one_shot_small():
    from tcuscan_b200 import stream

    x = torch.randint(-8, 9, (1000,), dtype=torch.int8).pin_memory()
    out = stream.scan_host(x)
    assert torch.equal(out, torch.cumsum(x.long(), 0).int())
