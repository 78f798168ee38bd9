"""Device-side failure detection, tested without faulting the GPU.

Every wait in the kernels is bounded by %globaltimer; when one runs out the
kernel records TCU_ERR_TIMEOUT (and where) in its workspace and returns.  The
self-test entry point runs that same wait code on an mbarrier phase and a
look-back descriptor that nothing ever completes, with a 50 ms limit.  The
test reads the recorded status through the C ABI, then runs an ordinary scan
on the same stream and workspace and checks it is exact: the context is still
usable and the stale look-back state cannot leak into the next launch.
"""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.mark.parametrize("which,site", [(0, 900), (1, 100)])
def test_bounded_wait_runs_out_and_reports(which, site):
    import tcuscan_ops
    from tcuscan_ops import _lib as L

    n = 3_000_001
    ws, wsb = L.workspace(torch.device(DEV), L.lib.tcu_workspace_bytes(n, 128))
    sp = ctypes.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)
    code, _, _ = L.workspace_error(DEV, clear=True)  # start clean
    assert code == 0
    st = L.lib.tcu_selftest_wait_timeout(which, 50_000_000, ws, wsb, sp)
    assert st == 0
    code, where, _ = L.workspace_error(DEV, clear=True)
    assert code == L.TCU_ERR_TIMEOUT and where == site
    assert L.workspace_error(DEV, clear=True)[0] == 0  # cleared
    # the context and the workspace still work
    x = torch.randint(-8, 9, (n,), dtype=torch.int8, device=DEV)
    z = tcuscan_ops.run_scan_multi_core(x, 128)
    assert torch.equal(z, torch.cumsum(x.long(), 0).int())
    tcuscan_ops.raise_device_error(DEV)


def test_selftest_rejects_bad_arguments():
    from tcuscan_ops import _lib as L

    ws, wsb = L.workspace(torch.device(DEV), 1 << 20)
    sp = ctypes.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)
    assert L.lib.tcu_selftest_wait_timeout(2, 1000, ws, wsb, sp) == L.TCU_ERR_ARG
    assert L.lib.tcu_selftest_wait_timeout(0, 3_000_000_000, ws, wsb, sp) == L.TCU_ERR_ARG
    assert L.lib.tcu_selftest_wait_timeout(0, 1000, None, 0, sp) == L.TCU_ERR_WORKSPACE
