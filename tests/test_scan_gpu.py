"""GPU parity of the tensor-core scan family against the oracle (B200).

Tolerances: int8 -> int32 bit-exact; float16 -> float32 within 1e-3 of the
FP64 cumsum relative to max(|ref|, 1) (the reference's own
test uses atol=1e-3, rtol=1e-7 against an fp32 cumsum,
tests/test_scan_multi_core.py:53-55).  Shapes follow the reference's grids:
k * 20 * S^2 lengths, odd offsets and unaligned tails.
"""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu

FP16_TOL = 1e-3
DEV = "cuda:0"


def _x(n, dtype, seed=0):
    g = torch.Generator().manual_seed(seed)
    if dtype == torch.int8:
        return torch.randint(-8, 9, (n,), dtype=torch.int8, generator=g)
    return (torch.rand(n, generator=g) * 2 - 1).half()


def _check(z, x, start=0.0):
    import tcuscan_ops

    tcuscan_ops.raise_device_error(z.device)
    zc = z.cpu().numpy()
    if x.dtype == torch.int8:
        assert z.dtype == torch.int32
        ref = oracle.scan(x.numpy(), int(start))
        bad = np.nonzero(zc != ref)[0]
        assert bad.size == 0, f"first mismatch at {bad[:5]} of n={x.numel()}: got {zc[bad[:5]]} want {ref[bad[:5]]}"
    else:
        assert z.dtype == torch.float32
        ref = oracle.scan_f64(x.numpy().astype(np.float64), start)
        err = oracle.max_rel_err(zc, ref)
        assert err <= FP16_TOL, f"max rel err {err} n={x.numel()}"


SIZES = [1, 2, 15, 16, 17, 127, 1000, 4095, 4096, 4097, 8191, 8192, 8193, 20 * 64 * 64 - 13, 20 * 64 * 64,
         20 * 64 * 64 + 129, 3 * 20 * 128 * 128 + 7, 1_000_003]


@pytest.fixture(params=["simt", "tensor"])
def scan_path(request):
    """Full scans up to tcu_get_simt_scan_limit() elements run on the SIMT
    cores; "tensor" sets the limit to 0 so the same sizes run on the tensor
    cores (small tiles)."""
    from tcuscan_ops import _lib

    if request.param == "tensor":
        _lib.lib.tcu_set_simt_scan_limit(0)
    yield request.param
    _lib.lib.tcu_set_simt_scan_limit(-1)


@pytest.mark.parametrize("S", [32, 64, 128])
@pytest.mark.parametrize("n", SIZES)
def test_scan_int8(S, n, scan_path):
    import tcuscan_ops

    x = _x(n, torch.int8, seed=n)
    z = tcuscan_ops.run_scan_multi_core(x.to(DEV), S)
    _check(z, x)


@pytest.mark.parametrize("S", [16, 32, 64, 128])
@pytest.mark.parametrize("n", SIZES)
def test_scan_fp16(S, n, scan_path):
    import tcuscan_ops

    x = _x(n, torch.float16, seed=n)
    z = tcuscan_ops.run_scan_multi_core(x.to(DEV), S)
    _check(z, x)


@pytest.mark.parametrize("dtype", [torch.int8, torch.float16])
def test_scan_2e20_config(dtype, scan_path):
    """The 1-D fp16 prefix sum config (n = 2^20, uniform[-1,1), S=64) and its int8 twin."""
    import tcuscan_ops

    x = _x(1 << 20, dtype, seed=0)
    z = tcuscan_ops.run_scan_multi_core(x.to(DEV), 64)
    _check(z, x)


@pytest.mark.parametrize("dtype", [torch.int8, torch.float16])
def test_scan_single_core_starting_sum(dtype, scan_path):
    import tcuscan_ops

    for n, start in ((100, 7), (64 * 64 * 3 - 17, -11), (200_001, 5)):
        x = _x(n, dtype, seed=n)
        z = tcuscan_ops.run_scan_single_core(x.to(DEV), 64, starting_sum=start)
        _check(z, x, start)


def test_scan_no_l2_and_multi_cube_match():
    import tcuscan_ops

    x = _x(300_000, torch.float16, seed=3).to(DEV)
    a = tcuscan_ops.run_scan_multi_core(x, 64)
    b = tcuscan_ops.run_scan_multi_core_no_l2(x, 64)
    ones = torch.ones(64, 64, dtype=torch.float16, device=DEV)
    c = tcuscan_ops.run_scan_multi_cube(x, torch.triu(ones), torch.tril(ones, -1))
    _check(a, x.cpu())
    assert torch.allclose(a, b, rtol=0, atol=1e-3) and torch.allclose(a, c, rtol=0, atol=1e-3)


def test_scan_repeated_launches_reuse_workspace():
    """Epoch-tagged look-back flags: back-to-back launches on one workspace."""
    import tcuscan_ops

    x = _x(5_000_000, torch.int8, seed=9)
    xd = x.to(DEV)
    ref = torch.cumsum(xd, 0, dtype=torch.int32)
    for _ in range(5):
        z = tcuscan_ops.run_scan_multi_core(xd, 64)
        assert torch.equal(z, ref)
    tcuscan_ops.raise_device_error(xd.device)


def test_scan_unaligned_view():
    import tcuscan_ops

    x = _x(10_001, torch.int8, seed=4)
    xd = x.to(DEV)[1:]
    z = tcuscan_ops.run_scan_multi_core(xd, 64)
    _check(z, x[1:])


@pytest.mark.parametrize("S", [16, 32, 64, 128])
def test_row_scan_golden(golden, S):
    import tcuscan_ops

    x = torch.from_numpy(golden[f"row_scan_{S}_x"])
    z = tcuscan_ops.run_row_scan(x.to(DEV), S).cpu().numpy()
    assert oracle.max_rel_err(z, golden[f"row_scan_{S}_ref"]) < 1e-5
    assert oracle.max_rel_err(z, oracle.segment_scan_fixed(x.numpy().reshape(-1), S)) < 1e-6


@pytest.mark.parametrize("S", [32, 64, 128])
def test_row_scan_int8(S):
    import tcuscan_ops

    x = torch.randint(-100, 100, (1000, S), dtype=torch.int8)
    z = tcuscan_ops.run_row_scan(x.to(DEV), S).cpu().numpy()
    assert np.array_equal(z, oracle.segment_scan_fixed(x.numpy().reshape(-1), S))


@pytest.mark.parametrize("S", [16, 32])
def test_block_scan_golden(golden, S):
    import tcuscan_ops

    x = torch.from_numpy(golden[f"block_scan_{S}_x"])
    ones = torch.ones(S, S, dtype=torch.float16, device=DEV)
    z = tcuscan_ops.run_block_scan(x.to(DEV), torch.triu(ones), torch.tril(ones, -1)).cpu().numpy()
    assert oracle.max_rel_err(z, golden[f"block_scan_{S}_ref"]) < 1e-5


@pytest.mark.parametrize("S", [16, 32, 64, 128])
@pytest.mark.parametrize("m", [1, 3, 10, 15, 21, 24])
def test_block_scan(S, m):
    """Per-S^2-tile scans (the reference's grid: m tiles of 0.1 * N(0, 1) fp16;
    its own test allows atol 1e-2 / rtol 1e-3 against an fp32 matmul).  fp16 at
    S = 64 / 128 runs the tensor-only formulation (three products per block,
    FP32 accumulation of the row offsets: 1e-4 relative to FP64, floor 1);
    the engine's block mode (exact shuffle offsets) is held to 1e-5."""
    import tcuscan_ops

    n = m * S * S
    x = (0.1 * torch.randn(n, generator=torch.Generator().manual_seed(m * S))).half()
    ones = torch.ones(S, S, dtype=torch.float16, device=DEV)
    z = tcuscan_ops.run_block_scan(x.to(DEV), torch.triu(ones), torch.tril(ones, -1)).cpu().numpy()
    tcuscan_ops.raise_device_error(DEV)
    ref = oracle.segment_scan_fixed(x.numpy(), S * S)
    assert oracle.max_rel_err(z, ref) < (1e-4 if S in (64, 128) else 1e-5)


@pytest.mark.parametrize("S", [64, 128])
def test_block_scan_tensor_uses_the_callers_matrices(S):
    """The tensor-only block scan multiplies by the matrices it is given, as the
    reference's kernel does: z = A.upper + lower_strict.(A.J) per S x S tile."""
    import tcuscan_ops

    m = 5
    g = torch.Generator().manual_seed(S)
    x = (0.1 * torch.randn(m * S * S, generator=g)).half()
    upper = (torch.triu(torch.ones(S, S)) * 2).half()
    lower = (torch.tril(torch.ones(S, S), -1) * 0.5).half()
    z = tcuscan_ops.run_block_scan(x.to(DEV), upper.to(DEV), lower.to(DEV)).cpu().double()
    tcuscan_ops.raise_device_error(DEV)
    A = x.double().reshape(m, S, S)
    J = torch.ones(S, S, dtype=torch.float64)
    ref = (A @ upper.double() + lower.double() @ (A @ J)).reshape(-1)
    err = ((z - ref).abs() / ref.abs().clamp_min(1.0)).max().item()
    assert err < 1e-4, err


@pytest.mark.parametrize("S", [64, 128, None])
def test_scan_full_size_int8_property(S):
    """n = 2^28 int8: z[0] == x[0] and diff(z) == x[1:] exactly, which pins z = cumsum(x).
    S = 128 and S = None (autotuned) are the benchmark's headline configuration."""
    import tcuscan_ops

    n = 1 << 28
    g = torch.Generator(device=DEV).manual_seed(0)
    x = torch.randint(-8, 9, (n,), dtype=torch.int8, device=DEV, generator=g)
    z = tcuscan_ops.run_scan_multi_core(x, S)
    tcuscan_ops.raise_device_error(x.device)
    assert int(z[0]) == int(x[0])
    d = torch.diff(z)
    assert torch.equal(d, x[1:].to(torch.int32))
    assert int(z[-1]) == int(x.to(torch.int64).sum())


@pytest.mark.parametrize("S", [64, None])
def test_scan_full_size_fp16_vs_fp64(S):
    """n = 2^28 fp16 uniform[-1,1): max rel error vs an FP64 cumsum <= 1e-3."""
    import tcuscan_ops

    n = 1 << 28
    g = torch.Generator(device=DEV).manual_seed(0)
    x = (torch.rand(n, device=DEV, generator=g) * 2 - 1).half()
    z = tcuscan_ops.run_scan_multi_core(x, S)
    tcuscan_ops.raise_device_error(x.device)
    ref = torch.cumsum(x.double(), 0)
    err = ((z.double() - ref).abs() / ref.abs().clamp_min(1.0)).max().item()
    assert err <= FP16_TOL, err
