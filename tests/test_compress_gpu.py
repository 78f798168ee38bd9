"""GPU parity of stream compaction against the oracle and the golden fixtures.

All results are bit-exact (values and indices).  Lengths follow the
reference grids (k * 20 * S^2 with odd offsets, tests/test_compress.py) plus
edge cases: empty input, all-zero and all-one masks, ragged tails, masks with
values other than 0/1 (treated as boolean), and the 2^28-element config.
"""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"

_OFFSETS = [-127, -13, 13, 65, 129]


def _case(n, dtype, seed, p=0.5):
    g = torch.Generator().manual_seed(seed)
    if dtype in (torch.float16, torch.float32, torch.float64):
        x = torch.randn(n, generator=g).to(dtype)
    else:
        x = torch.randint(-(2 ** 7) + 1, 2 ** 7 - 1, (n,), generator=g).to(dtype)
    mask = (torch.rand(n, generator=g) < p).to(torch.int8)
    return x, mask


@pytest.mark.parametrize("dtype", [torch.float16, torch.int16, torch.float32, torch.int32, torch.int8, torch.float64])
@pytest.mark.parametrize("n", [1, 17, 4096, 8191, 8192, 8193, 20 * 32 * 32 - 127, 20 * 64 * 64 + 129, 1_000_003])
def test_compress_vs_oracle(dtype, n):
    import tcuscan_ops

    x, m = _case(n, dtype, n)
    z = tcuscan_ops.run_compress(x.to(DEV), m.to(DEV), 32).cpu()
    ref = oracle.compress(x.numpy(), m.numpy())
    assert z.dtype == x.dtype and np.array_equal(z.numpy(), ref)


@pytest.mark.parametrize("dtype", [torch.float16, torch.int16, torch.float32, torch.int32, torch.int8, torch.float64])
@pytest.mark.parametrize("n", [1, 17, 8191, 8192, 8193, 3 * 8192 + 77, 1_000_003])
def test_compress_positions_vs_oracle(dtype, n):
    """Positions of the selected elements (run_compress_ind_no_arange): the
    compaction keeps 16-bit tile-local offsets and adds the tile start on the
    way out, for every element size's tile length."""
    import tcuscan_ops

    x, m = _case(n, dtype, n + 5)
    z, pos = tcuscan_ops.run_compress_ind_no_arange(x.to(DEV), m.to(DEV), 64)
    ref = oracle.compress(x.numpy(), m.numpy())
    want = np.nonzero(m.numpy())[0].astype(np.int32)
    assert np.array_equal(z.cpu().numpy(), ref)
    assert pos.dtype == torch.int32 and np.array_equal(pos.cpu().numpy(), want)


@pytest.mark.parametrize("S", [32, 64, 128])
@pytest.mark.parametrize("mult", [1, 3])
@pytest.mark.parametrize("off", _OFFSETS)
def test_compress_reference_grid(S, mult, off):
    import tcuscan_ops

    n = mult * 20 * S * S - off
    x, m = _case(n, torch.float32, n)
    xd, md = x.to(DEV), m.to(DEV)
    z = tcuscan_ops.run_compress(xd, md, S)
    assert torch.equal(z, torch.masked_select(xd, md.bool()))
    zi, idx = tcuscan_ops.run_compress_ind(xd, torch.arange(n, dtype=torch.int32, device=DEV), md, S)
    assert torch.equal(zi, z) and torch.equal(idx, torch.nonzero(md).flatten().int())
    zn, pos = tcuscan_ops.run_compress_ind_no_arange(xd, md, S)
    assert torch.equal(zn, z) and pos.dtype == torch.int32 and torch.equal(pos, idx)
    zp = tcuscan_ops.run_compress_pos(xd, md, int(md.sum()), S)
    assert torch.equal(zp, z)


def test_compress_golden(golden):
    import tcuscan_ops

    keys = sorted({k[: -len("_ref")] for k in golden.files if k.startswith("compress_") and k.endswith("_ref")})
    assert keys
    for b in keys:
        x = torch.from_numpy(golden[b + "_x"]).to(DEV)
        m = torch.from_numpy(golden[b + "_mask"]).to(DEV)
        z = tcuscan_ops.run_compress(x, m, 32).cpu().numpy()
        assert np.array_equal(z, golden[b + "_ref"]), b
        z2, idx = tcuscan_ops.run_compress_ind(x, torch.arange(x.numel(), dtype=torch.int32, device=DEV), m, 32)
        assert np.array_equal(z2.cpu().numpy(), golden[b + "_ref"]), b
        assert np.array_equal(idx.cpu().numpy(), golden[b + "_refidx"]), b


def test_compress_edge_cases():
    import tcuscan_ops

    x = torch.arange(100_000, dtype=torch.float32, device=DEV)
    zeros = torch.zeros(100_000, dtype=torch.int8, device=DEV)
    ones = torch.ones(100_000, dtype=torch.int8, device=DEV)
    assert tcuscan_ops.run_compress(x, zeros, 64).numel() == 0
    assert torch.equal(tcuscan_ops.run_compress(x, ones, 64), x)
    # non-0/1 mask values select like a boolean mask
    m = torch.tensor([0, 2, -1, 0, 5] * 20_000, dtype=torch.int8, device=DEV)
    assert torch.equal(tcuscan_ops.run_compress(x, m, 64), x[m != 0])
    # empty input
    e = torch.empty(0, dtype=torch.float16, device=DEV)
    assert tcuscan_ops.run_compress(e, torch.empty(0, dtype=torch.int8, device=DEV), 64).numel() == 0
    # compress_pos with a shorter output keeps the first output_len elements
    zp = tcuscan_ops.run_compress_pos(x, ones, 1000, 64)
    assert torch.equal(zp, x[:1000])
    # int64 indices
    z, idx = tcuscan_ops.run_compress_ind(x, torch.arange(100_000, dtype=torch.int64, device=DEV), m, 64)
    assert idx.dtype == torch.int64 and torch.equal(idx, torch.nonzero(m).flatten())
    tcuscan_ops.raise_device_error(x.device)


def test_filters_and_where():
    import tcuscan_ops

    g = torch.Generator(device=DEV).manual_seed(3)
    x = torch.randn(300_001, device=DEV, generator=g).half()
    assert torch.equal(tcuscan_ops.run_filter_greater_eq(x, 0.25, 64), x[x >= 0.25])
    assert torch.equal(tcuscan_ops.run_filter_less_eq(x, -0.5, 64), x[x <= -0.5])
    w = tcuscan_ops.run_where(x, 0.25, 64)
    assert w.dtype == torch.int32 and torch.equal(w, torch.nonzero(x >= 0.25).flatten().int())


@pytest.mark.parametrize("dtype", [torch.float16, torch.int16, torch.float32])
def test_compress_full_size_config(dtype):
    """n = 2^28 with a Bernoulli(0.3) int8 mask: exact values and positions."""
    import tcuscan_ops

    n = 1 << 28
    g = torch.Generator(device=DEV).manual_seed(0)
    mask = (torch.rand(n, device=DEV, generator=g) < 0.3).to(torch.int8)
    x = torch.randint(-1000, 1000, (n,), device=DEV, generator=g).to(dtype)
    z, pos = tcuscan_ops.run_compress_ind_no_arange(x, mask, 64)
    ref_pos = torch.nonzero(mask).flatten()
    assert pos.numel() == ref_pos.numel() and torch.equal(pos.long(), ref_pos)
    assert torch.equal(z, x[ref_pos])
    tcuscan_ops.raise_device_error(x.device)
