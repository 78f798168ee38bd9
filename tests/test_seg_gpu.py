"""GPU parity of the segmented tensor-core operators against the oracle.

int8 inputs: bit-exact int32 results.  float16 inputs: float32 results within
1e-3 of the FP64 oracle relative to max(|ref|, 1) (the reference's own tests
use atol=1e-2, tests/test_seg_sum_multi_core.py:152-155 and
tests/test_seg_scan_single_core.py).  Shapes follow the reference grids
(segment counts {513, 1025, 2011} x column counts around S^2, densities 0,
0.01, 0.05) plus empty segments, segments spanning many 32768-element tiles,
ragged tails and the golden fixtures.
"""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL = 1e-3


def _x(n, dtype, seed):
    g = torch.Generator().manual_seed(seed)
    if dtype == torch.int8:
        return torch.randint(-8, 9, (n,), dtype=torch.int8, generator=g)
    return (torch.rand(n, generator=g) * 2 - 1).half()


def _assert_close(got, ref, exact):
    got = np.asarray(got)
    if exact:
        bad = np.nonzero(got != np.asarray(ref).astype(got.dtype))[0]
        assert bad.size == 0, f"{bad.size} mismatches, first {bad[:5]}"
    else:
        err = oracle.max_rel_err(got, ref)
        assert err <= TOL, err


# ---- flag segmented scan (starts) ----------------------------------------
@pytest.mark.parametrize("S", [32, 64])
@pytest.mark.parametrize("dens", [0.0, 0.01, 0.05, 0.5])
@pytest.mark.parametrize("n", [1, 100, 32 * 32 * 3, 64 * 64 * 9 + 13, 100_003, 1_000_000])
@pytest.mark.parametrize("dtype", [torch.float16, torch.int8])
def test_seg_scan_flags(S, dens, n, dtype):
    import tcuscan_ops

    x = _x(n, dtype, n)
    g = torch.Generator().manual_seed(n + 1)
    f = (torch.rand(n, generator=g) < dens).to(torch.int8)
    z = tcuscan_ops.run_seg_scan(x.to(DEV), f.to(DEV), S)
    tcuscan_ops.raise_device_error(DEV)
    ref = oracle.seg_scan_flags_f64(x.numpy().astype(np.float64), f.numpy())
    _assert_close(z.cpu().numpy(), ref.astype(np.int64).astype(np.int32) if dtype == torch.int8 else ref,
                  dtype == torch.int8)


def test_seg_scan_golden(golden):
    import tcuscan_ops

    keys = sorted({k[:-4] for k in golden.files if k.startswith("seg_scan_") and k.endswith("_ref")})
    assert keys
    for b in keys:
        x = torch.from_numpy(golden[b + "_x"]).to(DEV)
        f = torch.from_numpy(golden[b + "_f"]).to(DEV)
        for S in (32, 64, 128):
            z = tcuscan_ops.run_seg_scan(x, f, S).cpu().numpy()
            assert oracle.max_rel_err(z, golden[b + "_ref"]) <= 1e-6, (b, S)


# ---- flag segmented sum (ends) --------------------------------------------
def test_seg_sum_golden(golden):
    import tcuscan_ops

    keys = sorted({k[:-4] for k in golden.files if k.startswith("seg_sum_flags_") and k.endswith("_ref")})
    assert keys
    for b in keys:
        x = torch.from_numpy(golden[b + "_x"]).to(DEV)
        f = torch.from_numpy(golden[b + "_f"]).to(DEV)
        for S in (32, 64, 128):
            z = tcuscan_ops.run_seg_sum(x, f, S).cpu().numpy()
            assert z.shape == golden[b + "_ref"].shape
            assert oracle.max_rel_err(z, golden[b + "_ref"]) <= 1e-6, (b, S)


@pytest.mark.parametrize("mult", [1, 2, 5, 12])
@pytest.mark.parametrize("S", [32, 64, 128])
def test_seg_sum_flags_grid(mult, S):
    import tcuscan_ops

    n = mult * 20 * S * S
    g = torch.Generator().manual_seed(n)
    x = torch.randint(-2, 2, (n,), generator=g).half()
    f = (torch.rand(n, generator=g) < 0.01).to(torch.int8)
    f[-1] = 1
    z = tcuscan_ops.run_seg_sum(x.to(DEV), f.to(DEV), S).cpu().numpy()
    ref = oracle.seg_sum_flags_f64(x.numpy(), f.numpy())
    assert z.shape == ref.shape
    _assert_close(z, ref, False)


# ---- indptr segmented sums -------------------------------------------------
def _random_csr(rows, cols, density, seed):
    rng = np.random.default_rng(seed)
    nnz_per_row = rng.binomial(cols, density, size=rows)
    indptr = np.zeros(rows + 1, dtype=np.int64)
    np.cumsum(nnz_per_row, out=indptr[1:])
    return indptr


@pytest.mark.parametrize("rows", [513, 1025, 2011, 519, 2043])
@pytest.mark.parametrize("cols", [64 * 64 - 1, 128 * 128, 128 * 128 - 13, 128 * 128 + 13, 128 * 128 - 133])
@pytest.mark.parametrize("S", [32, 64, 128])
@pytest.mark.parametrize("dtype", [torch.int8, torch.float16])
def test_seg_sum_multi_core_grid(rows, cols, S, dtype):
    import tcuscan_ops

    indptr = _random_csr(rows, cols, 0.01, rows * cols + S)
    nnz = int(indptr[-1])
    x = _x(nnz, dtype, nnz + 7)
    ip = torch.from_numpy(indptr.astype(np.int32))
    z = tcuscan_ops.run_seg_sum_multi_core(x.to(DEV), ip.to(DEV), S).cpu().numpy()
    ref = oracle.seg_sum_indptr(x.numpy(), indptr)
    assert z.shape == (rows,)
    _assert_close(z, ref, dtype == torch.int8)


def test_seg_sum_golden_indptr(golden):
    import tcuscan_ops

    keys = sorted({k[:-4] for k in golden.files if k.startswith("seg_sum_") and k.endswith("_ref")
                   and not k.startswith("seg_sum_flags")})
    assert keys
    for b in keys:
        x = torch.from_numpy(golden[b + "_x"]).to(DEV)
        ip = torch.from_numpy(golden[b + "_indptr"]).to(DEV)
        ref = golden[b + "_ref"]
        for S in (32, 64):
            z = tcuscan_ops.run_seg_sum_multi_core(x, ip, S).cpu().numpy()
            if x.dtype == torch.int8:
                assert np.array_equal(z, ref), b
            else:
                assert oracle.max_rel_err(z, oracle.seg_sum_indptr(golden[b + "_x"], golden[b + "_indptr"])) < 1e-5, b


@pytest.mark.parametrize("dtype", [torch.int8, torch.float16])
def test_seg_sum_edge_segments(dtype):
    """Empty segments at the start, middle and end, single-element segments,
    and segments spanning many tiles (up to 200000 elements)."""
    import tcuscan_ops

    lens = [0, 0, 1, 5, 0, 200_000, 3, 0, 70_000, 1, 1, 0, 33_000, 0]
    indptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    n = int(indptr[-1])
    x = _x(n, dtype, 11)
    for S in (32, 64):
        for ipt in (torch.int32, torch.int64):
            z = tcuscan_ops.run_seg_sum_multi_core(x.to(DEV), torch.from_numpy(indptr).to(ipt).to(DEV), S).cpu().numpy()
            _assert_close(z, oracle.seg_sum_indptr(x.numpy(), indptr), dtype == torch.int8)
    tcuscan_ops.raise_device_error(DEV)


def test_seg_sum_variants_agree():
    import tcuscan_ops

    indptr = _random_csr(1025, 128 * 128 - 13, 0.01, 5)
    nnz = int(indptr[-1])
    x = _x(nnz, torch.float16, 3).to(DEV)
    ip = torch.from_numpy(indptr.astype(np.int32)).to(DEV)
    ref = oracle.seg_sum_indptr(x.cpu().numpy(), indptr)
    ones = torch.ones(64, 64, dtype=torch.float16, device=DEV)
    up, lo = torch.triu(ones), torch.tril(ones, -1)
    for z in (tcuscan_ops.run_seg_sum_multi_core(x, ip, 64, None),
              tcuscan_ops.run_seg_sum_single_core(x, ip, 64),
              tcuscan_ops.run_seg_sum_multi_cube(x, up, lo, ip),
              tcuscan_ops.run_seg_sum_single_cube(x, up, lo, ip[:-1], 64)):
        _assert_close(z.cpu().numpy(), ref, False)


# ---- batched rows ----------------------------------------------------------
@pytest.mark.parametrize("S", [32, 64, 128])
@pytest.mark.parametrize("mult", [1, 3, 11])
@pytest.mark.parametrize("batch", [2, 20, 44])
@pytest.mark.parametrize("delta", [0, -1, 1])
def test_scan_batch_fp16(S, mult, batch, delta):
    import tcuscan_ops

    L = mult * S * S + delta
    g = torch.Generator().manual_seed(L * batch)
    x = torch.rand((batch, L), generator=g).half()
    z = tcuscan_ops.run_scan_batch(x.to(DEV), S).cpu().numpy()
    ref = oracle.segment_scan_fixed(x.numpy().reshape(-1), L).reshape(batch, L)
    assert z.shape == (batch, L)
    _assert_close(z, ref, False)
