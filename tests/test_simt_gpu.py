"""GPU parity of the SIMT operators: csr_gather (bit-exact in its dtype),
reduce_tiles, complete_rows, complete_blocks (exact for integers, FP64 oracle
within 1e-5 relative for floats) and gen_lower (exact), against the oracle
and the golden fixtures from the reference's own test oracles."""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
FP_TOL = 1e-5


def _keys(golden, prefix):
    return sorted({k[: -len("_ref")] for k in golden.files if k.startswith(prefix) and k.endswith("_ref")})


def test_csr_gather_golden(golden):
    import tcuscan_ops

    keys = _keys(golden, "csr_gather_")
    assert keys
    for b in keys:
        v = torch.from_numpy(golden[b + "_v"]).to(DEV)
        c = torch.from_numpy(golden[b + "_c"]).to(DEV)
        x = torch.from_numpy(golden[b + "_x"]).to(DEV)
        z = tcuscan_ops.run_csr_gather(v, c, x).cpu().numpy()
        assert z.dtype == golden[b + "_ref"].dtype and np.array_equal(z, golden[b + "_ref"]), b


@pytest.mark.parametrize("dtype", [torch.float16, torch.int16, torch.float32])
@pytest.mark.parametrize("col_len", [16 * 1024, 61 * 1024 - 13, 1024 * 1024 - 31, 7])
@pytest.mark.parametrize("x_len", [256, 70000, 1 << 20])
def test_csr_gather_vs_oracle(dtype, col_len, x_len):
    import tcuscan_ops

    g = torch.Generator().manual_seed(col_len + x_len)
    if dtype == torch.int16:
        v = torch.randint(-300, 300, (col_len,), generator=g, dtype=dtype)
        x = torch.randint(-300, 300, (x_len,), generator=g, dtype=dtype)
    else:
        v = torch.randn(col_len, generator=g).to(dtype)
        x = torch.randn(x_len, generator=g).to(dtype)
    c = torch.randint(0, x_len, (col_len,), generator=g, dtype=torch.int32)
    z = tcuscan_ops.run_csr_gather(v.to(DEV), c.to(DEV), x.to(DEV)).cpu().numpy()
    assert np.array_equal(z, oracle.csr_gather(v.numpy(), c.numpy(), x.numpy()))


def test_csr_gather_argument_checks():
    import tcuscan_ops

    v = torch.ones(10, dtype=torch.float16, device=DEV)
    with pytest.raises(ValueError):
        tcuscan_ops.run_csr_gather(v, torch.zeros(9, dtype=torch.int32, device=DEV), v)
    with pytest.raises(TypeError):
        tcuscan_ops.run_csr_gather(v, torch.zeros(10, dtype=torch.int64, device=DEV), v)
    with pytest.raises(TypeError):
        tcuscan_ops.run_csr_gather(v, torch.zeros(10, dtype=torch.int32, device=DEV), v.float())


def test_csr_gather_out_of_range_is_reported():
    import tcuscan_ops

    v = torch.ones(64, dtype=torch.float32, device=DEV)
    x = torch.ones(8, dtype=torch.float32, device=DEV)
    c = torch.zeros(64, dtype=torch.int32, device=DEV)
    c[5] = 100
    z = tcuscan_ops.run_csr_gather(v, c, x)
    assert float(z[5]) == 0.0 and float(z[4]) == 1.0
    code, _, _ = tcuscan_ops.workspace_error(DEV)
    assert code == 1  # TCU_ERR_ARG recorded, no out-of-bounds read


def test_reduce_tiles_golden(golden):
    import tcuscan_ops

    keys = _keys(golden, "reduce_tiles_")
    assert keys
    for b in keys:
        n, tl, nb = (int(v) for v in b.split("_")[-3:])
        x = torch.from_numpy(golden[b + "_x"]).to(DEV)
        z = tcuscan_ops.run_reduce_tiles(x, tl, nb).cpu().numpy()
        ref = golden[b + "_ref"]
        if x.dtype == torch.int8:
            assert np.array_equal(z, ref), b
        else:
            assert oracle.max_rel_err(z, oracle.reduce_tiles(golden[b + "_x"], tl, nb)) < FP_TOL, b


@pytest.mark.parametrize("dtype", [torch.int8, torch.float16])
@pytest.mark.parametrize("s", [16, 32, 64, 128])
@pytest.mark.parametrize("offset", [-127, -1, 0, 11, 34])
def test_reduce_tiles_grid(dtype, s, offset):
    import tcuscan_ops

    n = 3 * 40 * 128 * 128 + offset
    g = torch.Generator().manual_seed(n)
    x = torch.randint(-3, 3, (n,), generator=g, dtype=torch.int8) if dtype == torch.int8 else (
        0.1 * torch.randn(n, generator=g)).half()
    tl = s * s // 2
    z = tcuscan_ops.run_reduce_tiles(x.to(DEV), tl, 40).cpu().numpy()
    ref = oracle.reduce_tiles(x.numpy(), tl, 40)
    if dtype == torch.int8:
        assert np.array_equal(z, ref)
    else:
        assert oracle.max_rel_err(z, ref) < FP_TOL


def test_complete_rows_golden(golden):
    import tcuscan_ops

    keys = _keys(golden, "complete_rows_")
    assert keys
    for b in keys:
        nb, tl = (int(v) for v in b.split("_")[-2:])
        x = torch.from_numpy(golden[b + "_x"]).to(DEV)
        sums = torch.from_numpy(golden[b + "_sums"]).to(DEV)
        z = tcuscan_ops.run_complete_rows(x, sums, tl, tl).cpu().numpy()
        if x.dtype == torch.int32:
            assert np.array_equal(z, golden[b + "_ref"]), b
        else:
            ref = oracle.complete_rows(golden[b + "_x"], golden[b + "_sums"], tl)
            assert oracle.max_rel_err(z, ref) < FP_TOL, b


@pytest.mark.parametrize("num_blocks", [2, 10, 20, 40])
@pytest.mark.parametrize("tile_len", [32, 128, 512])
def test_complete_rows_grid(num_blocks, tile_len):
    import tcuscan_ops

    n = num_blocks * tile_len * tile_len * 3
    g = torch.Generator().manual_seed(n)
    x = 0.1 * torch.randn(n, generator=g)
    sums = x.reshape(num_blocks, -1).sum(1)
    z = tcuscan_ops.run_complete_rows(x.to(DEV), sums.to(DEV), tile_len, tile_len).cpu().numpy()
    assert oracle.max_rel_err(z, oracle.complete_rows(x.numpy(), sums.numpy(), tile_len)) < FP_TOL


def test_complete_rows_rejects_non_positive_width():
    import tcuscan_ops

    x = torch.zeros(64, device=DEV)
    with pytest.raises(ValueError):
        tcuscan_ops.run_complete_rows(x, torch.zeros(2, device=DEV), 0, 0)


def test_complete_blocks_golden(golden):
    import tcuscan_ops

    keys = _keys(golden, "complete_blocks_")
    assert keys
    for b in keys:
        x = torch.from_numpy(golden[b + "_x"]).to(DEV)
        sums = torch.from_numpy(golden[b + "_sums"]).to(DEV)
        z = tcuscan_ops.run_complete_blocks(x, sums, 256).cpu().numpy()
        if x.dtype == torch.int32:
            assert np.array_equal(z, golden[b + "_ref"]), b
        else:
            assert oracle.max_rel_err(z, oracle.complete_blocks(golden[b + "_x"], golden[b + "_sums"])) < FP_TOL, b


@pytest.mark.parametrize("dtype", [torch.float32, torch.int32])
@pytest.mark.parametrize("num_blocks", [2, 10, 80])
@pytest.mark.parametrize("s", [32, 128])
def test_complete_blocks_grid(dtype, num_blocks, s):
    import tcuscan_ops

    n = num_blocks * s * s * 3
    g = torch.Generator().manual_seed(n)
    x = (0.1 * torch.randn(n, generator=g)) if dtype == torch.float32 else torch.randint(0, 3, (n,), generator=g,
                                                                                             dtype=torch.int32)
    sums = x.reshape(num_blocks, -1).sum(1, dtype=dtype)
    z = tcuscan_ops.run_complete_blocks(x.to(DEV), sums.to(DEV), s * s // 4).cpu().numpy()
    ref = oracle.complete_blocks(x.numpy(), sums.numpy())
    if dtype == torch.int32:
        assert np.array_equal(z, ref)
    else:
        assert oracle.max_rel_err(z, ref) < FP_TOL


@pytest.mark.parametrize("s", [32, 64, 128, 256, 1024])
@pytest.mark.parametrize("dtype", [torch.int8, torch.float16])
def test_gen_lower(s, dtype):
    import tcuscan_ops

    z = tcuscan_ops.run_gen_lower(s, torch.device(DEV), dtype)
    assert torch.equal(z, torch.tril(torch.ones((s, s), dtype=dtype, device=DEV)))


# ---- gather_spmv (the row-pointer gather of the v1 SpMV) -----------------------
@pytest.mark.parametrize("offset", [0, 7, 17])
@pytest.mark.parametrize("multiplier", [1, 4, 15])
@pytest.mark.parametrize("s", [64, 128])
def test_gather_spmv_reference_grid(offset, multiplier, s):
    """Grid of the reference test (tests/test_gather_spmv.py): nnz = m*20*s*s
    fp32 values, s*s - offset sorted uint32 indices in [0, nnz); exact."""
    import tcuscan_ops

    nnz = multiplier * 20 * s * s
    n_idx = s * s - offset
    rng = np.random.default_rng(nnz + n_idx)
    vals = rng.uniform(1, 100, nnz).astype(np.float32)
    idx = np.sort(rng.uniform(0, nnz, n_idx)).astype(np.uint32)
    expect = np.where(idx >= 1, vals[np.maximum(idx.astype(np.int64) - 1, 0)], 0).astype(np.float32)
    got = tcuscan_ops.run_gather_spmv(torch.from_numpy(vals).to(DEV), torch.from_numpy(idx).to(DEV), s)
    assert got.dtype == torch.float32 and got.shape == (n_idx,)
    assert np.array_equal(got.cpu().numpy(), expect)


@pytest.mark.parametrize("vdtype", [torch.float16, torch.float32, torch.float64])
@pytest.mark.parametrize("idtype", [torch.int32, torch.int64])
def test_gather_spmv_dtypes_and_v1_spmv(vdtype, idtype):
    """Other dtypes, and the reference's v1 SpMV built from the pieces:
    diff(gather_spmv(scan(products), indptr)) equals the row sums."""
    import tcuscan_ops

    rng = np.random.default_rng(3)
    n = 50_000
    vals = torch.from_numpy(rng.standard_normal(n)).to(vdtype)
    idx = torch.from_numpy(np.sort(rng.integers(0, n + 1, 4000))).to(idtype)
    got = tcuscan_ops.run_gather_spmv(vals.to(DEV), idx.to(DEV), 128).cpu()
    ref = torch.where(idx >= 1, vals[(idx - 1).clamp_min(0)], torch.zeros((), dtype=vdtype))
    assert torch.equal(got, ref)
    # v1 SpMV composition on fp32 products
    lens = rng.integers(0, 40, 3000)
    indptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    prod = rng.standard_normal(int(indptr[-1])).astype(np.float32)
    scanned = tcuscan_ops.run_scan_multi_core(torch.from_numpy(prod).to(DEV), 64)
    rows = torch.diff(tcuscan_ops.run_gather_spmv(scanned, torch.from_numpy(indptr).to(DEV), 128)).cpu().numpy()
    ref_rows = oracle.seg_sum_indptr(prod, indptr.astype(np.int64))
    assert oracle.max_rel_err(rows, ref_rows, floor=float(np.abs(np.cumsum(prod.astype(np.float64))).max())) <= 1e-4
