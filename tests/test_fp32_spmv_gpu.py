"""GPU parity of the split-precision fp32 paths and CSR SpMV.

fp32 inputs enter the tensor cores as two fp16 operands per value: each
64-element row is scaled by a power of two so its largest |x| lies in
[2^14, 2^15), hi is the scaled value rounded to a multiple of 16 and lo the
fp16 remainder (22 significant bits of the row's scale), with FP32
accumulation; every row's total is taken from the fp32 values themselves
(exact hi sum + FP32 remainder sum, in FP64) and carries are FP64.
Tolerances, all element-wise against the FP64 oracle with the floor
max(|ref|, 1):
- fp32 scans, segmented scans and uneven row scans: <= 1e-4 (FP32_TOL),
  on N(0,1) and uniform data;
- uniform[0,1) batch rows (the reference recipe, tests/test_scan_batch.py
  uses rtol 1e-3): <= 1e-4 as well;
- SpMV: |err| <= 1e-3 * max(|ref|, 1) against the FP64 oracle, and the
  reference test's atol=1e-1 on its own grid (tests/test_spmv_v2.py).
"""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


FP32_TOL = 1e-4


def _elementwise(got, ref):
    """max |got - ref| / max(|ref|, 1) over all elements."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if ref.size == 0:
        return 0.0
    return float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1.0)))


@pytest.fixture(params=["simt", "tensor"])
def scan_path(request):
    """Small full scans run on the SIMT cores; "tensor" sets the SIMT limit
    to 0 so the same sizes run on the tensor cores."""
    from tcuscan_ops import _lib

    if request.param == "tensor":
        _lib.lib.tcu_set_simt_scan_limit(0)
    yield request.param
    _lib.lib.tcu_set_simt_scan_limit(-1)


@pytest.mark.parametrize("n", [1, 63, 64, 65, 8191, 8192 * 4 + 17, 1_000_003, 5_000_000])
@pytest.mark.parametrize("start", [0.0, 7.5])
def test_scan_single_core_fp32(n, start, scan_path):
    import tcuscan_ops

    g = torch.Generator().manual_seed(n)
    x = torch.randn(n, generator=g)
    z = tcuscan_ops.run_scan_single_core(x.to(DEV), 64, starting_sum=start).cpu().numpy()
    tcuscan_ops.raise_device_error(DEV)
    assert z.dtype == np.float32
    assert _elementwise(z, oracle.scan_f64(x.numpy(), start)) <= FP32_TOL


def test_scan_fp32_full_size_normal():
    """n = 2^28 fp32 N(0, 1): element-wise error vs an FP64 cumsum <= 1e-4
    (floor 1), including the zero crossings of the long prefix."""
    import tcuscan_ops

    n = 1 << 28
    g = torch.Generator(device=DEV).manual_seed(3)
    x = torch.randn(n, device=DEV, generator=g)
    z = tcuscan_ops.run_scan_multi_core(x, 64)
    tcuscan_ops.raise_device_error(x.device)
    ref = torch.cumsum(x.double(), 0)
    err = ((z.double() - ref).abs() / ref.abs().clamp_min(1.0)).max().item()
    assert err <= FP32_TOL, err


def test_scan_batch_fp32_row_scales():
    """Rows of 64 values whose magnitudes differ by up to 2^+-120 (and rows of
    zeros, subnormals and single large values): each 64-element row is one
    batch row, so every row's result is checked against its own scale."""
    import tcuscan_ops

    rng = np.random.default_rng(7)
    rows = 4096
    e = rng.integers(-120, 121, size=rows).astype(np.float64)
    x = rng.standard_normal((rows, 64)) * np.exp2(e)[:, None]
    x[3] = 0.0
    x[5] = 1e-41  # fp32 subnormals
    x[9] = 0.0
    x[9, 17] = 3e38
    x[11, :] = 1.0
    x[11, 40] = 2.0 ** 100
    x32 = x.astype(np.float32)
    z = tcuscan_ops.run_scan_batch(torch.from_numpy(x32).to(DEV), 64).cpu().numpy().astype(np.float64)
    ref = np.cumsum(x32.astype(np.float64), axis=1)
    scale = np.maximum(np.abs(ref).max(axis=1, keepdims=True), np.abs(x32).max(axis=1, keepdims=True).astype(np.float64))
    scale = np.where(scale > 0, scale, 1.0)
    err = np.abs(z - ref) / scale
    assert np.all(np.isfinite(z)), "non-finite result from finite input"
    assert err.max() <= FP32_TOL, (err.max(), int(err.max(axis=1).argmax()))


@pytest.mark.parametrize("S", [32, 64, 128])
@pytest.mark.parametrize("mult", [1, 2, 11])
@pytest.mark.parametrize("batch", [2, 16, 44])
@pytest.mark.parametrize("delta", [0, -1, 1])
def test_scan_batch_fp32_reference_recipe(S, mult, batch, delta):
    import tcuscan_ops

    L = mult * S * S + delta
    g = torch.Generator().manual_seed(L + batch)
    x = torch.rand((batch, L), generator=g)
    z = tcuscan_ops.run_scan_batch(x.to(DEV), S).cpu().numpy()
    ref = oracle.segment_scan_fixed(x.numpy().reshape(-1), L).reshape(batch, L)
    assert z.shape == (batch, L)
    assert _elementwise(z, ref) <= FP32_TOL


def test_scan_batch_golden(golden):
    import tcuscan_ops

    keys = sorted({k[:-4] for k in golden.files if k.startswith("scan_batch_") and k.endswith("_ref")})
    assert keys
    for b in keys:
        x = torch.from_numpy(golden[b + "_x"]).to(DEV)
        for S in (32, 64):
            z = tcuscan_ops.run_scan_batch(x, S).cpu().numpy()
            assert oracle.max_rel_err(z, golden[b + "_ref"]) <= 1e-3, (b, S)
            xd = golden[b + "_x"].astype(np.float64).reshape(-1)
            L = golden[b + "_x"].shape[1]
            assert _elementwise(z.reshape(-1), oracle.segment_scan_fixed(xd, L)) <= FP32_TOL, (b, S)


@pytest.mark.parametrize("dens", [0.001, 0.02])
def test_seg_scan_fp32(dens):
    import tcuscan_ops

    n = 3_000_017
    g = torch.Generator().manual_seed(5)
    x = torch.randn(n, generator=g)
    f = (torch.rand(n, generator=g) < dens).to(torch.int8)
    z = tcuscan_ops.run_seg_scan(x.to(DEV), f.to(DEV), 64).cpu().numpy()
    assert _elementwise(z, oracle.seg_scan_flags_f64(x.numpy(), f.numpy())) <= FP32_TOL


def test_scan_rows_uneven_and_graph():
    """Uneven batch (log-uniform lengths, an empty and a 1-element row) scanned
    in one launch, then replayed from a CUDA graph with new data."""
    from tcuscan_b200 import batch

    rng = np.random.default_rng(0)
    lens = np.exp(rng.uniform(np.log(256), np.log(1 << 16), size=300)).astype(np.int64)
    lens[5] = 0
    lens[17] = 1
    offsets = np.concatenate([[0], np.cumsum(lens)])
    n = int(offsets[-1])
    x = torch.from_numpy(rng.standard_normal(n).astype(np.float32))
    off_d = torch.from_numpy(offsets).to(DEV)
    z = batch.scan_rows(x.to(DEV), off_d).cpu().numpy()
    ref = oracle.scan_offsets_f64(x.numpy(), offsets)
    assert _elementwise(z, ref) <= FP32_TOL
    graph = batch.ScanRowsGraph(x.to(DEV), off_d)
    out = graph.replay().cpu().numpy()
    assert _elementwise(out, ref) <= FP32_TOL
    x2 = torch.from_numpy(rng.standard_normal(n).astype(np.float32))
    graph.x.copy_(x2.to(DEV))
    out2 = graph.replay().cpu().numpy()
    assert _elementwise(out2, oracle.scan_offsets_f64(x2.numpy(), offsets)) <= FP32_TOL
    import tcuscan_ops

    tcuscan_ops.raise_device_error(DEV)


# ---- SpMV --------------------------------------------------------------------
def _csr(nrow, ncol, density, seed, dtype):
    from scipy.sparse import random as sp_random

    rs = np.random.RandomState(seed)
    A = sp_random(nrow, ncol, density=density, format="csr", dtype=np.float64, random_state=rs,
                  data_rvs=lambda k: 2 * rs.uniform(0, 1, size=k) - 1)
    vals = A.data.astype(np.float16 if dtype == torch.float16 else np.float32)
    return vals, A.indptr.astype(np.int32), A.indices.astype(np.int32)


@pytest.mark.parametrize("s", [32, 64, 128])
@pytest.mark.parametrize("density", [0.01, 0.001, 0.0001])
@pytest.mark.parametrize("nrow", [1024, 2048, 4096, 9216, 16384])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float16])
def test_spmv_v2_reference_grid(s, density, nrow, dtype):
    import tcuscan_ops

    vals, indptr, cols = _csr(nrow - 1, nrow - 1, density, nrow, dtype)
    rng = np.random.default_rng(seed=42)
    x = rng.uniform(1, 9, nrow - 1).astype(vals.dtype)
    y = tcuscan_ops.run_spmv_v2(torch.from_numpy(vals).to(DEV), torch.from_numpy(indptr).to(DEV),
                                torch.from_numpy(cols).to(DEV), torch.from_numpy(x).to(DEV), s).cpu().numpy()
    assert y.dtype == np.float32 and y.shape == (nrow - 1,)
    ref = oracle.spmv_f64(vals, indptr, cols, x)
    assert oracle.max_rel_err(y, ref) <= 1e-3
    assert np.allclose(y, ref, atol=1e-1)


def test_spmv_golden(golden):
    import tcuscan_ops

    keys = sorted({k[:-4] for k in golden.files if k.startswith("spmv_") and k.endswith("_ref")})
    assert keys
    for b in keys:
        args = [torch.from_numpy(golden[b + k]).to(DEV) for k in ("_vals", "_indptr", "_cols", "_x")]
        y = tcuscan_ops.run_spmv_v2(*args, 64).cpu().numpy()
        assert oracle.max_rel_err(y, golden[b + "_ref"]) <= 1e-3, b


def test_spmv_variants_and_long_rows():
    """Zipf-like rows (up to 4096 nnz, some empty) through every SpMV entry point."""
    import tcuscan_ops

    rng = np.random.default_rng(1)
    rows = 20000
    lens = np.minimum(rng.zipf(1.6, size=rows), 4096).astype(np.int64)
    lens[::97] = 0
    indptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    nnz = int(indptr[-1])
    cols = rng.integers(0, 1 << 20, size=nnz).astype(np.int32)
    vals = rng.standard_normal(nnz).astype(np.float32)
    x = rng.uniform(-1, 1, 1 << 20).astype(np.float32)
    ref = oracle.spmv_f64(vals, indptr, cols, x)
    a = [torch.from_numpy(t).to(DEV) for t in (vals, indptr, cols, x)]
    ones = torch.ones(64, 64, dtype=torch.float32, device=DEV)
    for y in (tcuscan_ops.run_spmv_v2(*a, 64), tcuscan_ops.run_spmv(*a, 64),
              tcuscan_ops.run_spmv_v2_multi_cube(*a, torch.triu(ones), torch.tril(ones, -1))):
        assert oracle.max_rel_err(y.cpu().numpy(), ref) <= 1e-3
    a16 = [torch.from_numpy(vals.astype(np.float16)).to(DEV), a[1], a[2], torch.from_numpy(x.astype(np.float16)).to(DEV)]
    ref16 = oracle.spmv_f64(vals.astype(np.float16), indptr, cols, x.astype(np.float16))
    assert oracle.max_rel_err(tcuscan_ops.run_spmv_v2(*a16, 64).cpu().numpy(), ref16) <= 1e-3
    tcuscan_ops.raise_device_error(DEV)
