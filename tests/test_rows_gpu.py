"""GPU parity of the two segment-sum / SpMV paths: the SIMT row kernels
(tcu_seg_sum_rows / tcu_spmv_rows, taken for short segments) and the
tensor-core segmented sum (tcu_seg_bounds / tcu_spmv_csr, long segments).
Every case runs through both by moving the dispatch threshold.

Tolerances: int8 sums bit-exact (int32); fp16 sums and SpMV
|err| <= 1e-3 * max(|ref|, 1) against the FP64 oracle (the SIMT path sums in
FP32 and is far inside it; the tensor-core path splits products into bf16
hi + lo).  Cases follow the reference's seg_sum grid (tests/test_seg_sum_multi_core.py:
row counts, columns around S^2) and the SpMV config (Zipf(1.6) rows up to
4096 long), plus empty rows, a leading non-zero bound, int32 / uint32 /
int64 indptr, rows of many 32-element steps and out-of-range columns.
"""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.fixture(params=["rows", "tensor"])
def path(request, monkeypatch):
    import tcuscan_ops

    monkeypatch.setattr(tcuscan_ops, "ROWS_MAX_MEAN", 1 << 40 if request.param == "rows" else -1)
    monkeypatch.setattr(tcuscan_ops, "ROWS_FP32", request.param == "rows")
    return request.param


def _rel(got, ref):
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    return float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1.0))) if ref.size else 0.0


def _indptr(lengths):
    return np.concatenate([[0], np.cumsum(lengths)]).astype(np.int64)


@pytest.mark.parametrize("dtype", [torch.float16, torch.int8, torch.float32])
@pytest.mark.parametrize("rows,mean", [(1, 5), (31, 3), (33, 40), (513, 16), (2011, 64), (20_000, 7), (300, 3000)])
def test_seg_sum_paths(path, dtype, rows, mean):
    import tcuscan_ops

    rng = np.random.default_rng(rows * 7 + mean)
    lengths = rng.geometric(1.0 / mean, rows) - 1  # includes empty rows
    ip = _indptr(lengths)
    n = int(ip[-1])
    if dtype == torch.int8:
        x = torch.from_numpy(rng.integers(-128, 127, n).astype(np.int8))
    else:
        x = torch.from_numpy(rng.uniform(-1, 1, n).astype(np.float32)).to(dtype)
    out = tcuscan_ops.run_seg_sum_multi_core(x.to(DEV), torch.from_numpy(ip).to(DEV), 64).cpu().numpy()
    tcuscan_ops.raise_device_error(DEV)
    ref = oracle.seg_sum_indptr(x.numpy(), ip)
    if dtype == torch.int8:
        assert out.dtype == np.int32 and np.array_equal(out, ref)
    else:
        assert out.dtype == np.float32 and _rel(out, ref) <= 1e-3


@pytest.mark.parametrize("idx_dtype", [torch.int32, torch.int64, "uint32"])
def test_seg_sum_index_types_and_offset_start(path, idx_dtype):
    import tcuscan_ops

    rng = np.random.default_rng(3)
    n = 50_000
    x = torch.from_numpy(rng.uniform(-1, 1, n).astype(np.float16))
    ip = np.sort(rng.integers(1000, n, 4001))  # first bound past 0; repeated bounds = empty rows
    if idx_dtype == "uint32":
        ipt = torch.from_numpy(ip.astype(np.uint32)) if hasattr(torch, "uint32") else torch.from_numpy(ip.astype(np.int32))
    else:
        ipt = torch.from_numpy(ip).to(idx_dtype)
    out = tcuscan_ops.run_seg_sum_multi_core(x.to(DEV), ipt.to(DEV), 32).cpu().numpy()
    ref = np.array([x.numpy()[ip[k]:ip[k + 1]].astype(np.float64).sum() for k in range(ip.size - 1)])
    assert _rel(out, ref) <= 1e-3


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16])
@pytest.mark.parametrize("rows,nnz_target", [(1, 100), (100, 5000), (1 << 14, 1 << 18), (1 << 20, 1 << 24)])
def test_spmv_paths(path, dtype, rows, nnz_target):
    import tcuscan_ops
    from tcuscan_b200 import workloads

    if rows == 1 << 20:
        vals, indptr, cols, xs = workloads.zipf_csr(dtype=dtype, device=DEV, seed=9)
    else:
        vals, indptr, cols, xs = workloads.zipf_csr(rows=rows, cols=max(rows, 64), target_nnz=nnz_target, dtype=dtype,
                                                    device=DEV, seed=rows)
    y = tcuscan_ops.run_spmv_v2(vals, indptr, cols, xs, 64).cpu().numpy()
    tcuscan_ops.raise_device_error(DEV)
    ref = oracle.spmv_f64(vals.cpu().float().numpy(), indptr.cpu().numpy(), cols.cpu().numpy(), xs.cpu().float().numpy())
    assert _rel(y, ref) <= 1e-3


def test_spmv_rows_is_fp32_accurate(monkeypatch):
    """The SIMT path sums fp32 products in FP32: error ~1e-6 relative."""
    import tcuscan_ops
    from tcuscan_b200 import workloads

    monkeypatch.setattr(tcuscan_ops, "ROWS_MAX_MEAN", 1 << 40)

    vals, indptr, cols, xs = workloads.zipf_csr(rows=1 << 16, cols=1 << 16, target_nnz=1 << 20, dtype=torch.float32,
                                                device=DEV, seed=4)
    y = tcuscan_ops.run_spmv_v2(vals, indptr, cols, xs, 64).cpu().numpy()
    ref = oracle.spmv_f64(vals.cpu().numpy(), indptr.cpu().numpy(), cols.cpu().numpy(), xs.cpu().numpy())
    assert _rel(y, ref) <= 2e-5


def test_spmv_rows_deterministic(monkeypatch):
    """The element-split path sums every row in a fixed order: bitwise equal
    results on repeated calls.  (The tensor-core path adds its FP64 look-back
    carries in the order predecessors publish, so its float results may
    differ in the last bit between runs.)"""
    import tcuscan_ops
    from tcuscan_b200 import workloads

    monkeypatch.setattr(tcuscan_ops, "ROWS_MAX_MEAN", 1 << 40)

    vals, indptr, cols, xs = workloads.zipf_csr(rows=1 << 15, cols=1 << 15, target_nnz=1 << 20, dtype=torch.float32,
                                                device=DEV, seed=5)
    a = tcuscan_ops.run_spmv_v2(vals, indptr, cols, xs, 64)
    b = tcuscan_ops.run_spmv_v2(vals, indptr, cols, xs, 64)
    assert torch.equal(a, b)


def test_spmv_rows_out_of_range_column_recorded(monkeypatch):
    import tcuscan_ops

    monkeypatch.setattr(tcuscan_ops, "ROWS_MAX_MEAN", 1 << 40)

    vals = torch.ones(40, device=DEV)
    cols = torch.zeros(40, dtype=torch.int32, device=DEV)
    cols[7] = 1000  # x has 16 entries
    indptr = torch.tensor([0, 10, 40], dtype=torch.int32, device=DEV)
    xs = torch.ones(16, device=DEV)
    y = tcuscan_ops.run_spmv_v2(vals, indptr, cols, xs, 64)
    assert y.tolist() == [9.0, 30.0]
    code, site, chunk = tcuscan_ops.workspace_error(DEV)
    assert code != 0 and site == 301 and chunk == 7
