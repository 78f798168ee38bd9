"""Pin the CPU oracle to the reference (CPU only).

tests/golden/golden.npz holds outputs of the reference's own run_scan_cpu and of
the reference test-suite oracles (see tests/golden/make_golden.py).  Every
oracle function must reproduce them: bit-exact for integer and index work, and
within a stated tolerance for floating point (the fixtures are fp32 results of
the reference; the oracle accumulates in FP64).
"""
import numpy as np
import pytest

import oracle

FP_RTOL = 1e-5  # fp32 reference vs FP64 oracle, relative to max(|ref|, 1)


def _keys(golden, prefix, suffix):
    return sorted({k[: -len(suffix)] for k in golden.files if k.startswith(prefix) and k.endswith(suffix)})


def _scan_keys(golden):
    return [b for b in _keys(golden, "scan_", "_ref") if b.split("_")[1] in ("i8", "f16", "f32")]


def test_blocked_scan_bit_exact_vs_reference_run_scan_cpu(golden):
    threads = int(golden["scan_threads"])
    bases = _scan_keys(golden)
    assert bases
    for b in bases:
        x, ref = golden[b + "_x"], golden[b + "_ref"]
        got = oracle.blocked_scan_like_reference(x.astype(np.int32) if x.dtype == np.int8 else x.astype(np.float32), threads)
        assert got.dtype == ref.dtype, b
        assert np.array_equal(got, ref), b


def test_scan_oracle_vs_reference_run_scan_cpu(golden):
    for b in _scan_keys(golden):
        x, ref = golden[b + "_x"], golden[b + "_ref"]
        got = oracle.scan(x)
        assert got.dtype == ref.dtype, b
        if x.dtype == np.int8:
            assert np.array_equal(got, ref), b
        else:
            assert oracle.max_rel_err(ref, oracle.scan_f64(x)) < FP_RTOL, b


@pytest.mark.parametrize("S", [16, 32, 64, 128])
def test_row_scan(golden, S):
    x, ref = golden[f"row_scan_{S}_x"], golden[f"row_scan_{S}_ref"]
    got = oracle.segment_scan_fixed(x.reshape(-1), S)
    assert oracle.max_rel_err(got, ref) < FP_RTOL


@pytest.mark.parametrize("S", [16, 32])
def test_block_scan(golden, S):
    x, ref = golden[f"block_scan_{S}_x"], golden[f"block_scan_{S}_ref"]
    got = oracle.segment_scan_fixed(x, S * S)
    assert oracle.max_rel_err(got, ref) < FP_RTOL


def test_complete_rows(golden):
    bases = _keys(golden, "complete_rows_", "_ref")
    assert bases
    for b in bases:
        nb, tl = (int(v) for v in b.split("_")[-2:])
        x, sums, ref = golden[b + "_x"], golden[b + "_sums"], golden[b + "_ref"]
        got = oracle.complete_rows(x, sums, tl)
        if x.dtype == np.int32:
            assert np.array_equal(got, ref), b
        else:
            assert oracle.max_rel_err(got, ref) < FP_RTOL, b


def test_complete_blocks(golden):
    bases = _keys(golden, "complete_blocks_", "_ref")
    assert bases
    for b in bases:
        x, sums, ref = golden[b + "_x"], golden[b + "_sums"], golden[b + "_ref"]
        got = oracle.complete_blocks(x, sums)
        if x.dtype == np.int32:
            assert np.array_equal(got, ref), b
        else:
            assert oracle.max_rel_err(got, ref) < FP_RTOL, b


def test_reduce_tiles(golden):
    bases = _keys(golden, "reduce_tiles_", "_ref")
    assert bases
    for b in bases:
        n, tl, nb = (int(v) for v in b.split("_")[-3:])
        x, ref = golden[b + "_x"], golden[b + "_ref"]
        got = oracle.reduce_tiles(x, tl, nb)
        if x.dtype == np.int8:
            assert np.array_equal(got, ref), b
        else:
            assert oracle.max_rel_err(got, ref) < FP_RTOL, b


def test_seg_sum_indptr(golden):
    bases = _keys(golden, "seg_sum_", "_ref")
    bases = [b for b in bases if not b.startswith("seg_sum_flags")]
    assert bases
    for b in bases:
        x, ip, ref = golden[b + "_x"], golden[b + "_indptr"], golden[b + "_ref"]
        got = oracle.seg_sum_indptr(x, ip)
        if x.dtype == np.int8:
            assert np.array_equal(got, ref), b
        else:
            assert oracle.max_rel_err(got, ref) < FP_RTOL, b


def test_seg_scan_flags(golden):
    bases = _keys(golden, "seg_scan_", "_ref")
    assert bases
    for b in bases:
        x, f, ref = golden[b + "_x"], golden[b + "_f"], golden[b + "_ref"]
        got = oracle.seg_scan_flags_f64(x, f)
        assert oracle.max_rel_err(got, ref) < FP_RTOL, b


def test_seg_sum_flags(golden):
    bases = _keys(golden, "seg_sum_flags_", "_ref")
    assert bases
    for b in bases:
        x, f, ref = golden[b + "_x"], golden[b + "_f"], golden[b + "_ref"]
        got = oracle.seg_sum_flags_f64(x, f)
        assert got.shape == ref.shape, b
        assert oracle.max_rel_err(got, ref) < FP_RTOL, b


def test_compress(golden):
    bases = _keys(golden, "compress_", "_ref")
    assert bases
    for b in bases:
        x, m, ref, refidx = golden[b + "_x"], golden[b + "_mask"], golden[b + "_ref"], golden[b + "_refidx"]
        got = oracle.compress(x, m)
        assert got.dtype == ref.dtype and np.array_equal(got, ref), b
        got2, idx2 = oracle.compress(x, m, idx_in=np.arange(x.size, dtype=np.int32))
        assert np.array_equal(got2, ref) and np.array_equal(idx2, refidx), b
        got3, idx3 = oracle.compress(x, m, want_idx=True)
        assert np.array_equal(got3, ref) and np.array_equal(idx3, refidx), b


def test_csr_gather(golden):
    bases = _keys(golden, "csr_gather_", "_ref")
    assert bases
    for b in bases:
        v, c, x, ref = golden[b + "_v"], golden[b + "_c"], golden[b + "_x"], golden[b + "_ref"]
        got = oracle.csr_gather(v, c, x)
        assert got.dtype == ref.dtype, b
        assert np.array_equal(got, ref), b


def test_spmv(golden):
    bases = _keys(golden, "spmv_", "_ref")
    assert bases
    for b in bases:
        y = oracle.spmv_f64(golden[b + "_vals"], golden[b + "_indptr"], golden[b + "_cols"], golden[b + "_x"])
        assert oracle.max_rel_err(y, golden[b + "_ref"]) < FP_RTOL, b


def test_scan_batch(golden):
    bases = _keys(golden, "scan_batch_", "_ref")
    assert bases
    for b in bases:
        x, ref = golden[b + "_x"], golden[b + "_ref"]
        L = x.shape[1]
        got = oracle.segment_scan_fixed(x.reshape(-1), L).reshape(x.shape)
        assert oracle.max_rel_err(got, ref) < FP_RTOL, b
        offs = np.arange(0, x.size + 1, L)
        got2 = oracle.scan_offsets_f64(x.reshape(-1), offs).reshape(x.shape)
        assert oracle.max_rel_err(got2, ref) < FP_RTOL, b


def test_oracle_planted_mistake_is_caught(golden):
    """A mistake planted in the oracle's output (on the CPU) must fail the pin."""
    b = "seg_sum_i8_513"
    got = oracle.seg_sum_indptr(golden[b + "_x"], golden[b + "_indptr"]).copy()
    got[7] += 1
    assert not np.array_equal(got, golden[b + "_ref"])
