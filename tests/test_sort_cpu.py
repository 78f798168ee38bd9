"""The split / radix-sort / top-k oracles pinned on CPU against the oracles of
the reference's own tests: torch.masked_select (tests/test_split.py:48-57,
tests/test_split_ind.py:49-70), torch.sort (tests/test_radix_sort.py:66-82)
and torch.topk (tests/test_topk.py:39-61), plus the literal restatements of
the reference's algorithms (sixteen one-bit splits; bisection over the value
range) against the direct forms the GPU tests use."""
import numpy as np
import pytest
import torch

import oracle


def _int16(rng, n):
    return rng.integers(-32768, 32767, n).astype(np.int16)


@pytest.mark.parametrize("n", [255, 1023, 4097, 8193])
def test_split_oracle_vs_masked_select(n):
    rng = np.random.default_rng(n)
    x = rng.integers(0, 127, n).astype(np.int16)
    m = (rng.standard_normal(n) > 0).astype(np.int8)
    ind = np.arange(1, n + 1, dtype=np.int32)
    z, iz = oracle.split(x, m, ind)
    xt, mt = torch.from_numpy(x), torch.from_numpy(m)
    k = int(m.sum())
    assert np.array_equal(z[:k], torch.masked_select(xt, mt == 1).numpy())
    assert np.array_equal(z[k:], torch.masked_select(xt, mt == 0).numpy())
    assert np.array_equal(iz[:k], (torch.nonzero(mt == 1, as_tuple=True)[0] + 1).int().numpy())
    assert np.array_equal(iz[k:], (torch.nonzero(mt == 0, as_tuple=True)[0] + 1).int().numpy())


@pytest.mark.parametrize("dtype", [np.int16, np.float16])
@pytest.mark.parametrize("n", [1024, 5000, 65536])
def test_radix_sort_restatement(dtype, n):
    rng = np.random.default_rng(n)
    x = _int16(rng, n) if dtype == np.int16 else rng.standard_normal(n).astype(np.float16)
    v1, i1 = oracle.radix_sort(x, "i" if dtype == np.int16 else "f")
    v2, i2 = oracle.radix_sort_like_reference(x)
    assert np.array_equal(v1.view(np.uint16), v2.view(np.uint16)) and np.array_equal(i1, i2)
    tv, ti = torch.sort(torch.from_numpy(x), stable=True)
    assert np.array_equal(tv.numpy(), v1) and np.array_equal(ti.numpy(), i1)


def test_radix_sort_float_encoding_edges():
    x = np.array([0.0, -0.0, 1.0, -1.0, np.inf, -np.inf, 65504, -65504, 6e-8, -6e-8], dtype=np.float16)
    v, i = oracle.radix_sort(x, "f")
    assert np.array_equal(i, [5, 7, 3, 9, 1, 0, 8, 2, 6, 4])  # -0 below +0
    v2, i2 = oracle.radix_sort_like_reference(x)
    assert np.array_equal(i, i2)


@pytest.mark.parametrize("kind,dtype", [("i", np.int8), ("u", np.uint8), ("i", np.int32), ("f", np.float32)])
def test_radix_sort_other_widths(kind, dtype):
    rng = np.random.default_rng(3)
    if dtype == np.float32:
        x = rng.standard_normal(3000).astype(dtype)
    else:
        info = np.iinfo(dtype)
        x = rng.integers(info.min, info.max, 3000, dtype=np.int64).astype(dtype)
    v, i = oracle.radix_sort(x, kind)
    tv, ti = torch.sort(torch.from_numpy(x.astype(np.int64) if dtype == np.uint8 else x), stable=True)
    assert np.array_equal(v.astype(np.float64), tv.numpy().astype(np.float64)) and np.array_equal(i, ti.numpy())


@pytest.mark.parametrize("dtype", [np.int16, np.float16])
@pytest.mark.parametrize("n,k", [(5 * 1024, 1), (5 * 1024, 2), (10 * 1024, 5), (10 * 1024, 101), (4000, 4000),
                                 (30000, 173)])
def test_topk_restatement_and_torch(dtype, n, k):
    rng = np.random.default_rng(n + k)
    x = _int16(rng, n) if dtype == np.int16 else rng.random(n).astype(np.float16)
    v, i = oracle.topk(x, k)
    assert np.array_equal(np.sort(i), i) and np.array_equal(x[i], v)
    rv, ri = oracle.topk_like_reference(x, k, x.min(), x.max())
    o = np.argsort(ri, kind="stable")
    assert np.array_equal(rv[o].view(np.uint16), v.view(np.uint16)) and np.array_equal(ri[o], i)
    tv, _ = torch.topk(torch.from_numpy(x).float(), k)
    assert np.array_equal(np.sort(tv.numpy()), np.sort(v.astype(np.float32)))


def test_topk_ties_keep_lowest_positions():
    x = np.array([3, 1, 3, 2, 3, 3, 0], dtype=np.int16)
    v, i = oracle.topk(x, 3)
    assert np.array_equal(i, [0, 2, 4]) and np.array_equal(v, [3, 3, 3])
    rv, ri = oracle.topk_like_reference(x, 3, 0, 3)
    assert np.array_equal(np.sort(ri), i)
    v, i = oracle.topk(x, 5)
    assert np.array_equal(i, [0, 2, 3, 4, 5])


def test_topk_pivot_is_lower_bound():
    rng = np.random.default_rng(7)
    x = (10 * rng.standard_normal(1 << 21)).astype(np.float16)
    est = oracle.topk_pivot(x, blocks=148)
    assert est.size == 148
    assert np.sort(x)[-2048] > est.max()
