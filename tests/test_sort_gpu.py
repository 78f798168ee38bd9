"""GPU parity of split, radix sort, top-k and the top-k pivot estimator
against the oracle (bit-exact values and positions).

Grids follow the reference's tests: tests/test_split.py / test_split_ind.py
(VEC_LENS, S in 32/64/128, int16 and fp16), tests/test_radix_sort.py
(_SORT_SIZES for fp16, k * 20 * 128^2 sizes for int16), tests/test_topk.py
(5 Ki .. 20 Mi elements, k = 1, 2, 5, sqrt(n)) and tests/test_topk_pivot.py
(10 * randn fp16, 10-40 Mi elements, the estimate below the 2048-th
largest).  Added: other element widths, ragged lengths, ties, NaN and +-0,
and the 2^28-element split.
"""
import math

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"

VEC_LENS = [255, 1023, 2047, 4095, 8191, 1024 * 1024 - 1, 257, 1025, 2049, 4097, 8193, 1024 * 1024 + 1,
            1024 * 1024 + 13, 1024 * 1024 + 27]


def _mask(n, seed):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(n, generator=g) > 0).to(torch.int8)


@pytest.mark.parametrize("dtype", [torch.int16, torch.float16])
@pytest.mark.parametrize("S", [32, 64, 128])
@pytest.mark.parametrize("n", VEC_LENS)
def test_split_reference_grid(dtype, S, n):
    import tcuscan_ops

    g = torch.Generator().manual_seed(n + S)
    x = torch.randint(0, 2 ** 7 - 1, (n,), generator=g).to(dtype)
    m = _mask(n, n)
    z = tcuscan_ops.run_split(x.to(DEV), m.to(DEV), S).cpu()
    assert z.dtype == dtype and np.array_equal(z.numpy(), oracle.split(x.numpy(), m.numpy()))
    ind = torch.arange(1, n + 1, dtype=torch.int32)
    zi, iz = tcuscan_ops.run_split_ind(x.to(DEV), m.to(DEV), ind.to(DEV), S)
    rz, ri = oracle.split(x.numpy(), m.numpy(), ind.numpy())
    assert np.array_equal(zi.cpu().numpy(), rz) and np.array_equal(iz.cpu().numpy(), ri)


@pytest.mark.parametrize("dtype", [torch.int8, torch.float32, torch.int32, torch.float64, torch.int64])
@pytest.mark.parametrize("n", [1, 63, 64, 65, 4096, 8191, 100_003])
@pytest.mark.parametrize("p", [0.0, 0.3, 1.0])
def test_split_widths_and_edges(dtype, n, p):
    import tcuscan_ops

    g = torch.Generator().manual_seed(n)
    x = (torch.randn(n, generator=g) * 100).to(dtype)
    m = (torch.rand(n, generator=g) < p).to(torch.int8)
    z = tcuscan_ops.run_split(x.to(DEV), m.to(DEV), 64).cpu()
    assert np.array_equal(z.numpy(), oracle.split(x.numpy(), m.numpy()))
    ind = torch.randperm(n, generator=g).to(torch.int64)
    zi, iz = tcuscan_ops.run_split_ind(x.to(DEV), m.to(DEV), ind.to(DEV), 64)
    rz, ri = oracle.split(x.numpy(), m.numpy(), ind.numpy())
    assert np.array_equal(zi.cpu().numpy(), rz) and np.array_equal(iz.cpu().numpy(), ri)


def test_split_empty():
    import tcuscan_ops

    x = torch.empty(0, dtype=torch.float16, device=DEV)
    assert tcuscan_ops.run_split(x, torch.empty(0, dtype=torch.int8, device=DEV), 64).numel() == 0


def test_split_2e28_fp16_properties():
    """Full-size split: the head is the compaction of the selected values and
    the tail the compaction of the others (both checked on the device)."""
    import tcuscan_ops

    n = 1 << 28
    g = torch.Generator(device=DEV).manual_seed(5)
    x = torch.randn(n, device=DEV, generator=g).half()
    m = (torch.rand(n, device=DEV, generator=g) < 0.3).to(torch.int8)
    z = tcuscan_ops.run_split(x, m, 128)
    k = int(m.sum())
    assert torch.equal(z[:k], torch.masked_select(x, m.bool()))
    assert torch.equal(z[k:], torch.masked_select(x, ~m.bool()))


_SORT_SIZES = [1024, 2048, 4096, 8192, 16384, 32768, 65536, 131072, 262144, 524288, 1179648, 4325376, 16908288,
               25165824]


@pytest.mark.parametrize("n", _SORT_SIZES)
def test_radix_sort_fp16_reference_sizes(n):
    import tcuscan_ops

    g = torch.Generator().manual_seed(n)
    x = torch.rand(n, generator=g).half()
    v, i = tcuscan_ops.run_radix_sort(x.to(DEV), 128)
    rv, ri = oracle.radix_sort(x.numpy(), "f")
    assert np.array_equal(v.cpu().numpy().view(np.uint16), rv.view(np.uint16))
    assert i.dtype == torch.int32 and np.array_equal(i.cpu().numpy(), ri)
    assert torch.equal(v.cpu(), torch.sort(x)[0])


@pytest.mark.parametrize("n", [20 * 128 * 128, 17 * 20 * 128 * 128, 1, 4095, 4097, 1_000_003])
def test_radix_sort_int16(n):
    import tcuscan_ops

    g = torch.Generator().manual_seed(n)
    x = torch.randint(-32768, 32767, (n,), generator=g, dtype=torch.int16)
    v, i = tcuscan_ops.run_radix_sort(x.to(DEV), 64)
    rv, ri = oracle.radix_sort(x.numpy(), "i")
    assert np.array_equal(v.cpu().numpy(), rv) and np.array_equal(i.cpu().numpy(), ri)


@pytest.mark.parametrize("dtype,kind", [(torch.int8, "i"), (torch.uint8, "u"), (torch.bfloat16, "f"),
                                        (torch.int32, "i"), (torch.float32, "f")])
@pytest.mark.parametrize("n", [1, 300, 4096, 70_001, 3_000_000])
def test_radix_sort_widths(dtype, kind, n):
    import tcuscan_ops

    g = torch.Generator().manual_seed(n)
    if dtype.is_floating_point:
        x = (torch.randn(n, generator=g) * 50).to(dtype)
    else:
        info = torch.iinfo(dtype)
        x = torch.randint(info.min, info.max, (n,), generator=g, dtype=torch.int64).to(dtype)
    v, i = tcuscan_ops.run_radix_sort(x.to(DEV), 64)
    xn = x.view(torch.int16).numpy().view(np.uint16) if dtype == torch.bfloat16 else x.numpy()
    order = np.argsort(oracle.sort_key(xn, kind), kind="stable").astype(np.int32)
    assert np.array_equal(i.cpu().numpy(), order)
    assert torch.equal(v.cpu(), x[torch.from_numpy(order).long()])


def test_radix_sort_float_specials():
    import tcuscan_ops

    vals = [0.0, -0.0, 1.0, -1.0, float("inf"), float("-inf"), float("nan"), 65504.0, -65504.0, 6e-8, -6e-8]
    x = torch.tensor(vals * 500, dtype=torch.float16)
    x[3::7] = -x[3::7]  # negative NaNs too
    v, i = tcuscan_ops.run_radix_sort(x.to(DEV), 64)
    rv, ri = oracle.radix_sort(x.numpy(), "f")
    assert np.array_equal(v.cpu().numpy().view(np.uint16), rv.view(np.uint16)) and np.array_equal(i.cpu().numpy(), ri)


_TOPK_LENS = [5 * 1024, 10 * 1024, 10 * 1024 * 1024 - 1, 20 * 1024 * 1024 - 10]


@pytest.mark.parametrize("dtype", [torch.float16, torch.int16])
@pytest.mark.parametrize("n", _TOPK_LENS)
@pytest.mark.parametrize("kk", ["1", "2", "5", "sqrt"])
def test_topk_reference_grid(dtype, n, kk):
    import tcuscan_ops

    k = int(math.sqrt(n)) if kk == "sqrt" else int(kk)
    g = torch.Generator().manual_seed(42)
    if dtype == torch.int16:
        x = torch.randint(-32768, 32767, (n,), generator=g).to(dtype)
        fn = tcuscan_ops.run_topk_int16
    else:
        x = torch.rand(n, generator=g).half()
        fn = tcuscan_ops.run_topk_fp16
    v, i = fn(x.to(DEV), k, x.min(), x.max(), 128)
    rv, ri = oracle.topk(x.numpy(), k)
    assert np.array_equal(i.cpu().numpy(), ri) and np.array_equal(v.cpu().numpy(), rv)
    tv, _ = torch.topk(x.float(), k)
    assert torch.equal(torch.sort(v.cpu().float())[0], torch.sort(tv)[0])


@pytest.mark.parametrize("n,k", [(1, 1), (7, 7), (4096, 4096), (4097, 2000), (100_000, 99_999), (300_000, 0)])
def test_topk_edges_and_ties(n, k):
    import tcuscan_ops

    g = torch.Generator().manual_seed(n + k)
    x = torch.randint(-3, 4, (n,), generator=g).to(torch.int16)  # heavy ties
    v, i = tcuscan_ops.run_topk_int16(x.to(DEV), k, -3, 3, 64)
    rv, ri = oracle.topk(x.numpy(), k)
    assert np.array_equal(i.cpu().numpy(), ri) and np.array_equal(v.cpu().numpy(), rv)
    if 0 < k and n <= 5000:
        # the literal bisection of the reference keeps the same set
        bv, bi = oracle.topk_like_reference(x.numpy(), k, -3, 3)
        assert np.array_equal(np.sort(bi), ri)


def test_topk_fp16_nan_and_signed_zero():
    import tcuscan_ops

    x = torch.zeros(10_000, dtype=torch.float16)
    x[::3] = -0.0
    x[17] = float("nan")
    x[5000] = 1.0
    x[9000] = -1.0
    v, i = tcuscan_ops.run_topk_fp16(x.to(DEV), 40, -1.0, 1.0, 64)
    rv, ri = oracle.topk(x.numpy(), 40)
    assert np.array_equal(i.cpu().numpy(), ri)
    assert ri[0] == 0 and 17 in ri and 5000 in ri  # NaN and 1.0 first, then the lowest-positioned zeros


def test_topk_rejects():
    import tcuscan_ops

    x = torch.zeros(10, dtype=torch.float16, device=DEV)
    with pytest.raises(ValueError):
        tcuscan_ops.run_topk_fp16(x, 11, 0, 0, 64)
    with pytest.raises(TypeError):
        tcuscan_ops.run_topk_int16(x, 1, 0, 0, 64)


@pytest.mark.parametrize("n", [10 * 1024 * 1024, 20 * 1024 * 1024, 40 * 1024 * 1024])
def test_topk_pivot_reference(n):
    import tcuscan_ops

    g = torch.Generator().manual_seed(42)
    x = (10 * torch.randn(n, generator=g)).half()
    est = tcuscan_ops.run_topk_pivot_fp16(x.to(DEV), 8).cpu()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    ref = oracle.topk_pivot(x.numpy(), blocks=sms)
    assert np.array_equal(est.numpy().view(np.uint16), ref.view(np.uint16))
    kth = torch.topk(x.float(), 2048)[0][-1]
    assert kth > est.float().max()


@pytest.mark.parametrize("n,ns", [(1000, 32), (5000, 4), (70_000, 33), (1 << 20, 16)])
def test_topk_pivot_small_and_ragged(n, ns):
    import tcuscan_ops

    g = torch.Generator().manual_seed(n)
    x = torch.randn(n, generator=g).half()
    est = tcuscan_ops.run_topk_pivot_fp16(x.to(DEV), 8, ns).cpu()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    ref = oracle.topk_pivot(x.numpy(), num_samples=ns, blocks=sms)
    assert np.array_equal(est.numpy().view(np.uint16), ref.view(np.uint16))
