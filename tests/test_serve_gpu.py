"""GPU tests of the serving loop and of the device steps it batches with.

- tcu_pack: every request's elements land at its offset, padding is zero,
  row pointers are widened and rebased exactly.
- tcu_compress_segments: the batched compaction equals the per-request
  compactions (bit-exact), with each request's output offset.
- Server: a mixed stream of scan / seg_sum / compress requests (int8, fp16,
  fp32; sizes log-uniform; segment lengths geometric with mean 64) gives, for
  every request, the same result in the mix as alone and as the single
  drop-in call: int8 bit-exact, floating results within 1e-3 relative to
  max(|ref|, 1) of the FP64 oracle; admission never exceeds the budget.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL = 1e-3


def _lib():
    from tcuscan_ops import _lib as L

    return L


def _items(rows):
    from tcuscan_b200 import serve

    a = np.zeros(len(rows), dtype=serve.PACK_ITEM)
    for i, (src, dst, n, ln, add) in enumerate(rows):
        a[i] = (src, dst, n, ln, add)
    return torch.from_numpy(a.view(np.uint8)).to(DEV)


@pytest.mark.parametrize("dtype", [torch.int8, torch.float16, torch.float32, torch.int64])
def test_pack_copies_and_pads(dtype):
    L = _lib()
    rng = np.random.default_rng(1)
    g = torch.Generator(device=DEV).manual_seed(2)
    pool = torch.randint(-100, 100, (1 << 16,), device=DEV, generator=g).to(dtype)
    eb = pool.element_size()
    rows, expect, dst = [], [], 0
    for k in range(40):
        n = int(rng.integers(1, 3000))
        off = int(rng.integers(0, (1 << 16) - n))  # any alignment, vector and scalar paths
        ln = n + int(rng.integers(0, 300))
        rows.append((pool.data_ptr() + off * eb, dst, n, ln, 0))
        expect.append(torch.cat([pool[off:off + n], torch.zeros(ln - n, dtype=dtype, device=DEV)]))
        dst += ln
    out = torch.full((dst,), 7, dtype=dtype, device=DEV)
    it = _items(rows)
    st = L.lib.tcu_pack(it.data_ptr(), len(rows), eb, eb, out.data_ptr(), dst,
                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    assert torch.equal(out, torch.cat(expect))


@pytest.mark.parametrize("src_dtype", [torch.int32, torch.int64])
def test_pack_rebases_row_pointers(src_dtype):
    L = _lib()
    rng = np.random.default_rng(3)
    rows, expect, dst, keep = [], [], 0, []
    for k in range(25):
        ip = np.concatenate([[0], np.cumsum(rng.geometric(1 / 64, size=int(rng.integers(0, 200))))])
        t = torch.from_numpy(ip).to(src_dtype).to(DEV)
        keep.append(t)
        base = int(rng.integers(0, 1 << 40)) if src_dtype == torch.int64 else int(rng.integers(0, 1 << 30))
        rows.append((t.data_ptr(), dst, t.numel(), t.numel(), base))
        expect.append(torch.from_numpy(ip.astype(np.int64) + base))
        dst += t.numel()
    out = torch.empty(dst, dtype=torch.int64, device=DEV)
    it = _items(rows)
    st = L.lib.tcu_pack(it.data_ptr(), len(rows), keep[0].element_size(), 8, out.data_ptr(), dst,
                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    assert torch.equal(out.cpu(), torch.cat(expect))


@pytest.mark.parametrize("dtype", [torch.int8, torch.float16, torch.float32])
def test_compress_segments_matches_per_request(dtype):
    L = _lib()
    rng = np.random.default_rng(4)
    sizes = [int(v) for v in np.exp(rng.uniform(np.log(1), np.log(200_000), size=30))]
    starts, xs, ms, pos = [], [], [], 0
    for n in sizes:
        starts.append(pos)
        x = torch.from_numpy(rng.integers(-50, 50, size=n)).to(dtype)
        m = torch.from_numpy((rng.random(n) < 0.3).astype(np.int8))
        pad = (-n) % 256
        xs.append(torch.cat([x, torch.zeros(pad, dtype=dtype)]))
        ms.append(torch.cat([m, torch.zeros(pad, dtype=torch.int8)]))
        pos += n + pad
    x = torch.cat(xs).to(DEV)
    m = torch.cat(ms).to(DEV)
    st_d = torch.tensor(starts, dtype=torch.int64, device=DEV)
    out = torch.empty(pos, dtype=dtype, device=DEV)
    sp = torch.empty(len(starts) + 1, dtype=torch.int64, device=DEV)
    ws, wsb = L.workspace(torch.device(DEV), L.lib.tcu_workspace_bytes(pos, 64))
    st = L.lib.tcu_compress_segments(x.data_ptr(), x.element_size(), m.data_ptr(), pos, st_d.data_ptr(), len(starts),
                                     out.data_ptr(), pos, sp.data_ptr(), ws, wsb,
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    spc = sp.cpu().numpy()
    xc, mc = x.cpu().numpy(), m.cpu().numpy()
    for i, s in enumerate(starts):
        e = s + sizes[i]
        ref = oracle.compress(xc[s:e], mc[s:e])
        got = out[spc[i]:spc[i + 1]].cpu().numpy()
        assert spc[i + 1] - spc[i] == ref.size
        assert np.array_equal(got, ref), i
    assert spc[-1] == int((mc != 0).sum())


# ---- the serving loop ----------------------------------------------------------
def _mixed_requests(count, seed, max_log2=18):
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=DEV).manual_seed(seed)
    reqs = []
    for i in range(count):
        op = ["scan", "seg_sum", "compress"][int(rng.choice(3, p=[0.5, 0.3, 0.2]))]
        dt = [torch.float16, torch.int8, torch.float32][int(rng.choice(3, p=[0.4, 0.4, 0.2]))]
        n = int(np.exp(rng.uniform(np.log(2 ** 10), np.log(2 ** max_log2))))
        if dt == torch.int8:
            x = torch.randint(-8, 9, (n,), dtype=torch.int8, device=DEV, generator=g)
        else:
            x = (torch.rand(n, device=DEV, generator=g) * 2 - 1).to(dt)
        aux = None
        if op == "seg_sum":
            cuts = np.cumsum(rng.geometric(1 / 64, size=n // 32 + 2))
            ip = np.concatenate([[0], cuts[cuts < n], [n]]).astype(np.int32)
            aux = torch.from_numpy(ip).to(DEV)
        elif op == "compress":
            aux = (torch.rand(n, device=DEV, generator=g) < 0.3).to(torch.int8)
        reqs.append((op, x, aux))
    return reqs


def _oracle(op, x, aux):
    xc = x.cpu().numpy()
    if op == "scan":
        r = oracle.scan_f64(xc.astype(np.float64), 0.0)
        return r
    if op == "seg_sum":
        return oracle.seg_sum_indptr(xc, aux.cpu().numpy().astype(np.int64))
    return oracle.compress(xc, aux.cpu().numpy())


def _close(got, ref, exact):
    got = np.asarray(got)
    if exact:
        return np.array_equal(got.astype(np.int64), np.asarray(ref).astype(np.int64))
    return oracle.max_rel_err(got, ref) <= TOL


def test_server_mix_equals_alone_and_oracle():
    import tcuscan_ops
    from tcuscan_b200 import serve

    reqs = _mixed_requests(120, 5)
    srv = serve.Server(DEV, budget_bytes=1 << 30, slots=3, max_batch=48, keep_results=True)
    ids = [srv.submit(op, x, aux) for op, x, aux in reqs]
    srv.run()
    assert srv.peak_used <= srv.budget
    assert srv.batches < len(reqs)  # requests were batched
    for rid, (op, x, aux) in zip(ids, reqs):
        mix = srv.result(rid).cpu()
        exact = x.dtype == torch.int8 or op == "compress"
        if op == "scan" and x.dtype == torch.int8:
            ref = torch.cumsum(x.cpu().long(), 0).int().numpy()
        else:
            ref = _oracle(op, x, aux)
        assert mix.shape[0] == np.asarray(ref).shape[0], (rid, op)
        assert _close(mix.numpy(), ref, exact), (rid, op, x.dtype)
        # alone: a server holding only this request, and the single drop-in call
        one = serve.Server(DEV, budget_bytes=1 << 30, slots=1, keep_results=True)
        r1 = one.submit(op, x, aux)
        one.run()
        alone = one.result(r1).cpu()
        S = tcuscan_ops._pick_S(None, x.dtype, x.numel())
        if op == "scan":
            single = tcuscan_ops.run_scan_multi_core(x, S).cpu()
        elif op == "seg_sum":
            single = tcuscan_ops.run_seg_sum_multi_core(x, aux, S).cpu()
        else:
            single = tcuscan_ops.run_compress(x, aux, S).cpu()
        if exact:
            assert torch.equal(mix, alone) and torch.equal(mix, single), (rid, op)
        else:
            d = (mix.double() - alone.double()).abs().max().item() if mix.numel() else 0.0
            assert d <= TOL * max(1.0, alone.double().abs().max().item() if alone.numel() else 1.0)
            assert _close(single.numpy(), ref, False)
        one.release()
    srv.release()
    assert srv.used == 0
    tcuscan_ops.raise_device_error(DEV)


def test_server_in_place_requests(monkeypatch):
    """Scan / seg_sum requests at or above SOLO_MIN run the single-call kernel
    on their own inputs (no pack copy), beside packed requests of the same
    batch: every result equals the oracle (integers bit for bit) and the
    single drop-in call."""
    import tcuscan_ops
    from tcuscan_b200 import serve

    monkeypatch.setattr(serve, "SOLO_MIN", 1 << 12)
    reqs = _mixed_requests(48, 11, max_log2=15)
    srv = serve.Server(DEV, budget_bytes=1 << 30, slots=2, max_batch=24, keep_results=True)
    ids = [srv.submit(op, x, aux) for op, x, aux in reqs]
    srv.run()
    n_solo = sum(1 for op, x, _ in reqs if op != "compress" and x.numel() >= (1 << 12))
    assert 0 < n_solo < len(reqs)
    for rid, (op, x, aux) in zip(ids, reqs):
        got = srv.result(rid).cpu()
        exact = x.dtype == torch.int8 or op == "compress"
        if op == "scan" and x.dtype == torch.int8:
            ref = torch.cumsum(x.cpu().long(), 0).int().numpy()
        else:
            ref = _oracle(op, x, aux)
        assert got.shape[0] == np.asarray(ref).shape[0], (rid, op)
        assert _close(got.numpy(), ref, exact), (rid, op, x.dtype)
        if op == "scan" and x.numel() >= (1 << 12):  # in place: the single call's own kernel
            single = tcuscan_ops.run_scan_multi_core(x, tcuscan_ops._pick_S(None, x.dtype, x.numel())).cpu()
            if exact:
                assert torch.equal(got, single), rid
            else:  # only the order of the FP64 tile carries may differ
                d = (got.double() - single.double()).abs().max().item()
                assert d <= TOL * max(1.0, single.double().abs().max().item()), rid
        elif op == "seg_sum" and x.numel() >= (1 << 12):
            single = tcuscan_ops.run_seg_sum_multi_core(x, aux, 64).cpu()
            assert torch.equal(got, single), rid
    srv.release()
    tcuscan_ops.raise_device_error(DEV)


def test_server_budget_admission_and_arrivals():
    from tcuscan_b200 import serve

    reqs = _mixed_requests(60, 7, max_log2=16)
    budget = 6 << 20
    srv = serve.Server(DEV, budget_bytes=budget, slots=4, max_batch=8)
    arrivals = np.cumsum(np.random.default_rng(8).exponential(2e-4, size=len(reqs)))
    srv.mark_start()
    for (op, x, aux), t in zip(reqs, arrivals):
        srv.submit(op, x, aux, arrival=float(t))
    srv.run()
    assert srv.peak_used <= budget
    lat = srv.latencies()
    assert np.all(np.isfinite(lat)) and np.all(lat >= 0)
    assert np.all(srv.admit[: len(reqs)] >= srv.arrival[: len(reqs)])
    big = torch.zeros(4 << 20, dtype=torch.float32, device=DEV)
    s2 = serve.Server(DEV, budget_bytes=4 << 20, slots=1)
    s2.submit("scan", big)
    with pytest.raises(MemoryError):
        s2.run()
