"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark configurations (no datasets ship with this project; these stand in
for the reference's SuiteSparse matrices and measurement inputs).

- ``scan_input``   1-D scans: int8 uniform in [-8, 8] or float16 uniform[-1, 1).
- ``bernoulli_mask`` int8 compaction masks, P(1) = p.
- ``zipf_csr``     CSR matrix, row lengths Zipf(alpha) clipped to
                   [1, max_len] and rescaled so nnz ~= target_nnz, columns
                   uniform and sorted within each row, values N(0, 1),
                   x uniform[-1, 1).
- ``uneven_rows``  row offsets with log-uniform lengths in [lo, hi].
"""
import math

import numpy as np
import torch


def scan_input(n, dtype, device, seed=0):
    g = torch.Generator(device=device).manual_seed(seed)
    if dtype == torch.int8:
        return torch.randint(-8, 9, (n,), dtype=torch.int8, device=device, generator=g)
    return (torch.rand(n, device=device, generator=g) * 2 - 1).to(dtype)


def bernoulli_mask(n, p, device, seed=0):
    g = torch.Generator(device=device).manual_seed(seed)
    return (torch.rand(n, device=device, generator=g) < p).to(torch.int8)


def zipf_row_lengths(rows, alpha=1.6, max_len=4096, target_nnz=1 << 24, seed=0):
    rng = np.random.default_rng(seed)
    lens = np.minimum(rng.zipf(alpha, size=rows), max_len).astype(np.float64)
    lens = np.clip(np.rint(lens * (target_nnz / lens.sum())), 1, max_len).astype(np.int64)
    return lens


def zipf_csr(rows=1 << 20, cols=1 << 20, alpha=1.6, max_len=4096, target_nnz=1 << 24, dtype=torch.float32,
             device="cuda", seed=0):
    """Returns (vals, indptr int32, cols int32, x) on `device`."""
    lens = zipf_row_lengths(rows, alpha, max_len, target_nnz, seed)
    indptr = np.zeros(rows + 1, dtype=np.int64)
    np.cumsum(lens, out=indptr[1:])
    nnz = int(indptr[-1])
    g = torch.Generator(device=device).manual_seed(seed + 1)
    col = torch.randint(0, cols, (nnz,), dtype=torch.int32, device=device, generator=g)
    # sort columns within each row: key = row * cols + col
    row_of = torch.repeat_interleave(torch.arange(rows, device=device, dtype=torch.int64),
                                     torch.from_numpy(lens).to(device))
    col = (row_of * cols + col.long()).sort().values.remainder(cols).to(torch.int32)
    vals = torch.randn(nnz, device=device, generator=g).to(dtype)
    x = (torch.rand(cols, device=device, generator=g) * 2 - 1).to(dtype)
    return vals, torch.from_numpy(indptr.astype(np.int32)).to(device), col, x


def uneven_rows(nrows=4096, lo=256, hi=1 << 20, seed=0):
    """int64 offsets [nrows + 1] of rows with log-uniform lengths in [lo, hi]."""
    rng = np.random.default_rng(seed)
    lens = np.exp(rng.uniform(math.log(lo), math.log(hi), size=nrows)).astype(np.int64)
    offsets = np.zeros(nrows + 1, dtype=np.int64)
    np.cumsum(lens, out=offsets[1:])
    return offsets


class ServedStream:
    """The served request stream: `count` requests, op mix 50% scan / 30%
    indptr seg_sum / 20% compress, dtypes 40% int8 / 40% float16 / 20%
    float32, sizes log-uniform in [lo, hi] elements, seg_sum segment lengths
    geometric with mean 64, compress masks Bernoulli(0.3).

    Request data are views into seeded device pools (one value pool per
    dtype, one mask pool) at random 16-element-aligned offsets; the row
    pointers of all seg_sum requests are built on the device in one int32
    array.  ``arrays()`` gives the request table for
    ``Server.submit_many``; ``request(i)`` gives (op, x, aux) tensors for the
    one-call loop."""

    def __init__(self, count=20000, device="cuda", seed=0, lo=1 << 10, hi=1 << 24, mean_seg=64):
        from tcuscan_b200 import serve

        rng = np.random.default_rng(seed)
        dev = torch.device(device)
        self.count = count
        self.op = rng.choice(3, size=count, p=[0.5, 0.3, 0.2]).astype(np.int8)
        self.dt = rng.choice(3, size=count, p=[0.4, 0.4, 0.2]).astype(np.int8)  # int8, float16, float32
        self.n = np.exp(rng.uniform(math.log(lo), math.log(hi), size=count)).astype(np.int64)
        psize = hi + (1 << 20)
        self.pools = []
        for i, dt in enumerate(serve.DTYPES):
            self.pools.append(scan_input(psize, dt, dev, seed=seed + 1 + i))
        self.mask_pool = bernoulli_mask(psize, 0.3, dev, seed=seed + 7)
        self.off = (rng.integers(0, (psize - self.n) // 16) * 16).astype(np.int64)
        self.moff = (rng.integers(0, (psize - self.n) // 16) * 16).astype(np.int64)
        eb = np.array([1, 2, 4], dtype=np.int64)
        base = np.array([p.data_ptr() for p in self.pools], dtype=np.uint64)
        self.xp = base[self.dt] + (self.off * eb[self.dt]).astype(np.uint64)
        self.ap = np.zeros(count, dtype=np.uint64)
        self.nseg = np.zeros(count, dtype=np.int64)
        self.iw = np.zeros(count, dtype=np.int8)
        cm = self.op == serve.COMPRESS
        self.ap[cm] = np.uint64(self.mask_pool.data_ptr()) + self.moff[cm].astype(np.uint64)
        # row pointers of every seg_sum request: segment starts are the
        # points of one geometric stream laid over the requests' elements
        sm = np.nonzero(self.op == serve.SEG_SUM)[0]
        self.ioff = np.zeros(count, dtype=np.int64)
        if sm.size:
            ns = torch.from_numpy(self.n[sm]).to(dev)
            vb = torch.cumsum(ns, 0) - ns  # virtual base of each request
            vtot = int(ns.sum())
            g = torch.Generator(device=dev).manual_seed(seed + 11)
            m = int(vtot / mean_seg * 1.02) + 1024
            steps = torch.empty(m, device=dev).geometric_(1.0 / mean_seg, generator=g).to(torch.int64)
            pts = torch.cumsum(steps, 0)
            pts = pts[pts < vtot]
            req = torch.searchsorted(vb, pts, right=True) - 1
            inner = pts != vb[req]  # a point on a request boundary is that request's start
            pts, req = pts[inner], req[inner]
            k = torch.bincount(req, minlength=sm.size)
            width = k + 2
            ooff = torch.cumsum(width, 0) - width
            kstart = torch.cumsum(k, 0) - k
            rank = torch.arange(pts.numel(), device=dev) - kstart[req]
            ip = torch.empty(int(width.sum()), dtype=torch.int32, device=dev)
            ip[ooff] = 0
            ip[ooff + k + 1] = ns.to(torch.int32)
            ip[ooff[req] + 1 + rank] = (pts - vb[req]).to(torch.int32)
            self.indptr = ip
            self.ioff[sm] = ooff.cpu().numpy()
            self.nseg[sm] = k.cpu().numpy() + 1
            self.iw[sm] = 4
            self.ap[sm] = np.uint64(ip.data_ptr()) + (self.ioff[sm] * 4).astype(np.uint64)
            del steps, pts, req, inner, rank
        else:
            self.indptr = torch.zeros(1, dtype=torch.int32, device=dev)

    def arrays(self, idx=None):
        s = slice(None) if idx is None else idx
        return (self.op[s], self.dt[s], self.n[s], self.xp[s], self.ap[s], self.nseg[s], self.iw[s])

    def request(self, i):
        from tcuscan_b200 import serve

        op, dt, n = int(self.op[i]), int(self.dt[i]), int(self.n[i])
        x = self.pools[dt][self.off[i]: self.off[i] + n]
        aux = None
        if op == serve.SEG_SUM:
            aux = self.indptr[self.ioff[i]: self.ioff[i] + self.nseg[i] + 1]
        elif op == serve.COMPRESS:
            aux = self.mask_pool[self.moff[i]: self.moff[i] + n]
        return op, x, aux

    def element_bytes(self):
        """Algorithmic bytes of every request (inputs read once, outputs written once)."""
        eb = np.array([1, 2, 4], dtype=np.int64)[self.dt]
        ob = np.where(self.dt == 0, 4, 4)
        scan = self.n * (eb + ob)
        seg = self.n * eb + (self.nseg + 1) * 4 + self.nseg * 4
        comp = self.n * (eb + 1) + (0.3 * self.n).astype(np.int64) * eb
        return np.where(self.op == 0, scan, np.where(self.op == 1, seg, comp))
