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
