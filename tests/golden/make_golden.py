"""Generate the golden fixtures that pin the oracle to the reference.

Run in the development container, where the reference checkout exists:

    OMP_NUM_THREADS=4 python tests/golden/make_golden.py [--ref /path/to/reference]

(the checkout is found as in oracle/build_ref.py: --ref, $TCUSCAN_REFERENCE,
or a ``reference`` directory next to this repository)

Two sources of expected outputs, both the reference's own code:

1. ``run_scan_cpu`` from src/torch/torch_scan_cpu.h, compiled unmodified into
   oracle/_ref by oracle/build_ref.py (scan fixtures, int8 / fp16 / fp32).
2. The reference test-suite oracles, executed from the reference's test files
   (their function definitions are extracted with ``ast`` and run on CPU
   tensors): ref_segsum (tests/test_segmented_sum.py), ref_segscan
   (tests/test_seg_scan_single_core.py), ref_complete_rows
   (tests/test_complete_rows.py), ref_complete_blocks
   (tests/test_complete_blocks.py), ref_reduce_tiles
   (tests/test_reduce_tiles.py), ref_csr_gather (tests/test_csr_gather.py),
   plus the expressions the tests compare against inline: torch.cumsum
   (test_scan_multi_core.py / test_scan_batch.py), F.linear(A, tril)
   (test_row_scan.py), A @ triu (test_block_scan.py), scipy ``A @ ones``
   (test_seg_sum_multi_core.py), torch.masked_select (test_compress*.py),
   scipy ``B @ vector`` (test_spmv_v2.py), torch.tril (test_gen_lower.py).

Inputs follow each test's own recipe (value ranges, seeds 42) at small sizes
so the fixtures stay a few hundred KB.  The fixtures travel with the repo, so
running the tests never needs the reference checkout.
"""
import argparse
import ast
import os
import sys
from math import ceil

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _extract(ref_root, test_file, names, extra_ns):
    """Execute the named top-level function definitions of a reference test file."""
    path = os.path.join(ref_root, "tests", test_file)
    with open(path) as fh:
        tree = ast.parse(fh.read(), filename=path)
    keep = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names]
    missing = set(names) - {n.name for n in keep}
    if missing:
        raise RuntimeError(f"{test_file}: functions not found: {missing}")
    mod = ast.Module(body=keep, type_ignores=[])
    ns = dict(extra_ns)
    exec(compile(mod, path, "exec"), ns)
    return [ns[n] for n in names]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    args = ap.parse_args()

    import torch
    import torch.nn.functional as F
    from scipy.sparse import random as sp_random

    sys.path.insert(0, REPO)
    from oracle import build_ref

    args.ref = build_ref.reference_root(args.ref)
    if args.ref is None:
        raise SystemExit("reference checkout not found (pass --ref or set TCUSCAN_REFERENCE)")

    # The reference oracles call .npu(); on CPU that is the identity.
    torch.Tensor.npu = lambda self, *a, **k: self
    import numpy.typing as npt

    ns = {"torch": torch, "np": np, "npt": npt, "ceil": ceil, "NPU_DEVICE": "cpu"}

    (ref_segsum,) = _extract(args.ref, "test_segmented_sum.py", ["ref_segsum"], ns)
    (ref_segscan,) = _extract(args.ref, "test_seg_scan_single_core.py", ["ref_segscan"], ns)
    (ref_complete_rows,) = _extract(args.ref, "test_complete_rows.py", ["ref_complete_rows"], ns)
    (ref_complete_blocks,) = _extract(args.ref, "test_complete_blocks.py", ["ref_complete_blocks"], ns)
    (ref_reduce_tiles,) = _extract(args.ref, "test_reduce_tiles.py", ["ref_reduce_tiles"], ns)
    (ref_csr_gather,) = _extract(args.ref, "test_csr_gather.py", ["ref_csr_gather"], ns)

    ref = build_ref.load_module()
    threads = int(ref.omp_max_threads())
    out = {}

    torch.manual_seed(42)
    np.random.seed(42)

    # 1. run_scan_cpu (reference CPU scan) -- test_scan_cpu.py input recipe.
    for n in (1, 1024 + 13, 5 * 1024, 16384 - 7):
        for name, x in (
            ("i8", torch.randint(0, 10, size=(n,), dtype=torch.int8)),
            ("f16", (0.1 * torch.randn(n)).half()),
            ("f32", 0.1 * torch.randn(n, dtype=torch.float32)),
        ):
            out[f"scan_{name}_{n}_x"] = x.numpy()
            out[f"scan_{name}_{n}_ref"] = ref.run_scan_cpu(x).numpy()
    out["scan_threads"] = np.array(threads)

    # 2. row scan (test_row_scan.py:34-40) and block scan (test_block_scan.py:28-38).
    for S in (16, 32, 64, 128):
        m = 2 * 128 - 5
        A = torch.randn(m, S).half()
        B = torch.tril(torch.ones((S, S)))
        out[f"row_scan_{S}_x"] = A.numpy()
        out[f"row_scan_{S}_ref"] = F.linear(A.float(), B).flatten().numpy()
    for S in (16, 32):
        m = 11
        A = (0.1 * torch.randn(m, S * S)).half()
        Bt = torch.triu(torch.ones((S * S, S * S)))
        out[f"block_scan_{S}_x"] = A.flatten().numpy()
        out[f"block_scan_{S}_ref"] = torch.matmul(A.float(), Bt).flatten().numpy()

    # 3. complete_rows / complete_blocks / reduce_tiles (reference oracles).
    for nb, tl in ((2, 32), (10, 32), (3, 64)):
        vec_len = nb * tl * tl * 3
        x = 0.1 * torch.randn(vec_len).float()
        sums = torch.sum(x.reshape(nb, -1), dim=1, dtype=torch.float32).flatten()
        out[f"complete_rows_f32_{nb}_{tl}_x"] = x.numpy()
        out[f"complete_rows_f32_{nb}_{tl}_sums"] = sums.numpy()
        out[f"complete_rows_f32_{nb}_{tl}_ref"] = ref_complete_rows(x.clone(), sums, tl, nb).numpy()
        xi = torch.randint(-3, 3, size=(vec_len,), dtype=torch.int32)
        si = torch.sum(xi.reshape(nb, -1), dim=1, dtype=torch.int32).flatten()
        out[f"complete_rows_i32_{nb}_{tl}_x"] = xi.numpy()
        out[f"complete_rows_i32_{nb}_{tl}_sums"] = si.numpy()
        out[f"complete_rows_i32_{nb}_{tl}_ref"] = ref_complete_rows(xi.clone(), si, tl, nb).numpy()
    for nb, S in ((2, 32), (10, 32), (3, 64)):
        vec_len = nb * S * S * 3
        x = 0.1 * torch.randn(vec_len).float()
        sums = torch.sum(x.reshape(nb, -1), dim=1, dtype=torch.float32).flatten()
        out[f"complete_blocks_f32_{nb}_{S}_x"] = x.numpy()
        out[f"complete_blocks_f32_{nb}_{S}_sums"] = sums.numpy()
        out[f"complete_blocks_f32_{nb}_{S}_ref"] = ref_complete_blocks(x.clone(), sums, nb).numpy()
        xi = torch.randint(0, 3, size=(vec_len,), dtype=torch.int32)
        si = torch.sum(xi.reshape(nb, -1), dim=1, dtype=torch.int32).flatten()
        out[f"complete_blocks_i32_{nb}_{S}_x"] = xi.numpy()
        out[f"complete_blocks_i32_{nb}_{S}_sums"] = si.numpy()
        out[f"complete_blocks_i32_{nb}_{S}_ref"] = ref_complete_blocks(xi.clone(), si, nb).numpy()
    for n, tl, nb in ((40 * 16 * 16 - 11, 128, 40), (40 * 32 * 32 + 17, 512, 40), (5000, 128, 7)):
        xh = (0.1 * torch.randn(n)).half()
        out[f"reduce_tiles_f16_{n}_{tl}_{nb}_x"] = xh.numpy()
        out[f"reduce_tiles_f16_{n}_{tl}_{nb}_ref"] = ref_reduce_tiles(xh.float(), torch.float32, tl, nb).numpy()
        xi = torch.randint(-3, 3, size=(n,), dtype=torch.int8)
        out[f"reduce_tiles_i8_{n}_{tl}_{nb}_x"] = xi.numpy()
        out[f"reduce_tiles_i8_{n}_{tl}_{nb}_ref"] = ref_reduce_tiles(xi.int(), torch.int32, tl, nb).numpy()

    # 4. indptr seg_sum: scipy A @ ones (test_seg_sum_multi_core.py:82-97).
    for rows, cols in ((513, 64 * 64 - 1), (1025, 64 * 64 + 13)):
        for dt in ("f16", "i8"):
            spd = np.float32 if dt == "f16" else np.int32
            rvs = (lambda k: (0.5 * np.random.uniform(0, 1, size=k) - 0.25)) if dt == "f16" else (
                lambda k: np.random.randint(-2, 2, size=k))
            A = sp_random(rows, cols, density=0.01, format="csr", dtype=spd, data_rvs=rvs)
            vals = A.data.astype(np.float16 if dt == "f16" else np.int8)
            A.data = vals.astype(spd)
            out[f"seg_sum_{dt}_{rows}_x"] = vals
            out[f"seg_sum_{dt}_{rows}_indptr"] = A.indptr.astype(np.int32)
            out[f"seg_sum_{dt}_{rows}_ref"] = (A @ np.ones(cols, dtype=spd)).astype(spd)

    # 5. flag seg-scan (starts) and flag seg-sum (ends), reference oracles.
    for n, dens in ((32 * 32 * 3, 0.01), (64 * 64 * 2, 0.05), (4096, 0.0)):
        rng = np.random.default_rng(seed=42)
        x = torch.Tensor(rng.integers(0, 10, n).astype(np.float16)).half()
        f = (torch.empty(n).uniform_(0, 1) < dens).to(torch.int8)
        out[f"seg_scan_{n}_{dens}_x"] = x.numpy()
        out[f"seg_scan_{n}_{dens}_f"] = f.numpy()
        out[f"seg_scan_{n}_{dens}_ref"] = ref_segscan(x.float(), f).numpy()
    for n in (20 * 32 * 32, 2 * 20 * 32 * 32):
        x = torch.randint(-2, 2, size=(n,)).half()
        f = (torch.rand(n) < 0.01).to(torch.int8)
        f[0] = 0
        f_ends = torch.concat([f[1:], torch.ones(1, dtype=torch.int8)]).contiguous()
        out[f"seg_sum_flags_{n}_x"] = x.numpy()
        out[f"seg_sum_flags_{n}_f"] = f_ends.numpy()
        out[f"seg_sum_flags_{n}_ref"] = ref_segsum(x, f).numpy()

    # 6. compress / compress_ind / no_arange: torch.masked_select.
    for n in (20 * 32 * 32 - 13, 20 * 32 * 32 + 129):
        for dt, tdt in (("f16", torch.float16), ("f32", torch.float32), ("i16", torch.int16)):
            x = torch.randint(0, 2**7 - 1, (n,)).to(tdt)
            mask = (torch.randn(n) > 0).to(torch.int8)
            idx = torch.arange(0, n, dtype=torch.int32)
            out[f"compress_{dt}_{n}_x"] = x.numpy()
            out[f"compress_{dt}_{n}_mask"] = mask.numpy()
            out[f"compress_{dt}_{n}_ref"] = torch.masked_select(x, mask.to(torch.bool)).numpy()
            out[f"compress_{dt}_{n}_refidx"] = torch.masked_select(idx, mask.to(torch.bool)).numpy()

    # 7. csr_gather: values * x[cols] (tests/test_csr_gather.py:60-61).
    for col_len, x_len in ((16 * 1024, 256), (20 * 1024 - 13, 20000)):
        for dt, tdt in (("f16", torch.float16), ("f32", torch.float32), ("i16", torch.int16)):
            if tdt == torch.int16:
                v = torch.randint(-300, 300, (col_len,), dtype=tdt)
                xx = torch.randint(-300, 300, (x_len,), dtype=tdt)
            else:
                v = torch.randn(col_len).to(tdt)
                xx = torch.randn(x_len).to(tdt)
            c = torch.randint(low=0, high=x_len, size=(col_len,), dtype=torch.int32)
            out[f"csr_gather_{dt}_{col_len}_v"] = v.numpy()
            out[f"csr_gather_{dt}_{col_len}_c"] = c.numpy()
            out[f"csr_gather_{dt}_{col_len}_x"] = xx.numpy()
            out[f"csr_gather_{dt}_{col_len}_ref"] = ref_csr_gather(v, c, xx).numpy()

    # 8. SpMV: scipy B @ vector (tests/test_spmv_v2.py:59-98), fp32 recipe.
    rng = np.random.default_rng(seed=42)
    for nrow, dens in ((1024, 0.01), (2048, 0.001)):
        B = sp_random(nrow - 1, nrow - 1, density=dens, format="csr", dtype=np.float32,
                      data_rvs=lambda k: 2 * np.random.uniform(0, 1, size=k) - 1)
        vec = rng.uniform(1, 9, nrow - 1).astype(np.float32)
        out[f"spmv_{nrow}_vals"] = B.data.astype(np.float32)
        out[f"spmv_{nrow}_indptr"] = B.indptr.astype(np.int32)
        out[f"spmv_{nrow}_cols"] = B.indices.astype(np.int32)
        out[f"spmv_{nrow}_x"] = vec
        out[f"spmv_{nrow}_ref"] = B @ vec

    # 9. scan_batch: torch.cumsum(x, dim=1) (tests/test_scan_batch.py:47-50).
    for bs, L in ((16, 32 * 32 + 1), (20, 64 * 64 // 4)):
        x = torch.rand((bs, L), dtype=torch.float32)
        out[f"scan_batch_{bs}_{L}_x"] = x.numpy()
        out[f"scan_batch_{bs}_{L}_ref"] = torch.cumsum(x, dim=1, dtype=torch.float).numpy()

    # 10. gen_lower: torch.tril(ones) (tests/test_gen_lower.py).
    for s in (32, 128):
        out[f"gen_lower_{s}_ref"] = torch.tril(torch.ones((s, s), dtype=torch.int8)).numpy()

    path = os.path.join(HERE, "golden.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path) / 1024:.1f} KiB, threads={threads}")


if __name__ == "__main__":
    main()
