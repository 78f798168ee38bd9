"""Autotuner for the tile parameters of the tensor-core scan family.

The reference fixes S per call (the caller passes it; tests sweep 16..128).
Here a caller may pass S=None (or 0) and the drop-in picks S -- and the
number of CTAs of the persistent launch -- from a table measured on the
device by ``tune()``:

    op        what is timed                               tuned over
    scan      tcuscan_ops.run_scan_multi_core              S (int8: 32/64/128,
                                                           fp16: 16..128), CTAs
    seg       batched uneven rows (sorted segment starts)  S (32/64), CTAs
    compress  tcuscan_ops.run_compress_pos                 CTAs

Entries are keyed by op, dtype and floor(log2(n)); lookups use the nearest
tuned size of the same op and dtype.  The table is JSON (``TCU_AUTOTUNE_CACHE``
or ``autotune.json`` next to this file) and records the device it was measured
on.  Without a table the defaults below apply (the fastest S measured on B200
at n = 2^28, one CTA per SM).
"""
import json
import math
import os

import torch

DTYPES = (torch.int8, torch.float16, torch.float32)
VALID_S = {
    ("scan", torch.int8): (32, 64, 128),
    ("scan", torch.float16): (16, 32, 64, 128),
    ("scan", torch.float32): (64,),
    ("seg", torch.int8): (32, 64),
    ("seg", torch.float16): (32, 64),
    ("seg", torch.float32): (64,),
    ("compress", torch.int8): (64,),
    ("compress", torch.float16): (64,),
    ("compress", torch.float32): (64,),
}
_DEFAULTS = {
    ("scan", torch.int8): 128,
    ("scan", torch.float16): 64,
    ("scan", torch.float32): 64,
}
CACHE = os.environ.get("TCU_AUTOTUNE_CACHE", os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotune.json"))
_table = None
_ctas_now = 0
_best_cache = {}  # (op, dtype, floor(log2 n)) -> (S, ctas): lookups on every call stay cheap


def _dname(dtype):
    return str(dtype).replace("torch.", "")


def _key(op, dtype, n):
    b = int(math.log2(max(int(n), 1)))
    return f"{op}/{_dname(dtype)}/{b}"


def _load():
    global _table
    if _table is None:
        _table = {}
        if os.environ.get("TCU_AUTOTUNE", "1") != "0" and os.path.exists(CACHE):
            try:
                with open(CACHE) as fh:
                    _table = json.load(fh).get("entries", {})
            except (OSError, ValueError, AttributeError):
                _table = {}
    return _table


def reload(path=None):
    """Drop the cached table (and read `path` instead of the default)."""
    global _table, CACHE
    if path is not None:
        CACHE = path
    _table = None
    _best_cache.clear()


def best(op, dtype, n=None):
    """(S, ctas) for a call; ctas 0 means one CTA per SM."""
    default = (_DEFAULTS.get((op, dtype), 64), 0)
    if n is None:
        return default
    ck = (op, dtype, max(int(n), 1).bit_length() - 1)
    hit = _best_cache.get(ck)
    if hit is not None:
        return hit
    r = _best_lookup(op, dtype, n, default)
    _best_cache[ck] = r
    return r


def _best_lookup(op, dtype, n, default):
    tab = _load()
    if not tab:
        return default
    e = tab.get(_key(op, dtype, n))
    if e is None:  # nearest tuned size of this op and dtype
        prefix = f"{op}/{_dname(dtype)}/"
        sizes = [int(k[len(prefix):]) for k in tab if k.startswith(prefix)]
        if not sizes:
            return default
        b = int(math.log2(max(int(n), 1)))
        e = tab[prefix + str(min(sizes, key=lambda s: abs(s - b)))]
    return int(e.get("S", default[0])), int(e.get("ctas", 0))


def best_S(op, dtype, n=None):
    return best(op, dtype, n)[0]


def apply_ctas(ctas):
    """Set the library's CTA cap (only when it changes)."""
    global _ctas_now
    ctas = int(ctas or 0)
    if ctas != _ctas_now:
        from tcuscan_ops import _lib

        _lib.lib.tcu_set_max_ctas(ctas)
        _ctas_now = ctas


def _device_timer(fn, steps, warmup):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        fn()
    b.record()
    b.synchronize()
    return a.elapsed_time(b) / steps


def _workload(op, dtype, n, device):
    """A callable fn(S) running one call of `op` on seeded data of size n."""
    import tcuscan_ops
    from tcuscan_b200 import batch, workloads

    if op == "scan":
        x = workloads.scan_input(n, dtype, device, seed=1)
        return lambda S: tcuscan_ops.run_scan_multi_core(x, S)
    if op == "seg":
        x = workloads.scan_input(n, dtype, device, seed=2)
        offs = torch.from_numpy(workloads.uneven_rows(nrows=max(n // 65536, 1), lo=256, hi=1 << 17, seed=3))
        offs = (offs * n // int(offs[-1])).to(device)
        return lambda S: batch.scan_rows(x, offs, S)
    if op == "compress":
        x = workloads.scan_input(n, dtype, device, seed=4)
        m = workloads.bernoulli_mask(n, 0.3, device, seed=5)
        k = int(m.sum().item())
        return lambda S: tcuscan_ops.run_compress_pos(x, m, k, S)
    raise ValueError(op)


def tune(device=None, ops=("scan", "seg", "compress"), dtypes=DTYPES, log2_sizes=(16, 20, 24, 28),
         cta_fracs=(1.0, 0.75, 0.5), steps=10, warmup=3, path=None, timer=None, workload=None, write=True):
    """Measure every (S, CTA count) candidate per op, dtype and size, keep the
    fastest, and write the table.  `timer(fn, steps, warmup) -> ms` and
    `workload(op, dtype, n, device) -> fn(S)` can be replaced (tests)."""
    device = torch.device(device or "cuda")
    timer = timer or _device_timer
    workload = workload or _workload
    if device.type == "cuda":
        sms = torch.cuda.get_device_properties(device).multi_processor_count
        name = torch.cuda.get_device_name(device)
    else:
        sms, name = 148, "unknown"
    ctas_opts = sorted({0 if f >= 1.0 else max(1, int(sms * f)) for f in cta_fracs})
    entries = {}
    try:
        for op in ops:
            for dtype in dtypes:
                for b in log2_sizes:
                    n = 1 << int(b)
                    fn = workload(op, dtype, n, device)
                    timings = {}
                    for S in VALID_S[(op, dtype)]:
                        for c in ctas_opts:
                            apply_ctas(c)
                            timings[f"S={S},ctas={c}"] = float(timer(lambda: fn(S), steps, warmup))
                    best_k = min(timings, key=timings.get)
                    S_best = int(best_k.split(",")[0][2:])
                    c_best = int(best_k.split("ctas=")[1])
                    entries[f"{op}/{_dname(dtype)}/{b}"] = {"S": S_best, "ctas": c_best, "ms": timings[best_k],
                                                            "timings_ms": timings}
                    del fn
    finally:
        apply_ctas(0)
    table = {"device": name, "sms": sms, "entries": entries}
    if write:
        path = path or CACHE
        with open(path, "w") as fh:
            json.dump(table, fh, indent=1, sort_keys=True)
        reload(path)
    return table


if __name__ == "__main__":  # python -m tcuscan_b200.autotune [--out PATH] [--sizes 16,20,24,28]
    import argparse

    ap = argparse.ArgumentParser(description="measure and write the tile-parameter table")
    ap.add_argument("--out", default=CACHE)
    ap.add_argument("--sizes", default="16,20,24,28")
    ap.add_argument("--ops", default="scan,seg,compress")
    a = ap.parse_args()
    t = tune(ops=tuple(a.ops.split(",")), log2_sizes=tuple(int(v) for v in a.sizes.split(",")), path=a.out)
    for k, v in sorted(t["entries"].items()):
        print(f"{k:24s} S={v['S']:<4d} ctas={v['ctas']:<4d} {v['ms'] * 1e3:10.1f} us")
