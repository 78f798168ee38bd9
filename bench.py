"""Benchmark of the tensor-core scan family on B200 (one JSON line on rank 0).

Headline workload: int8 1-D inclusive scan, n = 2^28 -> int32 (S autotuned:
128), one persistent tcgen05 launch per step.  ``value`` is whole-job
elements/s with the input resident in HBM (device time, CUDA events, max over
ranks); ``e2e`` is the same metric through the host-buffer scan
(``tcuscan_b200.stream``: the input copied from pinned host memory and the
full result read back every step, chunk by chunk on three streams so the two
copy directions and the scans overlap).  The input (256 MiB) and output
(1 GiB) are larger than L2 (126 MB), so no explicit flush is needed between
steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--op scan_i8|scan_f16]
    python bench.py --impl reference ...   # the reference CPU scan on host cores

Multi-GPU (torchrun): replicas only -- every rank scans its own array; the
path has no exchange step, so no collective is issued (scaling = weak).

Output: the other configured workloads in full detail on one JSON line
(``{"extras": ...}``), then the headline line, which carries a compact
``legs`` summary of the same workloads (value, time, HBM fraction, error).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "pytorch-tcuscan_b200")
for _p in (REPO, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "elem/s & %HBM peak, TC scan at 2^28; served p50/p99+req/s vs one-call loop"
SPEC_HBM_GBS = 8000.0
FALLBACK_HBM_GBS = 6650.0

OPS = {
    # op: (input dtype name, bytes per element read+written, description)
    "scan_i8": ("int8", 5, "int8 inclusive scan n=2^28 -> int32"),
    "scan_f16": ("float16", 6, "fp16 inclusive scan n=2^28 -> fp32"),
}


def measured_peak():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def profile_traffic(op):
    """DRAM bytes per launch from the committed ncu summary (profiles/), or None."""
    p = os.path.join(REPO, "profiles", f"{op}_traffic.txt")
    try:
        with open(p) as fh:
            for line in fh:
                if line.startswith("dram_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 20 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id):
        self.bus_id = bus_id
        self.samples = []
        self.proc = None
        self.t = None

    def start(self):
        try:
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "20"]
            if self.bus_id:
                cmd += ["-i", self.bus_id]
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [s.strip() for s in line.split(",")]
            if len(parts) >= 9:
                self.samples.append((time.time(), parts))

    def wait_for(self, t, timeout=3.0):
        """Wait (bounded) until a sample taken at or after wall time t arrives:
        nvidia-smi needs about a second before its first line."""
        end = time.time() + timeout
        while time.time() < end and self.proc is not None:
            if self.samples and self.samples[-1][0] >= t:
                return True
            time.sleep(0.01)
        return False

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, t0, t1):
        rows = [p for (t, p) in self.samples if t0 - 0.15 <= t <= t1 + 0.15] or [p for (_, p) in self.samples]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}

        def num(v):
            try:
                return float(v)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": num(rows[0][2]),
            "power_w_max": max((num(r[3]) or 0.0) for r in rows),
            "reasons": sorted(reasons),
            "samples": len(rows),
        }


def _device_ms(fn, steps, warmup):
    """Average device time per call of fn() (CUDA events on the current stream)."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(steps):
        fn()
    b.record(st)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps


def measure_extras(dev, steps=10, warmup=3):
    """The other configured workloads, device-timed (inputs resident in HBM,
    all larger than L2): fp16 scan at 2^28, compaction at 2^28 with a
    Bernoulli(0.3) mask, CSR SpMV on a 2^20 x 2^20 Zipf(1.6) matrix with
    ~2^24 nnz, and 4096 uneven fp32 rows (log-uniform 256..2^20) scanned by
    one CUDA-graph launch.  Errors are measured against FP64 on the device."""
    import torch

    import tcuscan_ops
    from tcuscan_b200 import batch, workloads

    peak, _ = measured_peak()
    out = {}

    def entry(elems, bytes_, ms, unit="elem/s", **kw):
        gbs = bytes_ / (ms * 1e-3) / 1e9
        d = {"value": elems / (ms * 1e-3), "unit": unit, "ms": ms, "GB/s": gbs, "hbm_frac": gbs / peak,
             "algorithmic_bytes": bytes_}
        d.update(kw)
        return d

    n = 1 << 28
    # fp16 scan, 2^28 -> fp32
    x = workloads.scan_input(n, torch.float16, dev, seed=7)
    S16 = tcuscan_ops._pick_S(None, torch.float16, n)
    ms = _device_ms(lambda: tcuscan_ops.run_scan_multi_core(x, S16), steps, warmup)
    z = tcuscan_ops.run_scan_multi_core(x, S16)
    ref = torch.cumsum(x.double(), 0)
    err = ((z.double() - ref).abs() / ref.abs().clamp_min(1.0)).max().item()
    out["scan_f16_2e28"] = entry(n, 6 * n, ms, S=S16, max_rel_err_vs_fp64=err)
    del x, z, ref

    # compaction, 2^28, mask Bernoulli(0.3): one single-pass kernel per step
    mask = workloads.bernoulli_mask(n, 0.3, dev, seed=8)
    k = int(mask.sum().item())
    mb = mask.bool()
    for name, dt in (("compress_f16", torch.float16), ("compress_i16", torch.int16), ("compress_f32", torch.float32)):
        xv = torch.randint(-1000, 1000, (n,), device=dev).to(dt)
        ms = _device_ms(lambda: tcuscan_ops.run_compress_pos(xv, mask, k, 64), steps, warmup)
        exact = bool(torch.equal(tcuscan_ops.run_compress_pos(xv, mask, k, 64), torch.masked_select(xv, mb)))
        eb = xv.element_size()
        out[name] = entry(n, n * (eb + 1) + k * eb, ms, selected=k, exact_vs_masked_select=exact,
                          max_rel_err_vs_fp64=0.0 if exact else None)
        del xv
    del mb
    xv = torch.randn(n, device=dev).half()
    ms = _device_ms(lambda: tcuscan_ops.run_compress_ind_no_arange(xv, mask, 64), 3, 1)
    out["compress_ind_no_arange_f16_incl_count_sync"] = entry(n, n * 3 + k * 6, ms, selected=k)
    ar = torch.arange(n, dtype=torch.int32, device=dev)
    ms = _device_ms(lambda: tcuscan_ops.run_compress_ind(xv, ar, mask, 64), 3, 1)
    out["compress_ind_f16_arange_incl_count_sync"] = entry(n, n * 7 + k * 6, ms, selected=k)
    # split (stable partition) of the same values: reads x and the mask, writes n
    ms = _device_ms(lambda: tcuscan_ops.run_split(xv, mask, 64), steps, warmup)
    out["split_f16_2e28"] = entry(n, n * 5, ms, selected=k)
    del xv, mask, ar

    # radix sort (values + int32 positions): the reference's largest sort size
    # and 2^28; algorithmic bytes = read 2 B, write 2 + 4 B per element
    for name, ns in (("radix_sort_f16_25165824", 25165824), ("radix_sort_f16_2e28", n)):
        xs = torch.rand(ns, device=dev).half()
        ms = _device_ms(lambda: tcuscan_ops.run_radix_sort(xs, 128), steps, warmup)
        out[name] = entry(ns, ns * 8, ms)
        del xs
    # top-k, fp16 U[0,1), n = 20 Mi - 10, k = sqrt(n) (the reference's largest
    # top-k test); algorithmic bytes = one read of x
    nt = 20 * 1024 * 1024 - 10
    xt = torch.rand(nt, device=dev).half()
    kt = int(nt ** 0.5)
    ms = _device_ms(lambda: tcuscan_ops.run_topk_fp16(xt, kt, 0.0, 1.0, 128), steps, warmup)
    out["topk_f16_20Mi_ksqrt"] = entry(nt, nt * 2, ms, k=kt)
    del xt

    # block scan (every S*S tile scanned), fp16, 2^26 elements, S = 128: the
    # reference's tensor-only formulation (three products per 128-row block,
    # tcu_block_scan_tensor, run_block_scan's path) against the scan engine's
    # block mode (one product, exact shuffle row offsets, tcu_block_scan)
    from tcuscan_ops import _lib as L

    nb = 1 << 26
    xb = workloads.scan_input(nb, torch.float16, dev, seed=14)
    ones = torch.ones(128, 128, dtype=torch.float16, device=dev)
    up, lo = torch.triu(ones), torch.tril(ones, -1)
    ms_t = _device_ms(lambda: tcuscan_ops.run_block_scan(xb, up, lo), steps, warmup)
    zt = tcuscan_ops.run_block_scan(xb, up, lo)
    zb = torch.empty(nb, dtype=torch.float32, device=dev)
    ws, wsb, sp = L.launch_context(dev, L.lib.tcu_workspace_bytes(nb, 128))

    def engine_block():
        tcuscan_ops.check(L.lib.tcu_block_scan(xb.data_ptr(), L.TCU_FLOAT16, nb, 128, zb.data_ptr(), ws, wsb, sp),
                          "tcu_block_scan")
    ms_e = _device_ms(engine_block, steps, warmup)
    engine_block()
    refb = torch.cumsum(xb.double().reshape(-1, 128 * 128), 1).reshape(-1)
    err_t = ((zt.double() - refb).abs() / refb.abs().clamp_min(1.0)).max().item()
    err_e = ((zb.double() - refb).abs() / refb.abs().clamp_min(1.0)).max().item()
    out["block_scan_f16_2e26_tensor_only"] = entry(nb, 6 * nb, ms_t, S=128, max_rel_err_vs_fp64=err_t,
                                                   kernel="block_scan_tc_kernel (A.U + L.(A.J))")
    out["block_scan_f16_2e26_engine"] = entry(nb, 6 * nb, ms_e, S=128, max_rel_err_vs_fp64=err_e,
                                              kernel="scan_tc_kernel kScanBlocks (A.U, shuffle offsets)")
    del xb, zt, zb, refb

    # flag-driven segmented scan (starts), fp16 2^28, flags Bernoulli(0.01)
    xf = workloads.scan_input(n, torch.float16, dev, seed=12)
    fl = workloads.bernoulli_mask(n, 0.01, dev, seed=13)
    ms = _device_ms(lambda: tcuscan_ops.run_seg_scan(xf, fl, 64), steps, warmup)
    zf = tcuscan_ops.run_seg_scan(xf, fl, 64)
    # FP64 reference: cumsum minus the cumsum just before each element's segment start
    cs = torch.cumsum(xf.double(), 0)
    sid = torch.cumsum(fl.long(), 0)  # segment index of every element (0 = before the first start)
    starts = torch.nonzero(fl).flatten()
    base = torch.cat([torch.zeros(1, dtype=torch.float64, device=dev),
                      torch.where(starts > 0, cs[(starts - 1).clamp_min(0)], torch.zeros_like(cs[:1]))])
    ref = cs - base[sid]
    err = ((zf.double() - ref).abs() / ref.abs().clamp_min(1.0)).max().item()
    out["seg_scan_flags_f16_2e28"] = entry(n, n * (2 + 1 + 4), ms, max_rel_err_vs_fp64=err)
    del xf, fl, zf, cs, sid, starts, base, ref

    # per-segment sums (run_seg_sum_multi_core), fp16 2^28, int64 CSR-style
    # bounds with geometric segment lengths of mean 64 and mean 4
    xs16 = workloads.scan_input(n, torch.float16, dev, seed=14)
    cs = torch.cumsum(xs16.double(), 0)
    for mean in (64, 4):
        g = torch.Generator(device=dev).manual_seed(15 + mean)
        stp = torch.empty(n // mean + 4096, device=dev).geometric_(1.0 / mean, generator=g).to(torch.int64)
        pts = torch.cumsum(stp, 0)
        bnd = torch.cat([torch.zeros(1, dtype=torch.int64, device=dev), pts[pts < n],
                         torch.full((1,), n, dtype=torch.int64, device=dev)])
        del stp, pts
        ms = _device_ms(lambda: tcuscan_ops.run_seg_sum_multi_core(xs16, bnd, 64), steps, warmup)
        ys = tcuscan_ops.run_seg_sum_multi_core(xs16, bnd, 64)
        hi = cs[bnd[1:] - 1]
        lo = torch.where(bnd[:-1] > 0, cs[(bnd[:-1] - 1).clamp_min(0)], torch.zeros_like(hi))
        refs = hi - lo
        err = ((ys.double() - refs).abs() / refs.abs().clamp_min(1.0)).max().item()
        nseg = bnd.numel() - 1
        out[f"seg_sum_f16_2e28_mean{mean}"] = entry(n, n * 2 + (nseg + 1) * 8 + nseg * 4, ms, segments=nseg,
                                                    max_rel_err_vs_fp64=err)
        del bnd, ys, hi, lo, refs
    del xs16, cs

    # CSR SpMV (products + indptr segment sums)
    for name, dt in (("spmv_f32", torch.float32), ("spmv_f16", torch.float16)):
        vals, indptr, cols, xs = workloads.zipf_csr(dtype=dt, device=dev, seed=9)
        nnz, rows = vals.numel(), indptr.numel() - 1
        ms = _device_ms(lambda: tcuscan_ops.run_spmv_v2(vals, indptr, cols, xs, 64), steps, warmup)
        y = tcuscan_ops.run_spmv_v2(vals, indptr, cols, xs, 64)
        try:  # FP64 reference on the device: per-row sums of the exact products
            prod = vals.double() * xs.double()[cols.long()]
            rowid = torch.repeat_interleave(torch.arange(rows, device=dev), (indptr[1:] - indptr[:-1]).long())
            yr = torch.zeros(rows, dtype=torch.float64, device=dev).index_add_(0, rowid, prod)
            err = ((y.double() - yr).abs() / yr.abs().clamp_min(1.0)).max().item()
            del prod, rowid, yr
        except RuntimeError as e:  # pragma: no cover - diagnostics only
            err = f"unmeasured: {e}"[:120]
        eb = vals.element_size()
        bytes_ = nnz * (eb + 4) + (rows + 1) * 4 + rows * 4 + xs.numel() * eb
        out[name] = entry(nnz, bytes_, ms, unit="nnz/s", rows=rows, nnz=nnz, max_rel_err_vs_fp64=err,
                          kernels=2)
        if dt == torch.float32:  # the segment sums alone, on fp32 products with the same row pointers
            prod = (vals * xs[cols.long()]).contiguous()
            ms = _device_ms(lambda: tcuscan_ops.run_seg_sum_multi_core(prod, indptr, 64), steps, warmup)
            out["seg_sum_f32_spmv_rows"] = entry(nnz, nnz * 4 + (rows + 1) * 4 + rows * 4, ms, unit="nnz/s",
                                                 rows=rows)
            del prod
        del vals, indptr, cols, xs, y

    # 4096 uneven fp32 rows, one CUDA-graph launch
    offs = workloads.uneven_rows(seed=10)
    tot = int(offs[-1])
    xr = torch.randn(tot, device=dev)
    od = torch.from_numpy(offs).to(dev)
    gph = batch.ScanRowsGraph(xr, od)
    ms = _device_ms(gph.replay, max(3, steps // 2), 2)
    zr = gph.replay()
    seg_start = torch.repeat_interleave(od[:-1], (od[1:] - od[:-1]))
    cs = torch.cumsum(xr.double(), 0)
    base = torch.where(seg_start > 0, cs[(seg_start - 1).clamp_min(0)], torch.zeros_like(cs))
    refr = cs - base
    err_norm = ((zr.double() - refr).abs().max() / refr.abs().max().clamp_min(1.0)).item()
    err_el = ((zr.double() - refr).abs() / refr.abs().clamp_min(1.0)).max().item()
    out["batch_rows_f32_4096"] = entry(tot, tot * 8 + offs.size * 8, ms, rows=4096,
                                       normwise_rel_err_vs_fp64=err_norm, max_rel_err_vs_fp64=err_el,
                                       launch="one CUDA-graph replay per step")
    del xr, zr, cs, base, refr, seg_start

    # small fp16 scan (n = 2^20, S = 64, values uniform[-1, 1)): latency-bound;
    # one call end to end on the host (launch included) and the kernel alone
    # replayed from a CUDA graph
    import time as _t

    n20 = 1 << 20
    x20 = workloads.scan_input(n20, torch.float16, dev, seed=0)
    for _ in range(20):
        tcuscan_ops.run_scan_single_core(x20, 64)
    torch.cuda.synchronize()
    t0 = _t.perf_counter()
    for _ in range(200):
        tcuscan_ops.run_scan_single_core(x20, 64)
        torch.cuda.synchronize()
    call_us = (_t.perf_counter() - t0) / 200 * 1e6
    g20 = torch.cuda.CUDAGraph()
    st20 = torch.cuda.Stream(dev)
    st20.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(st20):
        tcuscan_ops.run_scan_single_core(x20, 64)  # workspace of this stream exists before capture
        torch.cuda.synchronize()
        with torch.cuda.graph(g20, stream=st20):
            z20 = tcuscan_ops.run_scan_single_core(x20, 64)
    ms20 = _device_ms(g20.replay, 50, 5)
    ref20 = torch.cumsum(x20.double(), 0)
    err20 = ((z20.double() - ref20).abs() / ref20.abs().clamp_min(1.0)).max().item()
    out["scan_f16_2e20"] = entry(n20, 6 * n20, ms20, S=64, host_call_us=call_us, max_rel_err_vs_fp64=err20,
                                 note="kernel time from CUDA-graph replays; host_call_us = one synchronised call")
    del g20, x20, z20, ref20
    torch.cuda.empty_cache()
    return out


def cpu_baselines_other(seed=0):
    """Host-core baselines for the ops without a reference CPU implementation
    (bounded samples): compaction with torch.masked_select, indptr segment
    sums with numpy add.reduceat, CSR SpMV with SciPy, all on the host's cores."""
    import numpy as np
    import torch

    out = {}
    rng = np.random.default_rng(seed)
    n = 1 << 24
    x = torch.from_numpy(rng.standard_normal(n).astype(np.float16))
    m = torch.from_numpy(rng.random(n) < 0.3)
    torch.masked_select(x, m)
    t0 = time.perf_counter()
    for _ in range(5):
        torch.masked_select(x, m)
    dt = (time.perf_counter() - t0) / 5
    out["compress_f16_masked_select"] = {"value": n / dt, "unit": "elem/s", "cores": torch.get_num_threads(),
                                         "kind": "torch", "sample": "2^24 fp16, Bernoulli(0.3) mask, 5 runs"}
    lens = rng.geometric(1 / 64, size=n // 64)
    idx = np.concatenate([[0], np.cumsum(lens)])
    idx = idx[idx < n]
    xf = rng.standard_normal(n).astype(np.float32)
    np.add.reduceat(xf, idx)
    t0 = time.perf_counter()
    for _ in range(5):
        np.add.reduceat(xf, idx)
    dt = (time.perf_counter() - t0) / 5
    out["seg_sum_f32_reduceat"] = {"value": n / dt, "unit": "elem/s", "cores": 1, "kind": "numpy",
                                   "sample": "2^24 fp32, geometric(mean 64) segments, 5 runs"}
    try:
        from scipy.sparse import csr_matrix

        from tcuscan_b200 import workloads

        lens = workloads.zipf_row_lengths(1 << 20, target_nnz=1 << 22, seed=9)
        indptr = np.concatenate([[0], np.cumsum(lens)])
        nnz = int(indptr[-1])
        A = csr_matrix((rng.standard_normal(nnz).astype(np.float32), rng.integers(0, 1 << 20, nnz), indptr),
                       shape=(1 << 20, 1 << 20))
        xv = rng.uniform(-1, 1, 1 << 20).astype(np.float32)
        A @ xv
        t0 = time.perf_counter()
        for _ in range(5):
            A @ xv
        dt = (time.perf_counter() - t0) / 5
        out["spmv_f32_scipy"] = {"value": nnz / dt, "unit": "nnz/s", "cores": 1, "kind": "scipy",
                                 "sample": f"2^20 x 2^20 Zipf(1.6) rows, {nnz} nnz, 5 runs"}
    except ImportError:  # pragma: no cover
        pass
    return out


def measure_serving(dev, count=20000, seed=11, sample=240):
    """The served request stream (20000 requests: 50% scan / 30% indptr
    seg_sum / 20% compress; 40% int8 / 40% float16 / 20% float32; sizes
    log-uniform in [2^10, 2^24]; geometric(mean 64) segments; 24 GB admission
    budget) through the serving loop and through a loop of single drop-in
    calls.  Both arms read the same request data from HBM; completions are
    read on the device clock (CUDA events against a start event).
    Throughput: every request available at t = 0.  Latency: Poisson arrivals
    at half the served throughput, p50/p99 of completion - arrival.
    Accuracy: a sample of requests served in the mix is compared with the
    single calls (integer results bit-exact, floating max relative diff)."""
    import numpy as np
    import torch

    from tcuscan_b200 import serve, workloads

    wl = workloads.ServedStream(count, dev, seed=seed)
    nbytes = int(wl.element_bytes().sum())
    out = {"requests": count, "algorithmic_bytes": nbytes, "budget_bytes": 24 << 30, "slots": 4}

    def served(arrival):
        srv = serve.Server(dev, budget_bytes=24 << 30, slots=4, timing=True)
        torch.cuda.synchronize()
        srv.mark_start()
        srv.submit_many(*wl.arrays(), arrival)
        srv.run()
        torch.cuda.synchronize()
        lat = srv.done_gpu[:count] - srv.arrival[:count]
        return srv, float(np.nanmax(srv.done_gpu[:count])), lat

    def single(arrival):
        reqs = [wl.request(i) for i in range(count)]
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        start.record()
        t0 = time.perf_counter()
        evs = []
        for i, (op, x, aux) in enumerate(reqs):
            if arrival is not None:
                while time.perf_counter() - t0 < arrival[i]:
                    pass
            _, ev = serve.one_call_loop([(op, x, aux)])
            evs.append(ev[0])
        torch.cuda.synchronize()
        done = np.array([start.elapsed_time(e) * 1e-3 for e in evs])
        lat = done - (arrival if arrival is not None else 0.0)
        return float(done.max()), lat

    # warm-up: every class compiled / workspaces and pools allocated
    warm = np.arange(min(count, 400))
    srv = serve.Server(dev, budget_bytes=24 << 30, slots=4)
    srv.submit_many(*wl.arrays(warm), np.zeros(warm.size))
    srv.run()
    serve.one_call_loop([wl.request(int(i)) for i in warm[:60]])
    torch.cuda.synchronize()
    del srv

    srv, t_srv, _ = served(np.zeros(count))
    t_one, _ = single(None)
    out["served_req_per_s"] = count / t_srv
    out["one_call_req_per_s"] = count / t_one
    out["served_over_one_call"] = t_one / t_srv
    out["served_GB/s"] = nbytes / t_srv / 1e9
    out["batches"] = int(srv.batches)
    out["peak_admitted_bytes"] = int(srv.peak_used)
    del srv

    lam = 0.5 * count / t_srv
    rng = np.random.default_rng(seed + 1)
    arrival = np.cumsum(rng.exponential(1.0 / lam, size=count))
    srv, _, lat = served(arrival)
    _, lat1 = single(arrival)
    out["poisson_rate_req_per_s"] = lam
    out["served_p50_ms"] = float(np.percentile(lat, 50) * 1e3)
    out["served_p99_ms"] = float(np.percentile(lat, 99) * 1e3)
    out["one_call_p50_ms"] = float(np.percentile(lat1, 50) * 1e3)
    out["one_call_p99_ms"] = float(np.percentile(lat1, 99) * 1e3)
    out["poisson_batches"] = int(srv.batches)
    del srv

    # accuracy sample: each request served in the mix and as a single call,
    # both against an FP64 (int64) reference on the device; integer results
    # must be identical, floating results are reported as max relative error
    # with the floor max(|ref|, 1)
    idx = np.sort(np.random.default_rng(seed + 2).choice(count, size=min(sample, count), replace=False))
    srv = serve.Server(dev, budget_bytes=24 << 30, slots=4, keep_results=True)
    srv.submit_many(*wl.arrays(idx), np.zeros(idx.size))
    srv.run()
    exact_ok = True
    err_srv, err_one, diff = {}, {}, {}  # per float dtype

    def fp64_ref(op, x, aux):
        if op == serve.SCAN:
            return torch.cumsum(x.double(), 0)
        if op == serve.SEG_SUM:
            lens = (aux[1:] - aux[:-1]).long()
            rid = torch.repeat_interleave(torch.arange(lens.numel(), device=x.device), lens)
            return torch.zeros(lens.numel(), dtype=torch.float64, device=x.device).index_add_(0, rid, x.double())
        return None

    def rel(a, r):
        return ((a.double() - r).abs() / r.abs().clamp_min(1.0)).max().item() if r.numel() else 0.0

    for j, i in enumerate(idx):
        op, x, aux = wl.request(int(i))
        got = srv.result(j)
        one = serve.one_call_loop([(op, x, aux)])[0][0]
        if x.dtype == torch.int8 or op == serve.COMPRESS:
            exact_ok &= bool(torch.equal(got, one))
            if op != serve.COMPRESS:
                exact_ok &= bool(torch.equal(got.long(), fp64_ref(op, x, aux).long().to(got.dtype).long()))
        else:
            r = fp64_ref(op, x, aux)
            dk = str(x.dtype).replace("torch.", "")
            err_srv[dk] = max(err_srv.get(dk, 0.0), rel(got, r))
            err_one[dk] = max(err_one.get(dk, 0.0), rel(one, r))
            diff[dk] = max(diff.get(dk, 0.0), rel(got, one.double()))
    srv.release()
    out["sample_checked"] = int(idx.size)
    out["sample_integer_results_identical"] = exact_ok
    out["sample_max_rel_err_vs_fp64_served"] = err_srv
    out["sample_max_rel_err_vs_fp64_single_call"] = err_one
    out["sample_max_rel_diff_served_vs_single"] = diff
    del wl
    torch.cuda.empty_cache()
    return out


def _sig(v, digits=4):
    """A float rounded to `digits` significant digits (compact JSON); other values unchanged."""
    if isinstance(v, float) and v == v and v not in (float("inf"), float("-inf")) and v != 0.0:
        return float(f"{v:.{digits}g}")
    return v


LEG_KEYS = ("scan_f16_2e28", "compress_f16", "compress_f32", "seg_scan_flags_f16_2e28", "seg_sum_f16_2e28_mean64",
            "seg_sum_f16_2e28_mean4", "spmv_f32", "spmv_f16",
            "batch_rows_f32_4096", "scan_f16_2e20", "block_scan_f16_2e26_tensor_only", "block_scan_f16_2e26_engine")


def legs_summary(extras):
    """Compact per-workload summary for the headline line: throughput, time,
    fraction of the measured HBM peak and max relative error vs FP64 (0 for
    exact integer / compaction results), plus the served-stream figures."""
    if not extras:
        return None
    legs = {}
    for k in LEG_KEYS:
        e = extras.get(k)
        if not e:
            continue
        d = {"value": _sig(e["value"]), "unit": e["unit"], "ms": _sig(e["ms"]), "hbm_frac": _sig(e["hbm_frac"], 3),
             "max_rel_err": _sig(e.get("max_rel_err_vs_fp64"), 3)}
        if "host_call_us" in e:
            d["host_call_us"] = _sig(e["host_call_us"], 3)
        legs[k] = d
    sv = extras.get("served_stream")
    if sv:
        errs = sv.get("sample_max_rel_err_vs_fp64_served", {}) or {}
        legs["served"] = {
            "served_over_one_call": _sig(sv["served_over_one_call"], 3),
            "served_req_per_s": _sig(sv["served_req_per_s"]), "one_call_req_per_s": _sig(sv["one_call_req_per_s"]),
            "served_GB/s": _sig(sv["served_GB/s"]), "p50_ms": _sig(sv["served_p50_ms"], 3),
            "p99_ms": _sig(sv["served_p99_ms"], 3),
            "integer_results_identical": sv.get("sample_integer_results_identical"),
            "max_rel_err": _sig(max(errs.values()), 3) if errs else None,
        }
    return legs


def verify_headline(x, z):
    """Checks the headline scan's output on the device outside the timed
    region: z[0] == x[0], z[i] - z[i-1] == x[i] for every i >= 1 (int32
    two's-complement arithmetic, as the scan's own wrap) and z[-1] == the
    input total mod 2^32.  Together these pin z == cumsum(x) exactly."""
    import torch

    n = x.numel()
    ok = int(z[0]) == int(x[0])
    chunk = 1 << 26
    for a in range(1, n, chunk):
        b = min(n, a + chunk)
        d = z[a:b] - z[a - 1:b - 1]  # int32, wraps like the scan itself
        ok = ok and bool(torch.equal(d, x[a:b].to(torch.int32)))
    tot = int(x.to(torch.int64).sum().item())
    ok = ok and int(z[-1]) == ((tot + 2 ** 31) % 2 ** 32) - 2 ** 31
    return ok


def max_over_ranks(value, world, device):
    """Largest `value` over all ranks (the slowest rank's time); identity on one rank."""
    if world <= 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, units_per_rank, steps, max_ms):
    """Whole-job units per second of `world` independent replicas (weak scaling)."""
    return world * units_per_rank * steps / (max_ms * 1e-3)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_reference_scan(n_sample, steps, warmup, seed=0):
    """Time the reference's own run_scan_cpu (oracle/_ref, OpenMP, all host
    threads) on int8 inputs; falls back to the oracle port if it is not built."""
    import torch

    g = torch.Generator().manual_seed(seed)
    x = torch.randint(-8, 9, (n_sample,), dtype=torch.int8, generator=g)
    try:
        from oracle import build_ref

        mod = build_ref.load_module()
        fn = mod.run_scan_cpu
        kind = "reference"
        cores = int(mod.omp_max_threads())
    except Exception:
        import oracle

        xn = x.numpy()
        fn = lambda t: oracle.scan(xn)  # noqa: E731
        kind = "port"
        cores = 1
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32)
    for _ in range(warmup):
        fn(x)
    times = []
    for _ in range(steps):
        flush.zero_()  # evict caches between runs (reference CPU profiler protocol)
        t0 = time.perf_counter_ns()
        fn(x)
        times.append((time.perf_counter_ns() - t0) * 1e-9)
    return {"value": n_sample / statistics.mean(times), "unit": "elem/s", "cores": cores, "kind": kind,
            "sample": f"int8 scan of {n_sample} elements (2^{n_sample.bit_length() - 1}) x {steps} runs, "
                      f"mean {statistics.mean(times) * 1e3:.1f} ms/run, 512 MB cache flush between runs"}, times


def headline_config(op, n, world):
    """The workload description shared by both arms (identical dicts)."""
    dname = OPS[op][0]
    return {"workload": OPS[op][2], "n": n, "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (no flush needed)",
            "input": "uniform int in [-8,8]" if dname == "int8" else "uniform[-1,1) fp16"}


def run_reference_arm(args):
    """The reference's own CPU scan (run_scan_cpu, src/torch/torch_scan_cpu.h)
    on the full headline input (int8, n = 2^28), every step one call on all
    host threads with a 512 MB cache flush before it."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    n = args.n
    base, times = cpu_reference_scan(n, max(args.steps, 1), max(args.warmup, 0))
    line = {
        "impl": "reference", "metric": METRIC, "value": base["value"], "unit": "elem/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": statistics.mean(times) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "s8->s32", "data": "synthetic",
        "config": headline_config("scan_i8", n, world),
        "note": "reference run_scan_cpu (src/torch/torch_scan_cpu.h) on the host cores, full input every step",
        "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": "elem/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


PROFILE_OPS = ("compress_f16", "compress_f32", "compress_ind_f16", "spmv_f32", "spmv_f16", "serve", "segscan_i8",
               "segscan_f16", "segscan_f32", "segsum_i8", "segsum_f16", "segsum_f32", "split_f16", "sort_f16", "topk_f16",
               "rowsum_f16", "scan_i8", "scan_f16", "scan_f32", "segflags_f16")


def run_profile_op(args, dev):
    """Diagnostics for profiler captures: one extra workload only (`--n`
    elements for compaction, ~`--n` nonzeros on 2^20 rows for SpMV, `--requests`
    requests of the served stream), `--warmup` untimed then `--steps` timed
    runs; prints one JSON line with the device time per run."""
    import numpy as np
    import torch

    import tcuscan_ops
    from tcuscan_b200 import serve, workloads

    op, n = args.profile_op, args.n
    if op in ("scan_i8", "scan_f16", "scan_f32", "segflags_f16"):
        # plain scans (S from --S, 0 = tuned) and the flag-driven segmented
        # scan (start flags Bernoulli(0.01)); fp32 input is N(0, 1)
        dt = {"i8": torch.int8, "f16": torch.float16, "f32": torch.float32}[op.split("_")[1]]
        if dt == torch.float32:
            xv = torch.randn(n, device=dev, generator=torch.Generator(device=dev).manual_seed(5))
        else:
            xv = workloads.scan_input(n, dt, dev, seed=5)
        S = tcuscan_ops._pick_S(args.S or None, dt, n)
        eb = xv.element_size()
        if op == "segflags_f16":
            fl = workloads.bernoulli_mask(n, 0.01, dev, seed=13)
            fn = lambda: tcuscan_ops.run_seg_scan(xv, fl, 64)  # noqa: E731
            nbytes = n * (eb + 1 + 4)
        else:
            fn = lambda: tcuscan_ops.run_scan_multi_core(xv, S)  # noqa: E731
            nbytes = n * (eb + 4)
        units = n
        if args.phases:
            from tcuscan_ops import _lib as L

            fn()
            torch.cuda.synchronize()
            L.phase_times(dev, clear=True)
            L.set_phase_profile(True)
            for _ in range(5):
                fn()
            torch.cuda.synchronize()
            L.set_phase_profile(False)
            print(json.dumps({"phases_ns_sum_over_5_launches": L.phase_times(dev, clear=True)}), flush=True)
    elif op.startswith("compress"):
        dt = torch.float32 if op == "compress_f32" else torch.float16
        mask = workloads.bernoulli_mask(n, 0.3, dev, seed=8)
        k = int(mask.sum().item())
        xv = torch.randint(-1000, 1000, (n,), device=dev).to(dt)
        eb = xv.element_size()
        if op == "compress_ind_f16":
            fn = lambda: tcuscan_ops.run_compress_ind_no_arange(xv, mask, 64)  # noqa: E731
            nbytes = n * (eb + 1) + k * (eb + 4)
        else:
            fn = lambda: tcuscan_ops.run_compress_pos(xv, mask, k, 64)  # noqa: E731
            nbytes = n * (eb + 1) + k * eb
        units = n
    elif op == "rowsum_f16":
        # element-split segment sums (tcu_seg_sum_rows), geometric segments of mean --seg-mean
        xv = workloads.scan_input(n, torch.float16, dev, seed=5)
        stp = torch.empty(n // args.seg_mean + 1024, device=dev).geometric_(1 / args.seg_mean).to(torch.int64)
        pts = torch.cumsum(stp, 0)
        bnd = torch.cat([torch.zeros(1, dtype=torch.int64, device=dev), pts[pts < n],
                         torch.full((1,), n, dtype=torch.int64, device=dev)])
        out = torch.empty(bnd.numel() - 1, dtype=torch.float32, device=dev)
        from tcuscan_ops import _lib as L

        ws, wsb = L.workspace(dev, L.lib.tcu_rows_workspace_bytes(n))
        sp = tcuscan_ops.stream_ptr(dev)

        def fn():
            tcuscan_ops.check(L.lib.tcu_seg_sum_rows(xv.data_ptr(), L.TCU_FLOAT16, n, bnd.data_ptr(), L.TCU_INT64,
                                                     bnd.numel(), out.data_ptr(), ws, wsb, sp), op)
        nbytes = n * 2 + bnd.numel() * 8 + out.numel() * 4
        units = n
    elif op in ("split_f16", "sort_f16", "topk_f16"):
        xv = torch.rand(n, device=dev).half()
        units = n
        if op == "split_f16":
            mask = workloads.bernoulli_mask(n, 0.3, dev, seed=8)
            fn = lambda: tcuscan_ops.run_split(xv, mask, 64)  # noqa: E731
            nbytes = n * 5
        elif op == "sort_f16":
            fn = lambda: tcuscan_ops.run_radix_sort(xv, 128)  # noqa: E731
            nbytes = n * 8
        else:
            kt = int(n ** 0.5)
            fn = lambda: tcuscan_ops.run_topk_fp16(xv, kt, 0.0, 1.0, 128)  # noqa: E731
            nbytes = n * 2
    elif op.startswith("spmv"):
        dt = torch.float32 if op == "spmv_f32" else torch.float16
        vals, indptr, cols, xs = workloads.zipf_csr(target_nnz=min(n, 1 << 26), dtype=dt, device=dev, seed=9)
        fn = lambda: tcuscan_ops.run_spmv_v2(vals, indptr, cols, xs, 64)  # noqa: E731
        eb = vals.element_size()
        rows = indptr.numel() - 1
        nbytes = vals.numel() * (eb + 4) + (rows + 1) * 4 + rows * 4 + xs.numel() * eb
        units = vals.numel()
    elif op.startswith("seg"):
        # segmented scans over sorted bounds: "segscan" = few long segments
        # (one per 2^20 elements, scan output), "segsum" = CSR-like segments of
        # mean length 64 (per-segment sums)
        dt = {"i8": torch.int8, "f16": torch.float16, "f32": torch.float32}[op.split("_")[1]]
        xv = workloads.scan_input(n, dt, dev, seed=5)
        eb = xv.element_size()
        if op.startswith("segscan"):
            bnd = torch.arange(0, n, 1 << 20, dtype=torch.int64, device=dev)
            out = torch.empty(n, dtype=torch.int32 if dt == torch.int8 else torch.float32, device=dev)
            nbytes = n * (eb + 4) + bnd.numel() * 8
            sums = 0
        else:
            steps = torch.empty(n // args.seg_mean + 1024, device=dev).geometric_(1 / args.seg_mean).to(torch.int64)
            pts = torch.cumsum(steps, 0)
            bnd = torch.cat([torch.zeros(1, dtype=torch.int64, device=dev), pts[pts < n],
                             torch.full((1,), n, dtype=torch.int64, device=dev)])
            out = torch.empty(bnd.numel() - 1, dtype=torch.int32 if dt == torch.int8 else torch.float32, device=dev)
            nbytes = n * eb + bnd.numel() * 8 + out.numel() * 4
            sums = 1
        from tcuscan_ops import _lib as L

        ws, wsb = L.workspace(dev, L.lib.tcu_workspace_bytes(n, 64))
        sp = tcuscan_ops.stream_ptr(dev)

        def fn():
            tcuscan_ops.check(L.lib.tcu_seg_bounds(xv.data_ptr(), L.DTYPE_CODE[dt], n, 64, bnd.data_ptr(), L.TCU_INT64,
                                                   bnd.numel(), sums, out.data_ptr(), ws, wsb, sp), op)
        units = n
        if args.phases:
            fn()
            torch.cuda.synchronize()
            L.phase_times(dev, clear=True)
            L.set_phase_profile(True)
            for _ in range(5):
                fn()
            torch.cuda.synchronize()
            L.set_phase_profile(False)
            print(json.dumps({"phases_ns_sum_over_5_launches": L.phase_times(dev, clear=True)}), flush=True)
    else:
        wl = workloads.ServedStream(args.requests, dev, seed=11)
        nbytes = int(wl.element_bytes().sum())
        units = args.requests

        def fn():
            srv = serve.Server(dev, budget_bytes=24 << 30, slots=4)
            srv.submit_many(*wl.arrays(), np.zeros(args.requests))
            srv.run()
    ms = _device_ms(fn, args.steps, args.warmup)
    print(json.dumps({"profile_op": op, "units": units, "ms": ms, "GB/s": nbytes / (ms * 1e-3) / 1e9,
                      "algorithmic_bytes": nbytes}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--op", default="scan_i8", choices=sorted(OPS))
    ap.add_argument("--S", type=int, default=0, help="tile parameter (0 = autotuned default)")
    ap.add_argument("--n", type=int, default=1 << 28)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--phases", action="store_true", help="print a per-phase device-time breakdown (diagnostics)")
    ap.add_argument("--no-extras", action="store_true", help="headline workload only")
    ap.add_argument("--profile-op", default=None, choices=PROFILE_OPS,
                    help="diagnostics: run only this extra workload (for profiler captures)")
    ap.add_argument("--requests", type=int, default=2000, help="served-stream requests for --profile-op serve")
    ap.add_argument("--seg-mean", type=int, default=64, help="mean segment length for --profile-op segsum_*")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    if args.profile_op:
        return run_profile_op(args, dev)

    import tcuscan_ops

    dname, bpe, _ = OPS[args.op]
    n = args.n
    if not args.S:
        args.S = tcuscan_ops._pick_S(None, torch.int8 if dname == "int8" else torch.float16, n)
    g = torch.Generator(device=dev).manual_seed(1234 + rank)
    if dname == "int8":
        x = torch.randint(-8, 9, (n,), dtype=torch.int8, device=dev, generator=g)
    else:
        x = (torch.rand(n, device=dev, generator=g) * 2 - 1).half()

    def step():
        return tcuscan_ops.run_scan_multi_core(x, args.S)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    tcuscan_ops.raise_device_error(dev)
    if args.phases:
        from tcuscan_ops import _lib as L

        L.phase_times(dev, clear=True)
        L.set_phase_profile(True)
        for _ in range(10):
            step()
        torch.cuda.synchronize()
        L.set_phase_profile(False)
        ph = L.phase_times(dev, clear=True)
        print(json.dumps({"phases_ns_sum_over_10_launches": ph}), file=sys.stderr, flush=True)

    props = torch.cuda.get_device_properties(dev)
    bus = None
    if hasattr(props, "pci_bus_id"):
        bus = f"{getattr(props, 'pci_domain_id', 0):08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}.0"
    sampler = ClockSampler(bus)
    sampler.start()
    sampler.wait_for(time.time(), timeout=5.0)  # sampling has started before the timed region

    stream = torch.cuda.current_stream(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_all0, t_all1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    wall0 = time.time()
    t_all0.record(stream)
    for i in range(args.steps):
        evs[i][0].record(stream)
        step()
        evs[i][1].record(stream)
    t_all1.record(stream)
    torch.cuda.synchronize()
    wall1 = time.time()
    if world > 1:
        torch.distributed.barrier()
    total_ms = t_all0.elapsed_time(t_all1)
    per = [a.elapsed_time(b) for a, b in evs]
    tcuscan_ops.raise_device_error(dev)
    sampler.wait_for(wall1, timeout=2.0)  # a sample after the region closes the window
    clocks = sampler.summary(wall0, wall1)
    sampler.stop()

    total_ms = max_over_ranks(total_ms, world, dev)

    # ---- the timed output, checked once on the device outside the timed region ----
    z = step()
    torch.cuda.synchronize()
    if dname == "int8":
        check = {"exact": verify_headline(x, z), "method": "z[0] == x[0], diff(z) == x[1:] (int32), z[-1] == sum(x)"}
        if not check["exact"]:
            raise RuntimeError("headline scan output differs from cumsum(x)")
    else:
        ref = torch.cumsum(x.double(), 0)
        err = ((z.double() - ref).abs() / ref.abs().clamp_min(1.0)).max().item()
        check = {"max_rel_err_vs_fp64": err, "method": "FP64 cumsum on the device, floor max(|ref|, 1)"}
        del ref
        if err > 1e-3:
            raise RuntimeError(f"headline scan error {err} above 1e-3")
    del z

    # ---- e2e through the public API with host buffers: the host-buffer scan
    # (tcuscan_b200.stream) copies each 2^24-element chunk in, scans it and
    # copies it out on three streams, the chunks chained on the device ----
    from tcuscan_b200 import stream as host_stream

    x_host = torch.empty(n, dtype=x.dtype, pin_memory=True)
    x_host.copy_(x.cpu())
    out_dtype = torch.int32 if dname == "int8" else torch.float32
    z_host = torch.empty(n, dtype=out_dtype, pin_memory=True)
    scanner = host_stream.HostScanner(n, x.dtype, dev, chunk=1 << 24)
    e2e_steps = max(3, min(args.steps, 20))

    def e2e_step():
        scanner.scan(x_host, z_host, args.S)

    e2e_step()
    torch.cuda.synchronize()
    # the host result ends with the total of the input (int32 wrap for int8)
    if dname == "int8":
        tot = int(x.long().sum().item())
        ok = int(z_host[-1].item()) == ((tot + 2 ** 31) % 2 ** 32) - 2 ** 31
    else:
        tot = float(x.double().sum().item())
        ok = abs(float(z_host[-1].item()) - tot) <= 1e-3 * max(1.0, abs(tot))
    if not ok:
        raise RuntimeError("end-to-end scan result differs from the input total")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        torch.distributed.barrier()
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_ms = max_over_ranks(e2e_ms, world, dev)
    # the copy-only bound of the same step: both copies of the whole arrays,
    # concurrently on two streams, no scan
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    zd = scanner.z

    def copies():
        s_in.wait_stream(stream)
        s_out.wait_stream(stream)
        with torch.cuda.stream(s_in):
            x.copy_(x_host, non_blocking=True)
        with torch.cuda.stream(s_out):
            z_host.copy_(zd[:n], non_blocking=True)
        stream.wait_stream(s_in)
        stream.wait_stream(s_out)

    copies()
    torch.cuda.synchronize()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record(stream)
    for _ in range(3):
        copies()
    c1.record(stream)
    torch.cuda.synchronize()
    copy_ms = max_over_ranks(c0.elapsed_time(c1) / 3, world, dev)

    extras = None
    if rank == 0 and world == 1 and not args.no_extras:
        del x_host, z_host, scanner
        extras = measure_extras(dev)
        extras["served_stream"] = measure_serving(dev)
        if not args.no_cpu:
            extras["cpu_baselines_other_ops"] = cpu_baselines_other()

    cpu_base = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu_base, _ = cpu_reference_scan(n, 5, 1)

    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return 0

    peak, peak_kind = measured_peak()
    avg_launch_ms = statistics.mean(per)
    alg_bytes = n * bpe
    achieved = alg_bytes / (avg_launch_ms * 1e-3) / 1e9
    value = replica_throughput(world, n, args.steps, total_ms)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "elem/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "s8->s32" if dname == "int8" else "f16->f32",
        "data": "synthetic",
        "config": headline_config(args.op, n, world),
        "tile_S": args.S,
        "check": check,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "frac_of_spec_8TBs": achieved / SPEC_HBM_GBS,
                     "traffic": profile_traffic(args.op), "algorithmic_bytes_per_launch": alg_bytes,
                     "kernel": "scan_tc_kernel", "avg_launch_ms": avg_launch_ms},
        "cpu_baseline": cpu_base,
        "e2e": {"value": replica_throughput(world, n, e2e_steps, e2e_ms), "unit": "elem/s",
                "h2d_bytes_per_step": n * x.element_size(), "d2h_bytes_per_step": n * 4,
                "ms_per_step": e2e_ms / e2e_steps,
                # the same bytes copied with no scan (both directions at once): the PCIe bound
                "copy_only_ms_per_step": copy_ms, "frac_of_copy_bound": copy_ms / (e2e_ms / e2e_steps)},
        "clocks": clocks,
        "gpu_launches": args.steps,
        "median_ms_per_launch": statistics.median(per),
        "legs": legs_summary(extras),
    }
    if extras is not None:
        print(json.dumps({"extras": extras}), flush=True)
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
