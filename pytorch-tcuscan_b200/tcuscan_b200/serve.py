"""Serving loop: continuous batching of scan, seg_sum and compress requests.

The reference answers one request per call (``run_scan_multi_core``,
``run_seg_sum_multi_core``, ``run_compress`` in src/torch/torch_scan.h,
torch_seg_ops.h and torch_compress.h), each a separate launch that blocks on
its stream.  This module keeps the device busy with many requests at once:

- Requests of mixed ops, sizes and dtypes arrive over time (``submit`` one at
  a time, or ``submit_many`` with an arrival time per request).  They wait in
  one queue per class (op, dtype, index width).
- A batch is admitted when a stream slot is free and its device memory fits
  the HBM budget: every batch takes one block of a device arena allocated once
  at start (first fit, blocks coalesce when freed), holding the packed
  inputs, outputs, row pointers and the batch's request table.  Requests keep
  arriving while earlier batches run; the next batch takes whatever has
  arrived (continuous batching), oldest class first.
- Scan and seg_sum requests of ``SOLO_MIN`` (2^22) elements or more are
  read in place: each runs the single-call kernel (``tcu_scan`` /
  ``tcu_seg_sum_rows`` on its own values and row pointers) into its batch's
  block, so the bulk of the served bytes is never copied.  The smaller
  requests of a batch take one pack launch (``tcu_pack``: every request's
  elements copied back to back into the block, each request on a
  256-element boundary, padding zeroed; seg_sum row pointers rebased by the
  request's offset) and one segmented launch over the packed buffer:
  ``tcu_seg_bounds`` with the request starts as segment starts (scan), the
  element-split segment sums over the rebased row pointers (seg_sum), or
  ``tcu_compress_segments`` (compress -- every compress request is packed,
  with its output offset).  Batches on different slots run on different
  CUDA streams and overlap on the GPU.
- Completion is read from one CUDA event per slot (polled, never a device
  synchronisation).  A request's result is a view of its batch's block.

Every request's result equals what the single call returns for it: integer
results bit for bit, floating results within the scan family's tolerance
(the requests start on row boundaries of their own, so no neighbour enters
their rows; only the order in which FP64 carries are added may differ).
"""
import collections
import ctypes
import time

import numpy as np
import torch

import tcuscan_ops
from tcuscan_ops import _lib

SCAN, SEG_SUM, COMPRESS = 0, 1, 2
OP_NAMES = ("scan", "seg_sum", "compress")
DTYPES = (torch.int8, torch.float16, torch.float32)
_DT_INDEX = {d: i for i, d in enumerate(DTYPES)}
_EB = np.array([1, 2, 4], dtype=np.int64)
ALIGN = 256        # elements: every request starts on a 256-element boundary of its batch
# scan / seg_sum requests of at least this many elements are not packed: each
# runs the single-call kernel on its own input in place (the pack copy would
# read and write every input byte once more), writing into its batch's block.
# Each one costs a launch from the host loop, so the threshold trades copied
# bytes against launches: on the served stream (20000 requests, log-uniform
# sizes in [2^10, 2^24]) everything packed gave 2.39 TB/s, 2^20 2.15, 2^21
# 2.39, 2^22 2.54 and 2^23 2.55 TB/s.
SOLO_MIN = 1 << 22
BLOCK_ALIGN = 256  # bytes: arena blocks and the buffers inside them
BATCH_SLACK = 8192  # bytes per batch for buffer alignment inside its block

# matches tcu_pack_item_t (include/tcuscan.h)
PACK_ITEM = np.dtype([("src", "<u8"), ("dst", "<i8"), ("n", "<i8"), ("len", "<i8"), ("add", "<i8")])


def _roundup(a, m):
    return (a + (m - 1)) // m * m


class Arena:
    """First-fit allocator over one device buffer; freed blocks coalesce."""

    def __init__(self, nbytes, device):
        nbytes = int(nbytes) // BLOCK_ALIGN * BLOCK_ALIGN
        self.buf = torch.empty(nbytes, dtype=torch.uint8, device=device)
        self.base = self.buf.data_ptr()
        self.size = nbytes
        self.free = [(0, nbytes)]  # sorted, disjoint (offset, size)

    def largest(self):
        return max((s for _, s in self.free), default=0)

    def alloc(self, nbytes):
        nbytes = _roundup(int(nbytes), BLOCK_ALIGN)
        for i, (o, s) in enumerate(self.free):
            if s >= nbytes:
                if s == nbytes:
                    del self.free[i]
                else:
                    self.free[i] = (o + nbytes, s - nbytes)
                return o, nbytes
        return None, 0

    def release(self, off, nbytes):
        fl = self.free
        i = 0
        while i < len(fl) and fl[i][0] < off:
            i += 1
        fl.insert(i, (off, nbytes))
        if i + 1 < len(fl) and fl[i][0] + fl[i][1] == fl[i + 1][0]:  # merge with the next block
            fl[i] = (fl[i][0], fl[i][1] + fl[i + 1][1])
            del fl[i + 1]
        if i > 0 and fl[i - 1][0] + fl[i - 1][1] == fl[i][0]:  # and with the previous one
            fl[i - 1] = (fl[i - 1][0], fl[i - 1][1] + fl[i][1])
            del fl[i]


class _Slot:
    __slots__ = ("idx", "stream", "event", "pinned", "pos_host", "ws", "wsb")


class _Batch:
    __slots__ = ("id", "cls", "ids", "slot", "off", "bytes", "out_off", "out_dtype", "out_len")


class Server:
    """Continuous-batching request loop on one GPU.

    budget_bytes  device memory of the arena (admission) plus the per-slot
                  look-back workspaces.
    slots         concurrent batches (one CUDA stream each).
    max_batch     requests per batch; max_batch_bytes caps one batch's block.
    keep_results  keep every finished batch's block for ``result()`` until
                  ``release()``; otherwise blocks go back at completion.
    timing        record completions on the device clock (``done_gpu``)
                  against the event of ``mark_start()``.
    """

    def __init__(self, device="cuda", budget_bytes=24 << 30, slots=4, max_batch=4096, max_batch_bytes=None,
                 S=None, keep_results=False, timing=False):
        self.dev = torch.device(device)
        if self.dev.type != "cuda":
            raise ValueError("the serving loop runs on a CUDA device")
        if self.dev.index is None:
            self.dev = torch.device("cuda", torch.cuda.current_device())
        self.budget = int(budget_bytes)
        self.max_batch = int(max_batch)
        self.max_batch_bytes = int(max_batch_bytes) if max_batch_bytes else max(self.budget // max(slots, 1), 1 << 20)
        self.S = S
        self.keep = bool(keep_results)
        self.timing = bool(timing)
        # per-slot look-back workspace sized for the largest batch, then the arena
        ws_need = int(max(_lib.lib.tcu_workspace_bytes(self.max_batch_bytes, 64),
                          _lib.lib.tcu_rows_workspace_bytes(self.max_batch_bytes)))
        self.slots = []
        for i in range(slots):
            sl = _Slot()
            sl.idx = i
            sl.stream = torch.cuda.Stream(self.dev)
            sl.event = torch.cuda.Event(enable_timing=self.timing)
            sl.pinned = torch.empty(1 << 20, dtype=torch.uint8, pin_memory=True)
            sl.pos_host = torch.empty(max_batch + 1, dtype=torch.int64, pin_memory=True)
            sl.ws = torch.empty(ws_need, dtype=torch.uint8, device=self.dev)  # owned by the slot
            sl.wsb = ctypes.c_size_t(ws_need)
            st_ = _lib.lib.tcu_workspace_init(sl.ws.data_ptr(), sl.wsb, ctypes.c_void_p(sl.stream.cuda_stream))
            tcuscan_ops.check(st_, "serve workspace")
            self.slots.append(sl)
        ws_total = ws_need * slots
        if self.budget - ws_total < (1 << 20):
            raise ValueError("serving budget too small for its workspaces")
        self.arena = Arena(self.budget - ws_total, self.dev)
        self.free_slots = collections.deque(range(slots))
        self.inflight = {}  # slot index -> _Batch
        self.finished = {}  # batch id -> _Batch (keep_results)
        self.used = 0
        self.peak_used = 0
        self.batches = 0
        self.t0 = time.perf_counter()
        self.start_event = None
        # request table (structure of arrays, grown by doubling)
        self._cap = 0
        self._n = 0
        self._alloc(1024)
        self._next_arrival = 0  # requests [0, _next_arrival) have been moved to the class queues
        self.queues = collections.defaultdict(collections.deque)  # class -> deque of id arrays
        self._keepalive = {}

    # ---------------------------------------------------------------- table
    def _alloc(self, cap):
        def grow(a, dtype, fill=0):
            b = np.full(cap, fill, dtype=dtype)
            if a is not None:
                b[: a.size] = a
            return b

        g = lambda name: getattr(self, name, None)  # noqa: E731
        self.op = grow(g("op"), np.int8)
        self.dt = grow(g("dt"), np.int8)
        self.iw = grow(g("iw"), np.int8)           # row-pointer bytes (seg_sum: 4 or 8)
        self.n = grow(g("n"), np.int64)
        self.xp = grow(g("xp"), np.uint64)
        self.ap = grow(g("ap"), np.uint64)         # mask (compress) or row pointers (seg_sum)
        self.nseg = grow(g("nseg"), np.int64)
        self.arrival = grow(g("arrival"), np.float64, np.inf)
        self.admit = grow(g("admit"), np.float64, np.nan)
        self.done = grow(g("done"), np.float64, np.nan)
        self.done_gpu = grow(g("done_gpu"), np.float64, np.nan)  # device clock (timing=True)
        self.bid = grow(g("bid"), np.int64, -1)
        self.roff = grow(g("roff"), np.int64, -1)
        self.rlen = grow(g("rlen"), np.int64, -1)
        self._cap = cap

    def _reserve(self, k):
        if self._n + k > self._cap:
            cap = self._cap
            while cap < self._n + k:
                cap *= 2
            self._alloc(cap)

    def now(self):
        return time.perf_counter() - self.t0

    def mark_start(self):
        """Restart the clock: arrival times count from here, and (timing=True)
        completions are read on the device clock from an event recorded now."""
        self.start_event = torch.cuda.Event(enable_timing=True)
        self.start_event.record(torch.cuda.current_stream(self.dev))
        self.t0 = time.perf_counter()

    def submit(self, op, x, aux=None, arrival=None):
        """Queue one request; returns its id.  op: "scan" | "seg_sum" | "compress".
        seg_sum takes a CSR row-pointer tensor (int32/int64, R + 1 entries,
        leading 0), compress an int8 mask of x's length."""
        op = OP_NAMES.index(op) if isinstance(op, str) else int(op)
        x = tcuscan_ops._cuda_input(x)
        if x.device != self.dev:
            raise ValueError("request on another device")
        if x.dtype not in _DT_INDEX:
            raise TypeError(f"serving takes int8, float16 or float32 data, got {x.dtype}")
        nseg, iw, ap = 0, 0, 0
        if op == SEG_SUM:
            aux = tcuscan_ops._bounds_input(aux, x.device, "serve seg_sum")
            nseg, iw, ap = aux.numel() - 1, aux.element_size(), aux.data_ptr()
            if nseg < 0:
                raise ValueError("seg_sum needs at least one row pointer")
        elif op == COMPRESS:
            aux = tcuscan_ops._mask_input(aux, x.numel(), x.device)
            ap = aux.data_ptr()
        elif op != SCAN:
            raise ValueError(f"unknown op {op}")
        if x.numel() == 0:
            raise ValueError("empty request")
        rid = self.submit_many(np.array([op]), np.array([_DT_INDEX[x.dtype]]), np.array([x.numel()]),
                               np.array([x.data_ptr()], dtype=np.uint64), np.array([ap], dtype=np.uint64),
                               np.array([nseg]), np.array([iw]),
                               np.array([self.now() if arrival is None else arrival]))[0]
        self._keepalive[int(rid)] = (x, aux)
        return int(rid)

    def submit_many(self, op, dt, n, xp, ap, nseg, iw, arrival):
        """Queue a block of requests described by arrays (device pointers as
        uint64).  Arrival times (seconds since the server's clock started)
        must be non-decreasing; a request enters its queue once
        ``now() >= arrival``.  The caller keeps the data alive until the
        requests complete."""
        k = len(n)
        arrival = np.asarray(arrival, dtype=np.float64)
        if k and self._n and arrival[0] < self.arrival[self._n - 1]:
            raise ValueError("arrival times must be non-decreasing across submissions")
        self._reserve(k)
        s = slice(self._n, self._n + k)
        self.op[s], self.dt[s], self.n[s] = op, dt, n
        self.xp[s], self.ap[s], self.nseg[s], self.iw[s] = xp, ap, nseg, iw
        self.arrival[s] = arrival
        ids = np.arange(self._n, self._n + k, dtype=np.int64)
        self._n += k
        return ids

    # --------------------------------------------------------------- sizing
    def _bytes(self, ids):
        """Block bytes each request adds to its batch (inputs, outputs, row
        pointers and its entries of the batch's request table)."""
        npad = _roundup(self.n[ids], ALIGN)
        eb = _EB[self.dt[ids]]
        op = self.op[ids]
        b = npad * eb + 2 * PACK_ITEM.itemsize + 16
        b = b + np.where(op == SCAN, npad * 4, 0)
        b = b + np.where(op == SEG_SUM, (self.nseg[ids] + 1) * 12, 0)
        b = b + np.where(op == COMPRESS, npad * (1 + eb) + 8, 0)
        return b

    # ---------------------------------------------------------------- loop
    def _arrivals(self):
        t = self.now()
        hi = int(np.searchsorted(self.arrival[: self._n], t, side="right"))
        if hi > self._next_arrival:
            ids = np.arange(self._next_arrival, hi, dtype=np.int64)
            key = (self.op[ids].astype(np.int64) * 3 + self.dt[ids]) * 16 + self.iw[ids]
            order = np.argsort(key, kind="stable")
            ks, idx = np.unique(key[order], return_index=True)
            bounds = list(idx) + [len(order)]
            for j, kk in enumerate(ks):
                self.queues[int(kk)].append(ids[order[bounds[j]:bounds[j + 1]]])
            self._next_arrival = hi
        return t

    def _head_arrival(self, cls):
        q = self.queues.get(cls)
        return self.arrival[q[0][0]] if q else np.inf

    def _take(self, cls, room):
        """Pop the longest prefix of the class queue that fits `room` bytes."""
        q = self.queues[cls]
        parts, count, used = [], 0, 0
        room -= BATCH_SLACK
        while q and count < self.max_batch:
            ids = q[0]
            b = self._bytes(ids)
            cum = np.cumsum(b)
            k = int(np.searchsorted(cum, room - used, side="right"))
            k = min(k, self.max_batch - count)
            if k == 0:
                if count == 0 and b[0] + BATCH_SLACK > min(self.budget, self.max_batch_bytes):
                    raise MemoryError(f"request {int(ids[0])} needs {int(b[0])} bytes, over the serving budget")
                break
            parts.append(ids[:k])
            count += k
            used += int(cum[k - 1])
            if k == ids.size:
                q.popleft()
            else:
                q[0] = ids[k:]
                break
        if not q:
            self.queues.pop(cls, None)
        if not parts:
            return None, 0
        return np.concatenate(parts), used + BATCH_SLACK

    def _poll(self):
        for si in list(self.inflight):
            b = self.inflight[si]
            if self.slots[si].event.query():
                del self.inflight[si]
                self._complete(b)

    def _complete(self, b):
        t = self.now()
        ids = b.ids
        sl = self.slots[b.slot]
        self.done[ids] = t
        if self.timing and self.start_event is not None:
            self.done_gpu[ids] = self.start_event.elapsed_time(sl.event) * 1e-3
        if self.op[ids[0]] == COMPRESS:  # outputs are known now
            pos = sl.pos_host[: ids.size + 1].numpy()
            self.roff[ids] = pos[:-1]
            self.rlen[ids] = pos[1:] - pos[:-1]
        self.free_slots.append(b.slot)
        if self.keep:
            self.finished[b.id] = b
        else:
            self._free(b)
        if self._keepalive:
            for i in ids:
                self._keepalive.pop(int(i), None)

    def _free(self, b):
        self.arena.release(b.off, b.bytes)
        self.used -= b.bytes

    def step(self):
        """One pass of the loop: take arrivals, retire finished batches, launch
        new batches while slots and memory allow.  Returns the number launched."""
        self._arrivals()
        if self.inflight:
            self._poll()
        launched = 0
        while self.free_slots and self.queues:
            cls = min(self.queues, key=self._head_arrival)
            room = min(self.arena.largest(), self.max_batch_bytes)
            ids, nbytes = self._take(cls, room)
            if ids is None:
                break  # the oldest class does not fit yet: wait for memory
            self._launch(cls, ids, nbytes)
            launched += 1
        return launched

    def pending(self):
        return self._next_arrival < self._n or bool(self.queues) or bool(self.inflight)

    def run(self):
        """Drive the loop until every submitted request has completed."""
        while self.pending():
            if self.step() == 0 and not self.inflight:
                if self.queues:
                    raise MemoryError("the serving budget is held by kept results: call release()")
                if self._next_arrival < self._n:  # idle until the next arrival
                    wait = self.arrival[self._next_arrival] - self.now()
                    if wait > 2e-4:
                        time.sleep(wait - 1e-4)
        return self

    # -------------------------------------------------------------- launch
    def _launch(self, cls, ids, nbytes):
        op = int(self.op[ids[0]])
        dti = int(self.dt[ids[0]])
        dtype = DTYPES[dti]
        eb = int(_EB[dti])
        si = self.free_slots.popleft()
        sl = self.slots[si]
        off, nbytes = self.arena.alloc(nbytes)
        if off is None:  # cannot happen: room came from the largest free block
            raise MemoryError("arena allocation failed")
        self.used += nbytes
        self.peak_used = max(self.peak_used, self.used)
        self.admit[ids] = self.now()
        # requests read in place (large scan / seg_sum inputs, 16-byte aligned)
        # and the rest, which are packed back to back
        solo = np.zeros(ids.size, dtype=bool)
        if op in (SCAN, SEG_SUM):
            solo = (self.n[ids] >= SOLO_MIN) & (self.xp[ids] % 16 == 0)
            if op == SEG_SUM:
                solo &= self.ap[ids] % 8 == 0
        ids_p, ids_s = ids[~solo], ids[solo]
        n = self.n[ids_p]
        k = ids_p.size
        npad = _roundup(n, ALIGN)
        dst = np.zeros(k, dtype=np.int64)
        if k:
            np.cumsum(npad[:-1], out=dst[1:])
        total = int(npad.sum())

        # request table of the packed part, staged in the slot's pinned buffer
        items = np.empty(k, dtype=PACK_ITEM)
        items["src"], items["dst"], items["n"], items["len"], items["add"] = self.xp[ids_p], dst, n, npad, 0
        meta = [items.view(np.uint8)]
        if op == SEG_SUM:
            nb = self.nseg[ids_p] + 1
            boff = np.zeros(k, dtype=np.int64)
            if k:
                np.cumsum(nb[:-1], out=boff[1:])
            bitems = np.empty(k, dtype=PACK_ITEM)
            bitems["src"], bitems["dst"], bitems["n"], bitems["len"], bitems["add"] = self.ap[ids_p], boff, nb, nb, dst
            meta.append(bitems.view(np.uint8))
        elif op == COMPRESS:
            mitems = items.copy()
            mitems["src"] = self.ap[ids_p]
            meta += [mitems.view(np.uint8), dst.view(np.uint8)]
        else:
            meta.append(dst.view(np.uint8))
        mb = max(sum(m.size for m in meta), 16)
        if mb > sl.pinned.numel():
            sl.pinned = torch.empty(_roundup(mb, 1 << 20), dtype=torch.uint8, pin_memory=True)
        pn = sl.pinned.numpy()
        o = 0
        for m in meta:
            pn[o:o + m.size] = m
            o += m.size

        # buffers of the block: [meta | x | outputs ...]
        cur = [off]

        def carve(nb_):
            p = cur[0]
            cur[0] = _roundup(p + int(nb_), BLOCK_ALIGN)
            return p

        m_off = carve(mb)
        x_off = carve(total * eb)
        base = self.arena.base
        ab = self.arena.buf
        st = sl.stream
        sp = ctypes.c_void_p(st.cuda_stream)
        S = tcuscan_ops._pick_S(self.S, dtype, max(total, 1), op="seg")
        L = _lib.lib
        wsp = sl.ws.data_ptr()
        with torch.cuda.stream(st):
            if k:
                ab[m_off:m_off + mb].copy_(sl.pinned[:mb], non_blocking=True)
                tcuscan_ops.check(L.tcu_pack(base + m_off, k, eb, eb, base + x_off, total, sp), "serve pack")
            if op == SCAN:
                out_dtype = tcuscan_ops._scan_out_dtype(dtype)
                npad_s = _roundup(self.n[ids_s], ALIGN)
                z_off = carve((total + int(npad_s.sum())) * 4)
                if k:
                    s_ = L.tcu_seg_bounds(base + x_off, _lib.DTYPE_CODE[dtype], total, S, base + m_off + items.nbytes,
                                          _lib.TCU_INT64, k, 0, base + z_off, wsp, sl.wsb, sp)
                    tcuscan_ops.check(s_, "serve scan")
                    self.roff[ids_p], self.rlen[ids_p] = dst, n
                o_ = total
                for j, r in enumerate(ids_s):  # in place: the single call's scan
                    nr = int(self.n[r])
                    S_r = tcuscan_ops._pick_S(self.S, dtype, nr)
                    s_ = L.tcu_scan(int(self.xp[r]), _lib.DTYPE_CODE[dtype], nr, S_r, 0.0, base + z_off + o_ * 4,
                                    wsp, sl.wsb, sp)
                    tcuscan_ops.check(s_, "serve scan (in place)")
                    self.roff[r], self.rlen[r] = o_, nr
                    o_ += int(npad_s[j])
                out_len = max(o_, 1)
            elif op == SEG_SUM:
                out_dtype = tcuscan_ops._scan_out_dtype(dtype)
                iw = int(self.iw[ids[0]])
                nbt = int(nb.sum()) if k else 0
                b_off = carve(nbt * 8)
                out_p = max(nbt - 1, 0)
                z_off = carve(max(out_p + int(self.nseg[ids_s].sum()), 1) * 4)
                if k:
                    tcuscan_ops.check(L.tcu_pack(base + m_off + items.nbytes, k, iw, 8, base + b_off, nbt, sp),
                                      "serve pack row pointers")
                    if tcuscan_ops._rows_for(dtype, total, nbt - 1):  # same rule as run_seg_sum_*
                        s_ = L.tcu_seg_sum_rows(base + x_off, _lib.DTYPE_CODE[dtype], total, base + b_off,
                                                _lib.TCU_INT64, nbt, base + z_off, wsp, sl.wsb, sp)
                    else:
                        s_ = L.tcu_seg_bounds(base + x_off, _lib.DTYPE_CODE[dtype], total, S, base + b_off,
                                              _lib.TCU_INT64, nbt, 1, base + z_off, wsp, sl.wsb, sp)
                    tcuscan_ops.check(s_, "serve seg_sum")
                    self.roff[ids_p], self.rlen[ids_p] = boff, self.nseg[ids_p]
                o_ = out_p
                bdt = _lib.TCU_INT64 if iw == 8 else _lib.TCU_INT32
                for r in ids_s:  # in place: the request's own values and row pointers
                    nr, ns = int(self.n[r]), int(self.nseg[r])
                    if ns > 0:
                        s_ = L.tcu_seg_sum_rows(int(self.xp[r]), _lib.DTYPE_CODE[dtype], nr, int(self.ap[r]), bdt,
                                                ns + 1, base + z_off + o_ * 4, wsp, sl.wsb, sp)
                        tcuscan_ops.check(s_, "serve seg_sum (in place)")
                    self.roff[r], self.rlen[r] = o_, ns
                    o_ += ns
                out_len = max(o_, 1)
            else:
                out_dtype = dtype
                mk_off = carve(total)
                z_off = carve(total * eb)
                p_off = carve((k + 1) * 8)
                tcuscan_ops.check(L.tcu_pack(base + m_off + items.nbytes, k, 1, 1, base + mk_off, total, sp),
                                  "serve pack masks")
                starts = base + m_off + 2 * items.nbytes
                s_ = L.tcu_compress_segments(base + x_off, eb, base + mk_off, total, starts, k, base + z_off, total,
                                             base + p_off, wsp, sl.wsb, sp)
                tcuscan_ops.check(s_, "serve compress")
                sl.pos_host[: k + 1].copy_(ab[p_off:p_off + (k + 1) * 8].view(torch.int64), non_blocking=True)
                out_len = total
            sl.event.record(st)
        if cur[0] - off > nbytes:
            raise AssertionError("batch layout overran its block")
        b = _Batch()
        b.id, b.cls, b.ids, b.slot, b.off, b.bytes = self.batches, cls, ids, si, off, nbytes
        b.out_off, b.out_dtype, b.out_len = z_off, out_dtype, out_len
        self.bid[ids] = self.batches
        self.batches += 1
        self.inflight[si] = b

    # ------------------------------------------------------------- results
    def result(self, rid):
        """The result of a finished request (keep_results=True): scan -> the
        inclusive scan, seg_sum -> per-row sums, compress -> selected values.
        A view of the arena, valid until ``release()``."""
        rid = int(rid)
        if np.isnan(self.done[rid]):
            raise RuntimeError(f"request {rid} has not completed")
        b = self.finished.get(int(self.bid[rid]))
        if b is None:
            raise KeyError(f"request {rid}: result released (keep_results=False or release() called)")
        es = torch.empty((), dtype=b.out_dtype).element_size()
        out = self.arena.buf[b.out_off:b.out_off + b.out_len * es].view(b.out_dtype)
        return out[int(self.roff[rid]): int(self.roff[rid] + self.rlen[rid])]

    def release(self):
        """Drop every kept batch and return its block to the arena."""
        for b in self.finished.values():
            self._free(b)
        self.finished.clear()

    def latencies(self, ids=None):
        ids = np.arange(self._n) if ids is None else np.asarray(ids)
        return self.done[ids] - self.arrival[ids]


def one_call_loop(requests, S=None, arrival=None, t0=None):
    """The baseline the serving loop is compared against: every request in
    arrival order as its own drop-in call on the current stream (the
    reference's way), waiting for each arrival time.  ``requests`` is a list of
    (op, x, aux).  Returns (results, completion events)."""
    results, events = [], []
    t0 = time.perf_counter() if t0 is None else t0
    for i, (op, x, aux) in enumerate(requests):
        if arrival is not None:
            while time.perf_counter() - t0 < arrival[i]:
                pass
        s = tcuscan_ops._pick_S(S, x.dtype, x.numel(), op="seg" if op == SEG_SUM else "scan")
        if op == SCAN:
            r = tcuscan_ops.run_scan_multi_core(x, s)
        elif op == SEG_SUM:
            r = tcuscan_ops.run_seg_sum_multi_core(x, aux, s)
        else:
            r = tcuscan_ops.run_compress(x, aux, s)
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        results.append(r)
        events.append(ev)
    return results, events
