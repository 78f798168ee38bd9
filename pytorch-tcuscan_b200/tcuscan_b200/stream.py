"""Scans of host-resident data with the copies overlapped.

A scan of data that lives in host memory is bound by PCIe: on B200 the
input copy, the kernel and the (4x larger, int32/fp32) output copy of a
2^28-element int8 scan take ~5 ms, 0.25 ms and ~19 ms one after another.
``scan_host`` splits the input into chunks and runs three CUDA streams --
host-to-device copies, scans, device-to-host copies -- so the two copy
directions and the kernels overlap (the copy engines are full duplex).  Each
chunk's scan takes the previous chunk's last output as its starting value
from device memory (``tcu_scan_chained``), so the chunks are chained without
a host round trip and the result is the scan of the whole input.  The
reference's scans work on device tensors only; this is the host-buffer entry
point of this implementation.
"""
import ctypes

import torch

import tcuscan_ops
from tcuscan_ops import _lib


class HostScanner:
    """Reusable device buffers, streams and events for ``scan_host`` on
    inputs of up to `capacity` elements of `dtype`."""

    def __init__(self, capacity, dtype, device="cuda", chunk=1 << 24):
        self.dev = torch.device(device)
        if self.dev.index is None:
            self.dev = torch.device("cuda", torch.cuda.current_device())
        self.dtype = dtype
        self.out_dtype = tcuscan_ops._scan_out_dtype(dtype)
        self.capacity = int(capacity)
        self.chunk = int(chunk)
        self.x = torch.empty(self.capacity, dtype=dtype, device=self.dev)
        self.z = torch.empty(self.capacity, dtype=self.out_dtype, device=self.dev)
        self.s_in = torch.cuda.Stream(self.dev)
        self.s_scan = torch.cuda.Stream(self.dev)
        self.s_out = torch.cuda.Stream(self.dev)
        nchunks = (self.capacity + self.chunk - 1) // self.chunk
        self.ev_in = [torch.cuda.Event() for _ in range(nchunks)]
        self.ev_scan = [torch.cuda.Event() for _ in range(nchunks)]
        self.ev_done = torch.cuda.Event()
        with torch.cuda.stream(self.s_scan):
            self.ws, self.wsb = _lib.workspace(self.dev, _lib.lib.tcu_workspace_bytes(self.chunk, 64))

    def scan(self, x_host, out_host, S=None, start=0.0):
        """Inclusive scan of `x_host` (pinned, 1-D) into `out_host` (pinned,
        int32 for int8 input, fp32 otherwise).  Asynchronous: returns an event
        the caller's stream can wait on (the current stream already does)."""
        n = x_host.numel()
        if n > self.capacity or x_host.dtype != self.dtype or out_host.dtype != self.out_dtype:
            raise ValueError("scan_host: input larger than the scanner or of another dtype")
        if out_host.numel() != n:
            raise ValueError("scan_host: output length differs from the input")
        cur = torch.cuda.current_stream(self.dev)
        for s_ in (self.s_in, self.s_scan, self.s_out):
            s_.wait_stream(cur)  # earlier work on these buffers is ordered first
        S = tcuscan_ops._pick_S(S, self.dtype, n)
        code = _lib.DTYPE_CODE[self.dtype]
        es = torch.empty((), dtype=self.out_dtype).element_size()
        nchunks = (n + self.chunk - 1) // self.chunk
        for k in range(nchunks):
            a, b = k * self.chunk, min(n, (k + 1) * self.chunk)
            with torch.cuda.stream(self.s_in):
                self.x[a:b].copy_(x_host[a:b], non_blocking=True)
                self.ev_in[k].record(self.s_in)
            self.s_scan.wait_event(self.ev_in[k])
            start_dev = self.z.data_ptr() + (a - 1) * es if k > 0 else None
            st = _lib.lib.tcu_scan_chained(self.x.data_ptr() + a * self.x.element_size(), code, b - a, S,
                                           float(start) if k == 0 else 0.0, start_dev,
                                           self.z.data_ptr() + a * es, self.ws, self.wsb,
                                           ctypes.c_void_p(self.s_scan.cuda_stream))
            tcuscan_ops.check(st, "scan_host")
            self.ev_scan[k].record(self.s_scan)
            self.s_out.wait_event(self.ev_scan[k])
            with torch.cuda.stream(self.s_out):
                out_host[a:b].copy_(self.z[a:b], non_blocking=True)
        self.ev_done.record(self.s_out)
        cur.wait_event(self.ev_done)
        return self.ev_done


def scan_host(x_host, out_host=None, S=None, start=0.0, chunk=1 << 24):
    """One-shot form of ``HostScanner``: allocates the device buffers and a
    pinned output if none is given, runs the overlapped scan and waits."""
    sc = HostScanner(x_host.numel(), x_host.dtype, chunk=chunk)
    if out_host is None:
        out_host = torch.empty(x_host.numel(), dtype=sc.out_dtype, pin_memory=True)
    sc.scan(x_host, out_host, S, start)
    torch.cuda.current_stream(sc.dev).synchronize()
    return out_host
