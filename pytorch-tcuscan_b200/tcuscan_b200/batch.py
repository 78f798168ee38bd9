"""Batched scans over rows of uneven length, in one persistent launch.

``scan_rows(x, offsets)`` scans every row x[offsets[b]:offsets[b+1]] of a flat
tensor (float16, float32 or int8; float32 uses split-precision bf16 hi + lo
tensor-core operands with FP32 accumulation and FP64 carries between tiles).
All rows are segments of one tensor-core launch, so thousands of uneven rows
cost one kernel.  ``ScanRowsGraph`` captures that launch (and its output
buffer) in a CUDA graph for repeated calls on fixed shapes.

This extends the reference's run_scan_batch (src/torch/torch_scan.h:119-175),
which handles uniform rows only.
"""
import torch

import tcuscan_ops
from tcuscan_ops import _lib


def scan_rows(x, offsets, S=None, out=None):
    """Row-wise inclusive scans of x[offsets[b]:offsets[b+1]] (flat x, int32/int64 offsets).

    Elements outside [offsets[0], offsets[-1]) are scanned as their own
    segments.  Returns a flat float32 (int32 for int8) tensor like x."""
    x = tcuscan_ops._cuda_input(x)
    offsets = tcuscan_ops._bounds_input(offsets, x.device, "scan_rows")
    n = x.numel()
    if out is None:
        out = torch.empty(n, dtype=tcuscan_ops._scan_out_dtype(x.dtype), device=x.device)
    if n == 0 or offsets.numel() == 0:
        return out
    S = tcuscan_ops._pick_S(S, x.dtype, n, op="seg")
    ws, wsb = tcuscan_ops.workspace(x.device, _lib.lib.tcu_workspace_bytes(n, S))
    st = _lib.lib.tcu_seg_bounds(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, S, offsets.data_ptr(),
                                 _lib.DTYPE_CODE[offsets.dtype], offsets.numel(), 0, out.data_ptr(), ws, wsb,
                                 tcuscan_ops.stream_ptr(x.device))
    tcuscan_ops.check(st, "scan_rows")
    return out


class ScanRowsGraph:
    """A CUDA graph holding one scan_rows launch on fixed (x, offsets) buffers.

    Refill ``self.x`` / ``self.offsets`` in place and call ``replay()``; the
    result is in ``self.out``.  The look-back workspace is self-resetting
    (epoch-tagged), so replays need no memset node."""

    def __init__(self, x, offsets, S=None):
        self.x = tcuscan_ops._cuda_input(x)
        self.offsets = tcuscan_ops._bounds_input(offsets, self.x.device, "ScanRowsGraph")
        self.out = torch.empty(self.x.numel(), dtype=tcuscan_ops._scan_out_dtype(self.x.dtype), device=self.x.device)
        self.S = S
        self.stream = torch.cuda.Stream(self.x.device)
        self.stream.wait_stream(torch.cuda.current_stream(self.x.device))
        with torch.cuda.stream(self.stream):
            scan_rows(self.x, self.offsets, S, self.out)  # warm-up: workspace + kernel attributes
        self.stream.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=self.stream):
            scan_rows(self.x, self.offsets, S, self.out)

    def replay(self):
        self.graph.replay()
        return self.out
