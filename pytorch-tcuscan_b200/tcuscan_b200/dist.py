"""Inclusive scan of one array sharded over the ranks of a process group.

The reference scans one array on one device.  Split over GPUs, the scan has a
single exchange step: every rank needs the total of the ranks before it.

    z_local = scan_sharded(x_local)        # rank r holds the r-th piece

1. the local total (tcu_seg_sum_rows over the one segment [0, n): exact int32
   for int8 input, a fixed-order FP32 sum for fp16 / fp32);
2. one all_gather of that scalar (NCCL over NVLink, one value per rank);
3. the exclusive prefix of the totals, on the device (int32 sums wrap as the
   int8 -> int32 scan does);
4. one tensor-core scan of the local piece that reads the prefix as its start
   value from device memory (tcu_scan_chained), so nothing returns to the host.

The result on rank r is the r-th piece of the scan of the concatenation of
all pieces in rank order.  Each rank pays one extra read of its input for the
total (no second pass over the output).
"""
import torch

import tcuscan_ops
from tcuscan_ops import _lib


def _local_total(x):
    """Total of the local piece in the scan's output dtype (1-element tensor)."""
    out = torch.zeros(1, dtype=tcuscan_ops._scan_out_dtype(x.dtype), device=x.device)
    n = x.numel()
    if n == 0:
        return out
    bounds = torch.tensor([0, n], dtype=torch.int64, device=x.device)
    ws, wsb = tcuscan_ops.workspace(x.device, _lib.lib.tcu_rows_workspace_bytes(n))
    tcuscan_ops.check(_lib.lib.tcu_seg_sum_rows(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, bounds.data_ptr(),
                                                _lib.TCU_INT64, 2, out.data_ptr(), ws, wsb,
                                                tcuscan_ops.stream_ptr(x.device)), "scan_sharded total")
    return out


def _local_scan(x, S, prefix):
    """Scan of the local piece starting from the device scalar `prefix`."""
    n = x.numel()
    z = torch.empty(n, dtype=prefix.dtype, device=x.device)
    if n == 0:
        return z
    S = tcuscan_ops._pick_S(S, x.dtype, n)
    ws, wsb = tcuscan_ops.workspace(x.device, _lib.lib.tcu_workspace_bytes(n, S))
    tcuscan_ops.check(_lib.lib.tcu_scan_chained(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, S, 0.0, prefix.data_ptr(),
                                                z.data_ptr(), ws, wsb, tcuscan_ops.stream_ptr(x.device)),
                      "scan_sharded")
    return z


def exclusive_prefix(totals, rank):
    """Sum of the totals of ranks before `rank`, in the totals' dtype (int32
    wraps like the int8 -> int32 scan)."""
    if rank == 0:
        return torch.zeros_like(totals[0])
    acc = totals[0].clone()
    for t in totals[1:rank]:
        acc += t  # int32 + int32 wraps in two's complement
    return acc


def scan_sharded(x_local, S=None, group=None):
    """Inclusive scan of the concatenation of every rank's `x_local` (int8,
    fp16 or fp32; 1-D; any length per rank): returns this rank's piece of it.
    One all_gather of one scalar per rank; all ranks must call it."""
    import torch.distributed as dist

    x = tcuscan_ops._cuda_input(x_local) if x_local.device.type == "cuda" else x_local
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    total = _local_total(x)
    gathered = [torch.empty_like(total) for _ in range(world)]
    dist.all_gather(gathered, total, group=group)
    return _local_scan(x, S, exclusive_prefix(gathered, rank))
