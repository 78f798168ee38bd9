"""Inclusive scan of one array sharded over the ranks of a process group.

The reference scans one array on one device.  Split over GPUs, the scan has a
single exchange step: every rank needs the total of the ranks before it.

    z_local = scan_sharded(x_local)        # rank r holds the r-th piece

1. the local total (tcu_total: exact int64 for int8 input, a fixed-order
   FP64 sum for fp16 / fp32);
2. one all_gather of that scalar (NCCL over NVLink, one value per rank);
3. the exclusive prefix of the totals, on the device, in int64 / FP64;
4. one tensor-core scan of the local piece that reads the prefix as its start
   value from device memory (tcu_scan_chained_typed with an int64 / FP64
   start), so nothing returns to the host.  The carry between ranks is FP64,
   like the carry chain between tiles inside one GPU; int8 -> int32 results
   wrap in two's complement exactly as the unsharded scan's do.

The result on rank r is the r-th piece of the scan of the concatenation of
all pieces in rank order.  Each rank pays one extra read of its input for the
total (no second pass over the output).
"""
import torch

import tcuscan_ops
from tcuscan_ops import _lib


def total_dtype(dtype):
    """dtype of the exchanged totals: int64 for int8 pieces, float64 otherwise."""
    return torch.int64 if dtype == torch.int8 else torch.float64


def _local_total(x):
    """Total of the local piece (1-element int64 / float64 tensor)."""
    out = torch.zeros(1, dtype=total_dtype(x.dtype), device=x.device)
    n = x.numel()
    if n == 0:
        return out
    ws, wsb, sp = _lib.launch_context(x.device, _lib.lib.tcu_workspace_bytes(n, 64))
    tcuscan_ops.check(_lib.lib.tcu_total(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, out.data_ptr(), ws, wsb, sp),
                      "scan_sharded total")
    return out


def _local_scan(x, S, prefix):
    """Scan of the local piece starting from the device scalar `prefix`
    (int64 / float64)."""
    n = x.numel()
    z = torch.empty(n, dtype=tcuscan_ops._scan_out_dtype(x.dtype), device=x.device)
    if n == 0:
        return z
    S = tcuscan_ops._pick_S(S, x.dtype, n)
    ws, wsb, sp = _lib.launch_context(x.device, _lib.lib.tcu_workspace_bytes(n, S))
    tcuscan_ops.check(_lib.lib.tcu_scan_chained_typed(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, S, 0.0,
                                                      prefix.data_ptr(), _lib.DTYPE_CODE[prefix.dtype], z.data_ptr(),
                                                      ws, wsb, sp), "scan_sharded")
    return z


def exclusive_prefix(totals, rank):
    """Sum of the totals of ranks before `rank`, in the totals' dtype (int64
    or float64, summed in rank order)."""
    if rank == 0:
        return torch.zeros_like(totals[0])
    acc = totals[0].clone()
    for t in totals[1:rank]:
        acc += t
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
