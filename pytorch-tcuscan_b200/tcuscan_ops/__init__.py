"""tcuscan_ops -- B200 (sm_100a) drop-in for the reference's ``tcuscan_ops`` module.

Same function names, argument order, defaults and output dtypes as the
reference pybind module (src/pybind11.cpp:36-142); CUDA tensors replace NPU
tensors.  Every ``run_*`` below launches hand-written sm_100a kernels through
the C ABI of libtcuscan.so (include/tcuscan.h).  Calls are asynchronous on the
current CUDA stream unless the output size must be read back (compress, flag
segmented sum), exactly where the reference also synchronises.

``S`` / ``s`` is the tile parameter of the reference: the row length of the
S x S triangular tile multiplied on the tensor cores, one of 16, 32, 64, 128;
``None`` or 0 selects the autotuned value.
"""
import torch

from . import _lib
from ._lib import TcuError, check, raise_device_error, stream_ptr, workspace, workspace_error  # noqa: F401

_VALID_S = (16, 32, 64, 128)


def _cuda_input(x, name="x"):
    if not isinstance(x, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if x.device.type != "cuda":
        raise ValueError(f"{name} must be a CUDA tensor (got {x.device})")
    x = x.contiguous()
    if x.data_ptr() % 16 != 0:
        x = x.clone()  # fresh allocation: 16-byte aligned for TMA
    return x


def _pick_S(S, dtype, n=None):
    if S is None or int(S) == 0:
        from tcuscan_b200 import autotune

        return autotune.best_S("scan", dtype, n)
    S = int(S)
    if S not in _VALID_S:
        raise ValueError(f"S must be one of {_VALID_S} (got {S})")
    return S


def _scan_out_dtype(dtype):
    if dtype == torch.int8:
        return torch.int32
    if dtype in (torch.float16, torch.float32, torch.bfloat16):
        return torch.float32
    raise TypeError(f"unsupported dtype {dtype}: scans take int8, float16 or float32")


def _after(x):
    if _lib.SYNC_CHECK:
        raise_device_error(x.device)


def _scan(x, S, start, where):
    x = _cuda_input(x)
    n = x.numel()
    out_dtype = _scan_out_dtype(x.dtype)
    z = torch.empty(n, dtype=out_dtype, device=x.device)
    if n == 0:
        return z
    S = _pick_S(S, x.dtype, n)
    ws, wsb = workspace(x.device, _lib.lib.tcu_workspace_bytes(n, S))
    st = _lib.lib.tcu_scan(
        x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, S, float(start), z.data_ptr(), ws, wsb, stream_ptr(x.device)
    )
    check(st, where)
    _after(x)
    return z


def run_scan_multi_core(x, S):
    """Inclusive prefix sum of a 1-D tensor (reference: src/torch/torch_scan.h:184-241).

    int8 -> int32 (exact), float16 -> float32.  One persistent tensor-core
    launch with a decoupled look-back (the reference's three phases + grid
    barrier + L2 chunk loop collapse into a single pass)."""
    return _scan(x, S, 0.0, "run_scan_multi_core")


def run_scan_multi_core_no_l2(x, S):
    """Same as run_scan_multi_core (reference: src/torch/torch_scan.h:253-304).

    The reference variant only differs by skipping its L2 chunking loop, which
    a single-pass look-back scan does not have."""
    return _scan(x, S, 0.0, "run_scan_multi_core_no_l2")


def run_scan_single_core(x, S, starting_sum=0):
    """Prefix sum plus a starting value (reference: src/torch/torch_scan.h:47-110)."""
    return _scan(x, S, starting_sum, "run_scan_single_core")


def _check_tri(upper, lower_strict):
    if upper.dim() != 2 or upper.shape[0] != upper.shape[1]:
        raise ValueError("upper must be a square S x S matrix")
    if lower_strict.shape != upper.shape:
        raise ValueError("lower_strict must have the shape of upper")
    return int(upper.shape[0])


def run_scan_multi_cube(x, upper, lower_strict):
    """Prefix sum with the tile size taken from ``upper`` (reference:
    src/torch/torch_scan.h:416-466).  ``upper``/``lower_strict`` are the
    reference's caller-provided triu(ones)/tril(ones, -1); the kernel builds the
    same constant operand on chip, so only their shape is read."""
    S = _check_tri(upper, lower_strict)
    x = _cuda_input(x)
    if x.dtype != torch.float16:
        raise TypeError("run_scan_multi_cube: x must be float16")
    return _scan(x, S, 0.0, "run_scan_multi_cube")


def run_row_scan(x, S):
    """Scan of every length-S row (reference: src/torch/torch_scan.h:312-351).

    x is [M, S]; returns the flat [M*S] row prefixes (float16 -> float32,
    int8 -> int32)."""
    x = _cuda_input(x)
    S = _pick_S(S, x.dtype)
    if x.numel() % S != 0:
        raise ValueError(f"run_row_scan: numel {x.numel()} is not a multiple of S={S}")
    m = x.numel() // S
    out_dtype = _scan_out_dtype(x.dtype)
    z = torch.empty(m * S, dtype=out_dtype, device=x.device)
    if m == 0:
        return z
    ws, wsb = workspace(x.device, _lib.lib.tcu_workspace_bytes(m * S, S))
    st = _lib.lib.tcu_row_scan(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], m, S, z.data_ptr(), ws, wsb,
                               stream_ptr(x.device))
    check(st, "run_row_scan")
    _after(x)
    return z


def run_block_scan(x, upper, lower_strict):
    """Scan of every consecutive S*S block; n % S*S == 0 (reference:
    src/torch/torch_scan.h:362-405, kernel_block_scan.h:62-67)."""
    S = _check_tri(upper, lower_strict)
    x = _cuda_input(x)
    n = x.numel()
    if n % (S * S) != 0:
        raise ValueError(f"run_block_scan: numel {n} must be a multiple of S*S={S * S}")
    z = torch.empty(n, dtype=_scan_out_dtype(x.dtype), device=x.device)
    if n == 0:
        return z
    ws, wsb = workspace(x.device, _lib.lib.tcu_workspace_bytes(n, S))
    st = _lib.lib.tcu_block_scan(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, S, z.data_ptr(), ws, wsb,
                                 stream_ptr(x.device))
    check(st, "run_block_scan")
    _after(x)
    return z


def run_gen_lower(matrix_size, device, dtype):
    """torch.tril(ones(s, s)) (reference: src/torch/torch_gen_lower.h:31-59)."""
    return torch.tril(torch.ones((int(matrix_size), int(matrix_size)), dtype=dtype, device=device))


def run_scan_cpu(x):
    """The reference's CPU scan API (src/torch/torch_scan_cpu.h:88-107):
    float16/float32 -> float32, int8 -> int32, computed on the host.  This is
    a CPU operator of the reference's interface, not a fallback for any CUDA
    operator above."""
    if x.device.type != "cpu":
        raise ValueError("run_scan_cpu expects a CPU tensor")
    out = torch.float32 if x.dtype in (torch.float16, torch.float32) else torch.int32
    return torch.cumsum(x.to(out), dim=0)


__all__ = [n for n in dir() if n.startswith("run_")] + ["TcuError", "workspace_error", "raise_device_error"]
