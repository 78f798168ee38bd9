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
import os

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


def _pick_S(S, dtype, n=None, op="scan"):
    """S for a launch: validated when given; from the autotuner's table when
    None or 0 (which also applies its tuned CTA count; an explicit S runs
    with one CTA per SM)."""
    from tcuscan_b200 import autotune

    if S is None or int(S) == 0:
        S, ctas = autotune.best(op, dtype, n)
        autotune.apply_ctas(ctas)
        return S
    S = int(S)
    if S not in _VALID_S:
        raise ValueError(f"S must be one of {_VALID_S} (got {S})")
    autotune.apply_ctas(0)
    return S


def _scan_out_dtype(dtype):
    if dtype == torch.int8:
        return torch.int32
    if dtype in (torch.float16, torch.float32):
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
    ws, wsb, sp = _lib.launch_context(x.device, _lib.lib.tcu_workspace_bytes(n, S))
    st = _lib.lib.tcu_scan(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, S, float(start), z.data_ptr(), ws, wsb, sp)
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
    src/torch/torch_scan.h:362-405, kernel_block_scan.h:62-67).

    float16 at S = 64 / 128 runs the reference's tensor-only formulation
    (tcu_block_scan_tensor: z = A.upper + lower_strict.(A.J) per tile, every
    product on the tensor cores, the caller's matrices used as given);
    other S and int8 run the scan engine's block mode, which builds the
    standard triangular operand on chip and reads only the matrices' shape."""
    S = _check_tri(upper, lower_strict)
    x = _cuda_input(x)
    n = x.numel()
    if n % (S * S) != 0:
        raise ValueError(f"run_block_scan: numel {n} must be a multiple of S*S={S * S}")
    z = torch.empty(n, dtype=_scan_out_dtype(x.dtype), device=x.device)
    if n == 0:
        return z
    if x.dtype == torch.float16 and S in (64, 128):
        up = _cuda_input(upper.to(device=x.device, dtype=torch.float16), "upper")
        lo = _cuda_input(lower_strict.to(device=x.device, dtype=torch.float16), "lower_strict")
        ws, wsb, sp = _lib.launch_context(x.device, 256)
        st = _lib.lib.tcu_block_scan_tensor(x.data_ptr(), _lib.TCU_FLOAT16, n, S, up.data_ptr(), lo.data_ptr(),
                                            z.data_ptr(), ws, wsb, sp)
        check(st, "run_block_scan")
        _after(x)
        return z
    ws, wsb = workspace(x.device, _lib.lib.tcu_workspace_bytes(n, S))
    st = _lib.lib.tcu_block_scan(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, S, z.data_ptr(), ws, wsb,
                                 stream_ptr(x.device))
    check(st, "run_block_scan")
    _after(x)
    return z


def run_gen_lower(matrix_size, device, dtype):
    """tril(ones(s, s)) on the device (reference: src/torch/torch_gen_lower.h:31-59)."""
    s_ = int(matrix_size)
    dev = torch.device(device)
    z = torch.empty((s_, s_), dtype=dtype, device=dev)
    if dtype not in _lib.DTYPE_CODE:
        raise TypeError(f"run_gen_lower: unsupported dtype {dtype}")
    check(_lib.lib.tcu_gen_lower(s_, _lib.DTYPE_CODE[dtype], z.data_ptr(), stream_ptr(dev)), "run_gen_lower")
    return z


# ---------------------------------------------------------------------------
# stream compaction (src/torch/torch_compress.h)

def _mask_input(mask, n, x_device):
    mask = _cuda_input(mask, "mask")
    if mask.device != x_device:
        raise ValueError("mask must be on the device of x")
    if mask.dtype in (torch.bool, torch.uint8):
        mask = mask.view(torch.int8)
    if mask.dtype != torch.int8:
        raise TypeError(f"mask must be int8 (or bool/uint8), got {mask.dtype}")
    if mask.numel() != n:
        raise ValueError(f"mask has {mask.numel()} elements, x has {n}")
    return mask


def _count(mask):
    n = mask.numel()
    cnt = torch.empty(1, dtype=torch.int64, device=mask.device)
    check(_lib.lib.tcu_mask_count(mask.data_ptr(), n, cnt.data_ptr(), stream_ptr(mask.device)), "mask count")
    return cnt


def _compress(x, mask, out_len, idx_in=None, idx_mode=0, idx_dtype=torch.int32, where="run_compress"):
    """Compaction into outputs of out_len elements (None: sized by a count
    pass read back to the host, as the reference sizes its outputs)."""
    n = x.numel()
    ib = 0
    if idx_mode == 1:
        ib = idx_in.element_size()
    elif idx_mode == 2:
        ib = torch.empty((), dtype=idx_dtype).element_size()
    sp = stream_ptr(x.device)
    from tcuscan_b200 import autotune

    autotune.apply_ctas(autotune.best("compress", x.dtype, n)[1])
    ws, wsb = workspace(x.device, _lib.lib.tcu_workspace_bytes(n, 64))
    counted = out_len is None
    if counted:
        cnt = torch.empty(1, dtype=torch.int64, device=x.device)
        check(_lib.lib.tcu_compress_count(mask.data_ptr(), n, x.element_size(), idx_mode, ib, cnt.data_ptr(), ws, wsb,
                                          sp), where)
        out_len = int(cnt.item())
    z = torch.empty(out_len, dtype=x.dtype, device=x.device)
    idx_out = None
    if idx_mode == 1:
        idx_out = torch.empty(out_len, dtype=idx_in.dtype, device=x.device)
    elif idx_mode == 2:
        idx_out = torch.empty(out_len, dtype=idx_dtype, device=x.device)
    if n == 0:
        return z, idx_out
    zp = z.data_ptr() if out_len > 0 else x.data_ptr()
    ip = (idx_out.data_ptr() if out_len > 0 else x.data_ptr()) if idx_out is not None else None
    inp = idx_in.data_ptr() if idx_in is not None else None
    if counted:
        st = _lib.lib.tcu_compress_counted(x.data_ptr(), x.element_size(), mask.data_ptr(), n, inp, ib, idx_mode, zp,
                                           ip, out_len, ws, wsb, sp)
    else:
        st = _lib.lib.tcu_compress(x.data_ptr(), x.element_size(), mask.data_ptr(), n, inp, ib, idx_mode, zp, ip,
                                   out_len, None, ws, wsb, sp)
    check(st, where)
    _after(x)
    return z, idx_out


def _check_S_opt(S):
    if S is not None and int(S) != 0:
        _pick_S(S, torch.float16)


def run_compress(x, mask, S):
    """Stable x[mask != 0] (reference: src/torch/torch_compress.h:41-98).

    The reference selects mask == 1 and sizes the output with sum(mask); both
    agree for 0/1 masks.  One count pass (read back to size the output, as
    the reference does) and one streaming compaction pass."""
    _check_S_opt(S)
    x = _cuda_input(x)
    mask = _mask_input(mask, x.numel(), x.device)
    return _compress(x, mask, None)[0]


def run_compress_pos(x, mask, output_len, S):
    """Compaction into an output of the given length (reference:
    src/torch/torch_compress.h:109-161); no host round trip."""
    _check_S_opt(S)
    x = _cuda_input(x)
    mask = _mask_input(mask, x.numel(), x.device)
    return _compress(x, mask, int(output_len), where="run_compress_pos")[0]


def run_compress_ind(x, indices_in, mask, S):
    """(x[mask], indices_in[mask]) (reference: src/torch/torch_compress.h:172-239)."""
    _check_S_opt(S)
    x = _cuda_input(x)
    indices_in = _cuda_input(indices_in, "indices_in")
    if indices_in.numel() != x.numel():
        raise ValueError("indices_in must have the length of x")
    if indices_in.element_size() not in (4, 8):
        raise TypeError("indices_in must be a 32- or 64-bit integer tensor")
    mask = _mask_input(mask, x.numel(), x.device)
    z, idx = _compress(x, mask, None, idx_in=indices_in, idx_mode=1, where="run_compress_ind")
    return z, idx


def run_compress_ind_no_arange(x, mask, S):
    """(x[mask], positions of the selected elements as int32) (reference:
    src/torch/torch_compress.h:249-309)."""
    _check_S_opt(S)
    x = _cuda_input(x)
    mask = _mask_input(mask, x.numel(), x.device)
    return _compress(x, mask, None, idx_mode=2, where="run_compress_ind_no_arange")


def run_filter_greater_eq(x, pivot, S):
    """x[x >= pivot] (reference: src/torch/torch_compress.h:319-323)."""
    x = _cuda_input(x)
    return run_compress(x, (x >= pivot).to(torch.int8), S)


def run_filter_less_eq(x, pivot, S):
    """x[x <= pivot] (reference: src/torch/torch_compress.h:333-337)."""
    x = _cuda_input(x)
    return run_compress(x, (x <= pivot).to(torch.int8), S)


def run_where(x, pivot, S):
    """int32 positions where x >= pivot (reference: src/torch/torch_compress.h:347-398)."""
    x = _cuda_input(x)
    return run_compress_ind_no_arange(x, (x >= pivot).to(torch.int8), S)[1]


# ---------------------------------------------------------------------------
# split, radix sort, top-k (src/torch/torch_split.h, torch_sort.h, torch_topk.h)

def _split(x, mask, indices_in, where):
    n = x.numel()
    z = torch.empty_like(x)
    idx_out = torch.empty_like(indices_in) if indices_in is not None else None
    if n == 0:
        return z, idx_out
    from tcuscan_b200 import autotune

    autotune.apply_ctas(autotune.best("compress", x.dtype, n)[1])
    ib = indices_in.element_size() if indices_in is not None else 0
    ws, wsb = workspace(x.device, _lib.lib.tcu_workspace_bytes(n, 64))
    check(_lib.lib.tcu_split(x.data_ptr(), x.element_size(), mask.data_ptr(), n,
                             indices_in.data_ptr() if indices_in is not None else None, ib,
                             1 if indices_in is not None else 0, z.data_ptr(),
                             idx_out.data_ptr() if idx_out is not None else None, None, ws, wsb,
                             stream_ptr(x.device)), where)
    _after(x)
    return z, idx_out


def run_split(x, mask, S):
    """Stable partition: x[mask != 0] followed by x[mask == 0], n elements
    (reference: src/torch/torch_split.h:33-79, 16-bit dtypes only there; any
    1/2/4/8-byte dtype here).  One count pass, one offset scan, one streaming
    pass writing both runs; asynchronous (the reference synchronises)."""
    _check_S_opt(S)
    x = _cuda_input(x)
    mask = _mask_input(mask, x.numel(), x.device)
    return _split(x, mask, None, "run_split")[0]


def run_split_ind(x, mask, indices_in, S):
    """(split of x, indices_in permuted the same way) (reference:
    src/torch/torch_split.h:91-142; indices int32 there, int32 or int64
    here)."""
    _check_S_opt(S)
    x = _cuda_input(x)
    mask = _mask_input(mask, x.numel(), x.device)
    indices_in = _cuda_input(indices_in, "indices_in")
    if indices_in.numel() != x.numel():
        raise ValueError("indices_in must have the length of x")
    if indices_in.dtype not in (torch.int32, torch.int64):
        raise TypeError(f"indices_in must be int32 or int64, got {indices_in.dtype}")
    return _split(x, mask, indices_in, "run_split_ind")


_SORT_DTYPES = (torch.int8, torch.uint8, torch.int16, torch.float16, torch.bfloat16, torch.int32, torch.float32)


def run_radix_sort(x, S):
    """(ascending stable sort of x, int32 positions) (reference:
    src/torch/torch_sort.h:30-82; fp16 / int16 and lengths that are multiples
    of the tile there).  Byte-digit LSD passes: two for 16-bit keys.  Floats
    follow the reference's bit encoding: -0 sorts below +0, NaNs with the
    sign bit first and the others last."""
    _check_S_opt(S)
    x = _cuda_input(x)
    if x.dtype not in _SORT_DTYPES:
        raise TypeError(f"run_radix_sort: unsupported dtype {x.dtype}")
    n = x.numel()
    if n > 0x7FFFFFFF:
        raise ValueError("run_radix_sort: more than 2^31 - 1 elements (int32 positions)")
    out = torch.empty_like(x)
    idx = torch.empty(n, dtype=torch.int32, device=x.device)
    if n == 0:
        return out, idx
    code = _lib.DTYPE_CODE[x.dtype]
    tb = _lib.lib.tcu_radix_sort_tmp_bytes(code, n)
    tmp = torch.empty(tb, dtype=torch.uint8, device=x.device)
    check(_lib.lib.tcu_radix_sort(x.data_ptr(), code, n, out.data_ptr(), idx.data_ptr(), tmp.data_ptr(), tb,
                                  stream_ptr(x.device)), "run_radix_sort")
    _after(x)
    return out, idx


def _topk(x, k, dtype, where):
    x = _cuda_input(x)
    if x.dtype != dtype:
        raise TypeError(f"{where}: x must be {dtype}, got {x.dtype}")
    n = x.numel()
    k = int(k)
    if k < 0 or k > n:
        raise ValueError(f"{where}: k = {k} outside [0, {n}]")
    if n > 0x7FFFFFFF:
        raise ValueError(f"{where}: more than 2^31 - 1 elements (int32 positions)")
    out = torch.empty(k, dtype=x.dtype, device=x.device)
    idx = torch.empty(k, dtype=torch.int32, device=x.device)
    if k == 0:
        return out, idx
    tb = _lib.lib.tcu_topk_tmp_bytes(n)
    tmp = torch.empty(tb, dtype=torch.uint8, device=x.device)
    check(_lib.lib.tcu_topk(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, k, out.data_ptr(), idx.data_ptr(),
                            tmp.data_ptr(), tb, stream_ptr(x.device)), where)
    _after(x)
    return out, idx


def run_topk_int16(x, k, x_min, x_max, S):
    """(k largest of x, int32 positions), in input order (reference:
    src/torch/torch_topk.h:86-145, which bisects [x_min, x_max] with repeated
    splits and returns the same set band by band).  Ties at the k-th value
    keep the lowest positions, as the reference's stable splits do.  x_min and
    x_max are accepted for the signature; the radix select does not need
    them."""
    _check_S_opt(S)
    return _topk(x, k, torch.int16, "run_topk_int16")


def run_topk_fp16(x, k, x_min, x_max, S):
    """fp16 form of run_topk_int16 (reference: src/torch/torch_topk.h:157-211).
    NaN ranks above every number; -0 and +0 are equal."""
    _check_S_opt(S)
    return _topk(x, k, torch.float16, "run_topk_fp16")


def run_topk_pivot_fp16(x, k, num_samples=32):
    """Per-block lower-bound estimates of the k-th largest value (reference:
    src/torch/torch_topk.h:35-73; k is ignored there too, k_inner = 8,
    k_outer = 4).  One estimate per block, min(SM count, tiles of
    num_samples * 32 elements) blocks."""
    x = _cuda_input(x)
    if x.dtype != torch.float16:
        raise TypeError(f"run_topk_pivot_fp16: x must be float16, got {x.dtype}")
    n = x.numel()
    num_samples = int(num_samples)
    if n == 0 or num_samples <= 0:
        raise ValueError("run_topk_pivot_fp16: empty input or num_samples <= 0")
    b = _lib.lib.tcu_topk_pivot_blocks(n, num_samples)
    out = torch.empty(b, dtype=torch.float16, device=x.device)
    check(_lib.lib.tcu_topk_pivot(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, num_samples, 8, 4, out.data_ptr(),
                                  stream_ptr(x.device)), "run_topk_pivot_fp16")
    _after(x)
    return out


# ---------------------------------------------------------------------------
# gather (src/torch/torch_gather.h)

def run_csr_gather(values, cols, x):
    """z[i] = values[i] * x[cols[i]] in the values dtype (reference:
    src/torch/torch_gather.h:92-172, same argument checks).  x is read
    through L2, so unlike the reference it is not limited to what fits on
    chip."""
    if values.dim() != 1:
        raise ValueError(f"run_csr_gather: values must be 1D, got {values.dim()}D")
    if cols.dim() != 1:
        raise ValueError(f"run_csr_gather: cols must be 1D, got {cols.dim()}D")
    if x.dim() != 1:
        raise ValueError(f"run_csr_gather: x must be 1D, got {x.dim()}D")
    if cols.numel() != values.numel():
        raise ValueError(f"run_csr_gather: cols length ({cols.numel()}) must match values length ({values.numel()})")
    if values.dtype not in (torch.float16, torch.int16, torch.float32):
        raise TypeError(f"run_csr_gather: values dtype must be fp16, int16, or fp32, got {values.dtype}")
    if x.dtype != values.dtype:
        raise TypeError(f"run_csr_gather: x dtype ({x.dtype}) must match values dtype ({values.dtype})")
    if cols.dtype != torch.int32:
        raise TypeError(f"run_csr_gather: cols dtype must be int32, got {cols.dtype}")
    if not (values.is_contiguous() and cols.is_contiguous() and x.is_contiguous()):
        raise ValueError("run_csr_gather: values, cols and x must be contiguous")
    if values.device != cols.device or values.device != x.device:
        raise ValueError("run_csr_gather: values, cols and x must be on the same device")
    values, cols, x = _cuda_input(values, "values"), _cuda_input(cols, "cols"), _cuda_input(x)
    z = torch.empty_like(values)
    nnz = values.numel()
    if nnz == 0:
        return z
    ws, _ = workspace(x.device, 1 << 20)
    st = _lib.lib.tcu_csr_gather(values.data_ptr(), _lib.DTYPE_CODE[values.dtype], cols.data_ptr(), nnz,
                                 x.data_ptr(), x.numel(), z.data_ptr(), ws, stream_ptr(x.device))
    check(st, "run_csr_gather")
    _after(x)
    return z


# ---------------------------------------------------------------------------
# scan phases as standalone operators (src/torch/torch_reduce.h)

def run_gather_spmv(values, idxs, tile_len):
    """z[i] = values[idxs[i] - 1], 0 where idxs[i] == 0 (reference:
    src/torch/torch_gather.h:182-213; tests/test_gather_spmv.py).  Output has
    len(idxs) elements of the values dtype.  tile_len is the reference's
    vector-core tile and is validated but not needed here."""
    if int(tile_len) <= 0:
        raise ValueError("tile_len must be positive")
    values = _cuda_input(values, "values")
    idxs = _cuda_input(idxs, "idxs")
    if values.element_size() not in (2, 4, 8):
        raise TypeError(f"run_gather_spmv: unsupported values dtype {values.dtype}")
    code = _lib.DTYPE_CODE.get(idxs.dtype)
    if code not in (_lib.TCU_INT32, _lib.TCU_INT64, _lib.TCU_UINT32):
        raise TypeError(f"run_gather_spmv: indices must be int32, uint32 or int64, got {idxs.dtype}")
    z = torch.empty(idxs.numel(), dtype=values.dtype, device=values.device)
    if idxs.numel() == 0:
        return z
    ws, _ = workspace(values.device, 1 << 20)
    check(_lib.lib.tcu_gather_spmv(values.data_ptr(), values.element_size(), values.numel(), idxs.data_ptr(), code,
                                   idxs.numel(), z.data_ptr(), ws, stream_ptr(values.device)), "run_gather_spmv")
    _after(values)
    return z


def run_reduce_tiles(x, tile_len, num_blocks):
    """Per-block sums (reference: src/torch/torch_reduce.h:42-75):
    block = tile_len * ceil(ceil(n / tile_len) / num_blocks) elements;
    int8 -> int32, float16 -> float32."""
    x = _cuda_input(x)
    if x.dtype not in (torch.int8, torch.float16):
        raise TypeError(f"run_reduce_tiles: x must be int8 or float16, got {x.dtype}")
    tile_len, num_blocks = int(tile_len), int(num_blocks)
    if tile_len <= 0 or num_blocks <= 0:
        raise ValueError("run_reduce_tiles: tile_len and num_blocks must be positive")
    z = torch.empty(num_blocks, dtype=_scan_out_dtype(x.dtype), device=x.device)
    ws, wsb = workspace(x.device, 128 + 8 * num_blocks * 64)
    st = _lib.lib.tcu_reduce_tiles(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], x.numel(), tile_len, num_blocks,
                                   z.data_ptr(), ws, wsb, stream_ptr(x.device))
    check(st, "run_reduce_tiles")
    _after(x)
    return z


def run_complete_rows(x, sums, tile_width, tile_height):
    """MCSCAN down-sweep over rows (reference: src/torch/torch_reduce.h:143-182,
    semantics of tests/test_complete_rows.py ref_complete_rows).  x float32 ->
    float32, int32 -> int32 (the reference routes int64 keys to its int32
    kernel; here int64 is rejected)."""
    x = _cuda_input(x)
    sums = _cuda_input(sums, "sums")
    if x.dtype not in (torch.float32, torch.int32):
        raise TypeError(f"run_complete_rows: x must be float32 or int32, got {x.dtype}")
    sums = sums.to(x.dtype)
    nb = sums.numel()
    n = x.numel()
    if nb == 0 or n % nb != 0:
        raise ValueError("run_complete_rows: len(x) must be a multiple of len(sums)")
    width = int(tile_width)
    if width <= 0:
        raise ValueError(f"run_complete_rows: tile_width must be positive, got {width}")
    rows = (n // nb + width - 1) // width
    z = torch.empty(n, dtype=x.dtype, device=x.device)
    if n == 0:
        return z
    ws, wsb = workspace(x.device, 128 + 8 * nb * rows)
    st = _lib.lib.tcu_complete_rows(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, sums.data_ptr(), nb, width,
                                    z.data_ptr(), ws, wsb, stream_ptr(x.device))
    check(st, "run_complete_rows")
    _after(x)
    return z


def run_complete_blocks(x, sums, tile_length):
    """z[block b] = x[block b] + sum(sums[:b]) (reference:
    src/torch/torch_reduce.h:197-231).  float32 or int32."""
    x = _cuda_input(x)
    sums = _cuda_input(sums, "sums")
    if x.dtype not in (torch.float32, torch.int32):
        raise TypeError(f"run_complete_blocks: x must be float32 or int32, got {x.dtype}")
    sums = sums.to(x.dtype)
    nb, n = sums.numel(), x.numel()
    if nb == 0 or n % nb != 0:
        raise ValueError("run_complete_blocks: len(x) must be a multiple of len(sums)")
    z = torch.empty_like(x)
    if n == 0:
        return z
    st = _lib.lib.tcu_complete_blocks(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, sums.data_ptr(), nb, z.data_ptr(),
                                      stream_ptr(x.device))
    check(st, "run_complete_blocks")
    _after(x)
    return z


# ---------------------------------------------------------------------------
# segmented operators (src/torch/torch_seg_ops.h)

def _seg_x(x, where):
    x = _cuda_input(x)
    if x.dtype not in (torch.float16, torch.int8, torch.float32):
        raise TypeError(f"{where}: x must be float16, int8 or float32, got {x.dtype}")
    return x


def _flags_input(f, n, device, where):
    f = _cuda_input(f, "f")
    if f.device != device:
        raise ValueError(f"{where}: f must be on the device of x")
    if f.dtype in (torch.bool, torch.uint8):
        f = f.view(torch.int8)
    if f.dtype != torch.int8:
        raise TypeError(f"{where}: f must be int8, got {f.dtype}")
    if f.numel() != n:
        raise ValueError(f"{where}: f has {f.numel()} elements, x has {n}")
    return f


def _seg_scan_flags(x, f, S, ends, where):
    n = x.numel()
    z = torch.empty(n, dtype=_scan_out_dtype(x.dtype), device=x.device)
    if n == 0:
        return z
    S = _pick_S(S, x.dtype, n, op="seg")
    ws, wsb = workspace(x.device, _lib.lib.tcu_workspace_bytes(n, S))
    st = _lib.lib.tcu_seg_scan(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, S, f.data_ptr(), int(ends), z.data_ptr(),
                               ws, wsb, stream_ptr(x.device))
    check(st, where)
    _after(x)
    return z


def run_seg_scan(x, f, S):
    """Segmented scan; f[i] != 0 starts a segment at i (reference:
    src/torch/torch_seg_ops.h:165-193, single-core there).  One multi-CTA
    tensor-core launch; float16 -> float32 (int8 -> int32 as an extension)."""
    x = _seg_x(x, "run_seg_scan")
    f = _flags_input(f, x.numel(), x.device, "run_seg_scan")
    return _seg_scan_flags(x, f, S, False, "run_seg_scan")


def run_seg_sum(x, f, S):
    """Segmented sums; f[i] != 0 ENDS a segment at i, one output per end flag,
    elements after the last end are dropped (reference:
    src/torch/torch_seg_ops.h:85-107, semantics of tests/test_segmented_sum.py).

    The reference scans, compresses the scan at the flags and takes
    differences; here a segmented tensor-core scan yields each segment's sum
    at its end directly (no cancellation between large prefixes) and the
    single-pass compaction picks the ends."""
    x = _seg_x(x, "run_seg_sum")
    f = _flags_input(f, x.numel(), x.device, "run_seg_sum")
    k = int(_count(f).item())
    seg = _seg_scan_flags(x, f, S, True, "run_seg_sum")
    return _compress(seg, f, k, where="run_seg_sum")[0]


def _bounds_input(indptr, device, where):
    if not isinstance(indptr, torch.Tensor):
        raise TypeError(f"{where}: indptr must be a tensor")
    indptr = indptr.to(device)
    if hasattr(torch, "uint32") and indptr.dtype == torch.uint32:
        indptr = indptr.view(torch.int32)
    if indptr.dtype not in (torch.int32, torch.int64):
        raise TypeError(f"{where}: indptr must be int32, uint32 or int64, got {indptr.dtype}")
    return indptr.contiguous()


# Mean segment length up to which segment sums and SpMV take the element-split
# SIMT kernels (tcu_seg_sum_rows / tcu_spmv_rows: per-tile start/end bitmaps)
# instead of the tensor-core segmented sum; 0 = every length, a negative
# value = none (the tensor-core path for every length).  Measured on
# B200 at 2^28 fp16 (geometric segment lengths): the bitmap path takes 0.71 /
# 0.25 / 0.20 ms at mean 4 / 64 / 1024, the tensor-core path 0.48 / 0.36 ms
# at mean 64 / 1024, so the split path serves every length by default.
ROWS_MAX_MEAN = int(os.environ.get("TCU_ROWS_MAX_MEAN", "0"))


def _use_rows(n, nseg):
    if nseg <= 0 or ROWS_MAX_MEAN < 0:
        return False
    return ROWS_MAX_MEAN == 0 or n <= ROWS_MAX_MEAN * nseg


# float32 segment sums (and SpMV, whose products are float32) always take
# the element-split path: the tensor-core form takes segment sums as
# differences of bf16 hi + lo prefix sums, which carry ~1e-3 absolute error
# from the split representation accumulated along the prefix, while the split
# path sums in FP32; for SpMV it is also the faster one at every row length
# (both are bound by the x gathers).
ROWS_FP32 = os.environ.get("TCU_ROWS_FP32", "1") != "0"


def _rows_for(dtype, n, nseg):
    """Whether segment sums of `dtype` take the element-split path."""
    return nseg > 0 and ((ROWS_FP32 and dtype == torch.float32) or _use_rows(n, nseg))


def _rows_ws(device, n):
    """The stream's workspace, sized for the element-split row kernels."""
    return workspace(device, _lib.lib.tcu_rows_workspace_bytes(n))


def _seg_sum_bounds(x, bounds, S, where):
    x = _seg_x(x, where)
    bounds = _bounds_input(bounds, x.device, where)
    nb = bounds.numel()
    out = torch.empty(max(nb - 1, 0), dtype=_scan_out_dtype(x.dtype), device=x.device)
    if nb < 2:
        return out
    n = x.numel()
    if _rows_for(x.dtype, n, nb - 1):
        _check_S_opt(S)
        ws, wsb = _rows_ws(x.device, n)
        check(_lib.lib.tcu_seg_sum_rows(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, bounds.data_ptr(),
                                        _lib.DTYPE_CODE[bounds.dtype], nb, out.data_ptr(), ws, wsb,
                                        stream_ptr(x.device)), where)
        _after(x)
        return out
    S = _pick_S(S, x.dtype, n, op="seg")
    ws, wsb = workspace(x.device, _lib.lib.tcu_workspace_bytes(n, S))
    st = _lib.lib.tcu_seg_bounds(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], n, S, bounds.data_ptr(),
                                 _lib.DTYPE_CODE[bounds.dtype], nb, 1, out.data_ptr(), ws, wsb, stream_ptr(x.device))
    check(st, where)
    _after(x)
    return out


def run_seg_sum_multi_core(x, indptr, s, segm_offsets=None):
    """out[r] = sum x[indptr[r]:indptr[r+1]] for a CSR indptr of R+1 entries
    (reference: src/torch/torch_seg_ops.h:333-426).  float16 -> float32,
    int8 -> int32 (exact).  Empty segments give 0.  ``segm_offsets`` is the
    reference's per-core segment-range hint; segment boundaries are located
    on the device here (a per-tile search of indptr), so it is accepted for
    signature compatibility and not read."""
    return _seg_sum_bounds(x, indptr, s, "run_seg_sum_multi_core")


def run_seg_sum_single_core(x, indptr, s):
    """Same contract as run_seg_sum_multi_core (reference:
    src/torch/torch_seg_ops.h:211-266, one core there)."""
    return _seg_sum_bounds(x, indptr, s, "run_seg_sum_single_core")


def run_seg_sum_multi_cube(x, upper, lower_strict, indptr, segm_offsets=None):
    """Indptr segmented sum with S taken from ``upper`` (reference:
    src/torch/torch_seg_ops.h:443-522; float16 only there and here)."""
    S = _check_tri(upper, lower_strict)
    if x.dtype != torch.float16:
        raise TypeError(f"run_seg_sum_multi_cube: x must be fp16, got {x.dtype}")
    return _seg_sum_bounds(x, indptr, S, "run_seg_sum_multi_cube")


def run_seg_sum_single_cube(x, upper, lower_strict, indptr, s):
    """Segmented sum where ``indptr`` lists segment STARTS only (R entries, the
    last segment runs to the end of x) -- the convention of the reference's
    single-cube variant (src/torch/torch_seg_ops.h:278-322)."""
    _check_tri(upper, lower_strict)
    x = _cuda_input(x)
    starts = _bounds_input(indptr, x.device, "run_seg_sum_single_cube")
    bounds = torch.cat([starts, torch.tensor([x.numel()], dtype=starts.dtype, device=x.device)])
    return _seg_sum_bounds(x, bounds, s, "run_seg_sum_single_cube")


def run_scan_batch(x, S):
    """Row-wise scan of a 2-D [B, L] tensor (reference: src/torch/torch_scan.h:119-175):
    float16 -> float32.  Rows are segments of one tensor-core launch."""
    x = _cuda_input(x)
    if x.dim() < 1:
        raise ValueError("run_scan_batch: x must have at least one dimension")
    L = x.shape[-1]
    B = x.numel() // L if L else 0
    if x.dtype not in (torch.float16, torch.int8, torch.float32):
        raise TypeError(f"run_scan_batch: x must be float16, int8 or float32, got {x.dtype}")
    z = torch.empty((B, L), dtype=_scan_out_dtype(x.dtype), device=x.device)
    if B == 0 or L == 0:
        return z
    S = _pick_S(S, x.dtype, B * L, op="seg")
    ws, wsb = workspace(x.device, _lib.lib.tcu_workspace_bytes(B * L, S))
    st = _lib.lib.tcu_scan_batch(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], B, L, S, z.data_ptr(), ws, wsb,
                                 stream_ptr(x.device))
    check(st, "run_scan_batch")
    _after(x)
    return z


# ---------------------------------------------------------------------------
# CSR SpMV (src/torch/torch_spmv.h)

def _spmv(vals, indptr, cols, x, S, where):
    if vals.dtype != x.dtype or vals.dtype not in (torch.float16, torch.float32):
        raise TypeError(f"{where}: vals and x must both be fp16 or both be fp32, got vals={vals.dtype} x={x.dtype}")
    vals, x = _cuda_input(vals, "vals"), _cuda_input(x)
    cols = _cuda_input(cols, "cols")
    if hasattr(torch, "uint32") and cols.dtype == torch.uint32:
        cols = cols.view(torch.int32)
    if cols.dtype != torch.int32:
        cols = cols.to(torch.int32)
    indptr = _bounds_input(indptr, x.device, where)
    rows = indptr.numel() - 1
    nnz = vals.numel()
    if cols.numel() != nnz:
        raise ValueError(f"{where}: cols and vals lengths differ")
    y = torch.empty(max(rows, 0), dtype=torch.float32, device=x.device)
    if rows <= 0:
        return y
    if _rows_for(torch.float32, nnz, rows):
        _check_S_opt(S)
        ws, wsb = _rows_ws(x.device, nnz)
        check(_lib.lib.tcu_spmv_rows(vals.data_ptr(), _lib.DTYPE_CODE[vals.dtype], indptr.data_ptr(),
                                     _lib.DTYPE_CODE[indptr.dtype], rows, cols.data_ptr(), nnz, x.data_ptr(),
                                     x.numel(), y.data_ptr(), ws, wsb, stream_ptr(x.device)), where)
        _after(x)
        return y
    prod = torch.empty(max((nnz + 63) // 64 * 64, 64), dtype=torch.float32, device=x.device)  # pre-split rows
    S = _pick_S(S, torch.float32, nnz, op="seg")
    ws, wsb = workspace(x.device, _lib.lib.tcu_workspace_bytes(nnz, S))
    st = _lib.lib.tcu_spmv_csr(vals.data_ptr(), _lib.DTYPE_CODE[vals.dtype], indptr.data_ptr(),
                               _lib.DTYPE_CODE[indptr.dtype], rows, cols.data_ptr(), nnz, x.data_ptr(), x.numel(), S,
                               y.data_ptr(), prod.data_ptr(), ws, wsb, stream_ptr(x.device))
    check(st, where)
    _after(x)
    return y


def run_spmv_v2(vals, indptr, cols, x, s, segm_offsets=None):
    """y = A x for CSR (vals, indptr, cols) (reference: src/torch/torch_spmv.h:112-209).

    vals and x both fp16 or both fp32; y is fp32.  Products are formed in fp32
    (the reference rounds fp16 products to fp16 first) and summed per row in
    FP32 by the element-split SIMT kernel (tcu_spmv_rows); with ROWS_FP32 off
    they go to the tensor-core segmented sum instead (tcu_spmv_csr:
    split-precision bf16 hi + lo, FP64 carries for rows spanning tiles).
    ``segm_offsets`` is accepted for signature compatibility and not read."""
    return _spmv(vals, indptr, cols, x, s, "run_spmv_v2")


def run_spmv(vals, indptr, cols, x, s):
    """Same product as run_spmv_v2 (reference v1: src/torch/torch_spmv.h:63-94)."""
    return _spmv(vals, indptr, cols, x, s, "run_spmv")


def run_spmv_v2_multi_cube(vals, indptr, cols, x, upper, lower_strict):
    """SpMV with S taken from ``upper`` (reference: src/torch/torch_spmv.h:235-302)."""
    S = _check_tri(upper, lower_strict)
    return _spmv(vals, indptr, cols, x, S, "run_spmv_v2_multi_cube")


def run_spmv_multi_cube(vals, indptr, cols, x, upper, lower_strict):
    """SpMV with S taken from ``upper`` (reference: src/torch/torch_spmv.h:32-46)."""
    S = _check_tri(upper, lower_strict)
    return _spmv(vals, indptr, cols, x, S, "run_spmv_multi_cube")


def run_scan_cpu(x):
    """The reference's CPU scan (src/torch/torch_scan_cpu.h:24-107) on a host
    tensor: float16/float32 -> float32, int8 -> int32.

    Runs the library's host scan (tcu_scan_cpu) with the reference's blocked
    three-phase order: torch.get_num_threads() contiguous blocks (the
    reference uses omp_get_max_threads(), the same count in a torch process),
    each scanned sequentially in the output type, then the serial scan of the
    block totals added per block, so fp32 results round exactly as the
    reference's do for the same thread count.  This is a CPU operator of the
    reference's interface, not a fallback for any CUDA operator above."""
    if not isinstance(x, torch.Tensor):
        raise TypeError("x must be a torch.Tensor")
    if x.device.type != "cpu":
        raise ValueError("run_scan_cpu expects a CPU tensor")
    if x.dtype not in (torch.int8, torch.float16, torch.float32):
        raise TypeError(f"unsupported dtype {x.dtype}: run_scan_cpu takes int8, float16 or float32")
    x = x.contiguous().reshape(-1)
    out = torch.empty(x.numel(), dtype=torch.int32 if x.dtype == torch.int8 else torch.float32)
    if x.numel() == 0:
        return out
    st = _lib.lib.tcu_scan_cpu(x.data_ptr(), _lib.DTYPE_CODE[x.dtype], x.numel(), out.data_ptr(),
                               torch.get_num_threads())
    check(st, "run_scan_cpu")
    return out


__all__ = [n for n in dir() if n.startswith("run_")] + ["TcuError", "workspace_error", "raise_device_error"]
