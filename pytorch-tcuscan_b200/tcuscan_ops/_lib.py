"""ctypes binding of libtcuscan.so (the C ABI in include/tcuscan.h).

The shared library is the product: this module only declares its signatures,
owns the per-(device, stream) look-back workspaces, and turns non-OK status
codes into Python exceptions.  There is no CPU fallback: importing
tcuscan_ops without the built library raises ImportError.
"""
import ctypes
import os
import threading

import torch

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("TCUSCAN_LIB", os.path.join(PKG, "lib", "libtcuscan.so"))

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"libtcuscan.so not found at {LIB_PATH}; build it with `python pytorch-tcuscan_b200/build.py`"
    )
lib = ctypes.CDLL(LIB_PATH)

# status codes (include/tcuscan.h)
TCU_OK, TCU_ERR_ARG, TCU_ERR_DTYPE, TCU_ERR_LAUNCH, TCU_ERR_TIMEOUT = 0, 1, 2, 3, 4
TCU_ERR_OOM, TCU_ERR_ALIGN, TCU_ERR_DEVICE, TCU_ERR_WORKSPACE = 5, 6, 7, 8

# dtype codes
TCU_INT8, TCU_INT16, TCU_INT32, TCU_INT64 = 1, 2, 3, 4
TCU_FLOAT16, TCU_BFLOAT16, TCU_FLOAT32, TCU_FLOAT64, TCU_UINT32 = 5, 6, 7, 8, 9
TCU_UINT8 = 10

DTYPE_CODE = {
    torch.int8: TCU_INT8,
    torch.int16: TCU_INT16,
    torch.int32: TCU_INT32,
    torch.int64: TCU_INT64,
    torch.float16: TCU_FLOAT16,
    torch.bfloat16: TCU_BFLOAT16,
    torch.float32: TCU_FLOAT32,
    torch.float64: TCU_FLOAT64,
    torch.uint8: TCU_UINT8,
}
if hasattr(torch, "uint32"):
    DTYPE_CODE[torch.uint32] = TCU_UINT32

_P, _I, _I64, _U64, _SZ, _D = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_double
_ST = ctypes.c_int


def _sig(name, restype, *argtypes):
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = list(argtypes)
    return f


_sig("tcu_version", _I)
_sig("tcu_status_string", ctypes.c_char_p, _I)
_sig("tcu_last_error_message", ctypes.c_char_p)
_sig("tcu_set_timeout_ns", None, _U64)
_sig("tcu_get_timeout_ns", _U64)
_sig("tcu_workspace_bytes", _SZ, _I64, _I)
_sig("tcu_workspace_init", _ST, _P, _SZ, _P)
_sig("tcu_workspace_error", _ST, _P, ctypes.POINTER(ctypes.c_uint32), _I, _P)
_sig("tcu_set_phase_profile", None, _I)
_sig("tcu_set_max_ctas", None, _I)
_sig("tcu_selftest_wait_timeout", _ST, _I, _U64, _P, _SZ, _P)
_sig("tcu_get_max_ctas", _I)
_sig("tcu_set_small_tile_limit", None, _I)
_sig("tcu_get_small_tile_limit", _I)
_sig("tcu_set_simt_scan_limit", None, _I64)
_sig("tcu_get_simt_scan_limit", _I64)
_sig("tcu_workspace_phase_ns", _ST, _P, ctypes.POINTER(ctypes.c_uint64), _I, _P)
_sig("tcu_scan", _ST, _P, _I, _I64, _I, _D, _P, _P, _SZ, _P)
_sig("tcu_scan_cpu", _ST, _P, _I, _I64, _P, _I)
_sig("tcu_scan_chained", _ST, _P, _I, _I64, _I, _D, _P, _P, _P, _SZ, _P)
_sig("tcu_scan_chained_typed", _ST, _P, _I, _I64, _I, _D, _P, _I, _P, _P, _SZ, _P)
_sig("tcu_total", _ST, _P, _I, _I64, _P, _P, _SZ, _P)
_sig("tcu_row_scan", _ST, _P, _I, _I64, _I, _P, _P, _SZ, _P)
_sig("tcu_block_scan", _ST, _P, _I, _I64, _I, _P, _P, _SZ, _P)
_sig("tcu_block_scan_tensor", _ST, _P, _I, _I64, _I, _P, _P, _P, _P, _SZ, _P)
_sig("tcu_seg_scan", _ST, _P, _I, _I64, _I, _P, _I, _P, _P, _SZ, _P)
_sig("tcu_seg_bounds", _ST, _P, _I, _I64, _I, _P, _I, _I64, _I, _P, _P, _SZ, _P)
_sig("tcu_scan_batch", _ST, _P, _I, _I64, _I64, _I, _P, _P, _SZ, _P)
_sig("tcu_spmv_csr", _ST, _P, _I, _P, _I, _I64, _P, _I64, _P, _I64, _I, _P, _P, _P, _SZ, _P)
_sig("tcu_spmv_products", _ST, _P, _I, _P, _I64, _P, _I64, _P, _P, _P)
_sig("tcu_compress", _ST, _P, _I, _P, _I64, _P, _I, _I, _P, _P, _I64, _P, _P, _SZ, _P)
_sig("tcu_mask_count", _ST, _P, _I64, _P, _P)
_sig("tcu_compress_count", _ST, _P, _I64, _I, _I, _I, _P, _P, _SZ, _P)
_sig("tcu_compress_counted", _ST, _P, _I, _P, _I64, _P, _I, _I, _P, _P, _I64, _P, _SZ, _P)
_sig("tcu_compress_segments", _ST, _P, _I, _P, _I64, _P, _I64, _P, _I64, _P, _P, _SZ, _P)
_sig("tcu_rows_workspace_bytes", _SZ, _I64)
_sig("tcu_seg_sum_rows", _ST, _P, _I, _I64, _P, _I, _I64, _P, _P, _SZ, _P)
_sig("tcu_spmv_rows", _ST, _P, _I, _P, _I, _I64, _P, _I64, _P, _I64, _P, _P, _SZ, _P)
_sig("tcu_split", _ST, _P, _I, _P, _I64, _P, _I, _I, _P, _P, _P, _P, _SZ, _P)
_sig("tcu_radix_sort_tmp_bytes", _SZ, _I, _I64)
_sig("tcu_radix_sort", _ST, _P, _I, _I64, _P, _P, _P, _SZ, _P)
_sig("tcu_topk_tmp_bytes", _SZ, _I64)
_sig("tcu_topk", _ST, _P, _I, _I64, _I64, _P, _P, _P, _SZ, _P)
_sig("tcu_topk_pivot_blocks", _I, _I64, _I)
_sig("tcu_topk_pivot", _ST, _P, _I, _I64, _I, _I, _I, _P, _P)
_sig("tcu_pack", _ST, _P, _I64, _I, _I, _P, _I64, _P)
_sig("tcu_csr_gather", _ST, _P, _I, _P, _I64, _P, _I64, _P, _P, _P)
_sig("tcu_gather_spmv", _ST, _P, _I, _I64, _P, _I, _I64, _P, _P, _P)
_sig("tcu_reduce_tiles", _ST, _P, _I, _I64, _I64, _I, _P, _P, _SZ, _P)
_sig("tcu_complete_rows", _ST, _P, _I, _I64, _P, _I, _I64, _P, _P, _SZ, _P)
_sig("tcu_complete_blocks", _ST, _P, _I, _I64, _P, _I, _P, _P)
_sig("tcu_gen_lower", _ST, _I64, _I, _P, _P)


class TcuError(RuntimeError):
    """A libtcuscan call or a device-side bounded wait failed."""

    def __init__(self, status, where, detail=""):
        self.status = int(status)
        msg = lib.tcu_status_string(int(status)).decode()
        last = lib.tcu_last_error_message().decode()
        super().__init__(f"{where}: {msg}" + (f" ({detail})" if detail else "") + (f" [{last}]" if last else ""))


def check(status, where):
    if status != TCU_OK:
        if status in (TCU_ERR_ARG, TCU_ERR_DTYPE, TCU_ERR_ALIGN):
            raise ValueError(f"{where}: {lib.tcu_status_string(int(status)).decode()} "
                             f"[{lib.tcu_last_error_message().decode()}]")
        raise TcuError(status, where)


_raw_stream_fn = getattr(torch._C, "_cuda_getCurrentRawStream", None)


def _stream_key(dev):
    """(device index, cudaStream_t as an int) of the current stream of
    torch.device `dev` (the raw accessor skips building a torch.cuda.Stream
    object: ~2 us per call of the small scans)."""
    idx = dev.index if dev.index is not None else torch.cuda.current_device()
    if _raw_stream_fn is not None:
        return idx, _raw_stream_fn(idx)
    return idx, torch.cuda.current_stream(torch.device("cuda", idx)).cuda_stream


def stream_ptr(device):
    dev = device if isinstance(device, torch.device) else torch.device(device)
    return ctypes.c_void_p(_stream_key(dev)[1])


class _Workspace:
    __slots__ = ("buf", "bytes", "ptr")

    def __init__(self):
        self.buf = None
        self.bytes = 0
        self.ptr = None


_ws_lock = threading.Lock()
_workspaces = {}

SYNC_CHECK = os.environ.get("TCU_SYNC_CHECK", "0") == "1"


def workspace(device, need_bytes):
    """Return (ptr, bytes) of the look-back workspace of (device, current stream).

    One workspace per stream keeps launches that may overlap on the GPU from
    sharing look-back state; launches on one stream are ordered, and each one
    leaves the workspace reset for the next (epoch-tagged flags)."""
    ws, wsb, _ = launch_context(device, need_bytes)
    return ws, wsb


def launch_context(device, need_bytes):
    """(workspace ptr, workspace bytes, stream ptr) of (device, current
    stream): one current-stream lookup for both (the per-call host cost of
    the small scans is a few microseconds)."""
    dev = device if isinstance(device, torch.device) else torch.device(device)
    key = _stream_key(dev)
    sid = key[1]
    with _ws_lock:
        ws = _workspaces.get(key)
        if ws is None:
            ws = _workspaces[key] = _Workspace()
        if ws.bytes < need_bytes:
            nbytes = max(int(need_bytes), 1 << 20, 2 * ws.bytes)
            ws.buf = torch.empty(nbytes, dtype=torch.uint8, device=dev)
            ws.bytes = nbytes
            ws.ptr = None
            check(lib.tcu_workspace_init(ctypes.c_void_p(ws.buf.data_ptr()), _SZ(nbytes), ctypes.c_void_p(sid)),
                  "tcu_workspace_init")
        if ws.ptr is None:
            ws.ptr = (ctypes.c_void_p(ws.buf.data_ptr()), _SZ(ws.bytes), ctypes.c_void_p(sid))
        return ws.ptr


def workspace_error(device=None, clear=True):
    """Synchronise and return (code, site, chunk) of the current stream's workspace."""
    dev = torch.device(device if device is not None else torch.cuda.current_device())
    if dev.type == "cuda" and dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    ws = _workspaces.get((dev.index, stream.cuda_stream))
    if ws is None or ws.buf is None:
        return (0, 0, 0)
    info = (ctypes.c_uint32 * 3)()
    lib.tcu_workspace_error(ctypes.c_void_p(ws.buf.data_ptr()), info, int(clear), ctypes.c_void_p(stream.cuda_stream))
    return (int(info[0]), int(info[1]), int(info[2]))


def raise_device_error(device=None):
    code, site, chunk = workspace_error(device, clear=True)
    if code != TCU_OK:
        raise TcuError(code, "device", f"site {site}, chunk {chunk}")


def set_timeout_ns(ns):
    lib.tcu_set_timeout_ns(_U64(int(ns)))


def get_timeout_ns():
    return int(lib.tcu_get_timeout_ns())


PHASE_NAMES = ("epilogue_wait_mma", "row_totals", "lookback", "drain", "producer_wait_stage", "summer",
               "summer_wait_data", "tiles")


def set_phase_profile(enable):
    lib.tcu_set_phase_profile(int(bool(enable)))


def phase_times(device=None, clear=True):
    """Per-phase device time counters of the current stream's workspace (diagnostics)."""
    dev = torch.device(device if device is not None else torch.cuda.current_device())
    if dev.type == "cuda" and dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    ws = _workspaces.get((dev.index, stream.cuda_stream))
    if ws is None or ws.buf is None:
        return {}
    out = (ctypes.c_uint64 * 8)()
    check(lib.tcu_workspace_phase_ns(ctypes.c_void_p(ws.buf.data_ptr()), out, int(clear),
                                     ctypes.c_void_p(stream.cuda_stream)), "tcu_workspace_phase_ns")
    return {n: int(v) for n, v in zip(PHASE_NAMES, out)}
