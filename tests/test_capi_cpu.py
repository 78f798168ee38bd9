"""C-ABI checks that need no GPU: the library loads, exports every symbol that
include/*.h declares, and rejects bad arguments before touching the device."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest
import torch

from conftest import LIB_PATH, REPO

HEADERS = sorted(glob.glob(os.path.join(REPO, "include", "*.h")))


def _declared():
    names = []
    for h in HEADERS:
        txt = open(h).read()
        names += re.findall(r"TCU_API\s+[\w\s\*]+?\b(tcu_\w+)\s*\(", txt)
    return sorted(set(names))


def test_headers_exist():
    assert HEADERS, "include/*.h missing"
    assert len(_declared()) >= 8


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


_C_TYPES = {"tcu_status_t": ctypes.c_int, "tcu_dtype_t": ctypes.c_int, "int": ctypes.c_int,
            "int64_t": ctypes.c_int64, "uint64_t": ctypes.c_uint64, "uint32_t": ctypes.c_uint32,
            "size_t": ctypes.c_size_t, "double": ctypes.c_double, "void": None}


def _header_signatures():
    """(return type, name, [parameter types]) of every TCU_API declaration;
    pointer and array parameters read as 'ptr'."""
    def ctype(t):
        t = " ".join(t.replace("const", "").split())
        if "char" in t and "*" in t:
            return ctypes.c_char_p
        return "ptr" if ("*" in t or "[" in t) else _C_TYPES[t]

    sigs = []
    for h in HEADERS:
        txt = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for ret, name, params in re.findall(r"TCU_API\s+([\w\s\*]+?)\s*\b(tcu_\w+)\s*\(([^)]*)\)\s*;", txt):
            args = []
            for p in params.split(","):
                p = p.strip()
                if p in ("", "void"):
                    continue
                m = re.match(r"(.*?)\w+\s*(\[\d*\])?$", p)
                args.append(ctype(m.group(1) + (m.group(2) or "")))
            sigs.append((ctype(ret), name, args))
    return sigs


def test_bindings_match_header_signatures():
    """Every signature tcuscan_ops._lib declares to ctypes agrees with the
    header: return type, arity, and each argument's width (a 64-bit size
    passed as a C int would be truncated silently)."""
    import tcuscan_ops._lib as L

    sigs = _header_signatures()
    assert len(sigs) == len(_declared())
    bound, bad = 0, []
    for ret, name, args in sigs:
        f = getattr(L.lib, name)
        if f.argtypes is None:
            continue  # not bound by the package (a test binds it itself)
        bound += 1
        if f.restype is not ret:
            bad.append((name, "return", f.restype, ret))
        if len(f.argtypes) != len(args):
            bad.append((name, "arity", len(f.argtypes), len(args)))
            continue
        for i, (got, want) in enumerate(zip(f.argtypes, args)):
            if want == "ptr":
                ok = got is ctypes.c_void_p or (isinstance(got, type) and issubclass(got, ctypes._Pointer))
            else:
                ok = got is want
            if not ok:
                bad.append((name, i, got, want))
    assert bound >= 40 and not bad, bad


def test_status_strings_and_version():
    import tcuscan_ops._lib as L

    assert L.lib.tcu_version() >= 100
    for code in range(0, 9):
        assert L.lib.tcu_status_string(code)
    assert L.lib.tcu_status_string(999) == b"unknown status"


def test_workspace_bytes_monotone():
    import tcuscan_ops._lib as L

    prev = 0
    for n in (1, 1000, 1 << 20, 1 << 28):
        b = L.lib.tcu_workspace_bytes(n, 64)
        assert b >= prev and b >= 128
        prev = b
    # one 16-byte look-back descriptor per 32768-element tile, whatever S is
    assert L.lib.tcu_workspace_bytes(1 << 28, 16) == L.lib.tcu_workspace_bytes(1 << 28, 128)
    assert L.lib.tcu_workspace_bytes(1 << 28, 64) >= 16 * ((1 << 28) // 32768)


def test_argument_errors_before_device():
    import tcuscan_ops._lib as L

    # n == 0 is a no-op; negative n, unaligned pointers, bad S are rejected on the host
    assert L.lib.tcu_scan(None, L.TCU_INT8, 0, 64, 0.0, None, None, 0, None) == L.TCU_OK
    assert L.lib.tcu_scan(None, L.TCU_INT8, -1, 64, 0.0, None, None, 0, None) == L.TCU_ERR_ARG
    assert L.lib.tcu_scan(ctypes.c_void_p(0x1001), L.TCU_INT8, 10, 64, 0.0, ctypes.c_void_p(0x2000), None, 0,
                          None) == L.TCU_ERR_ALIGN
    assert L.lib.tcu_block_scan(ctypes.c_void_p(0x1000), L.TCU_FLOAT16, 100, 16, ctypes.c_void_p(0x2000), None, 0,
                                None) == L.TCU_ERR_ARG


def test_python_layer_rejects_cpu_tensors():
    import tcuscan_ops

    with pytest.raises(ValueError):
        tcuscan_ops.run_scan_multi_core(torch.zeros(10, dtype=torch.int8), 64)
    with pytest.raises(ValueError):
        tcuscan_ops.run_scan_multi_core(torch.zeros(10, dtype=torch.int8, device="meta"), 64)


@pytest.mark.parametrize("dtype", [torch.bfloat16, torch.int16, torch.float64])
def test_scan_output_dtype_rejects_unsupported_inputs(dtype):
    """Scans and sums take int8, float16 or float32; anything else is a
    TypeError before any launch."""
    import tcuscan_ops

    assert tcuscan_ops._scan_out_dtype(torch.int8) == torch.int32
    assert tcuscan_ops._scan_out_dtype(torch.float16) == torch.float32
    with pytest.raises(TypeError):
        tcuscan_ops._scan_out_dtype(dtype)


def test_run_scan_cpu_api():
    import tcuscan_ops

    x = torch.randint(0, 10, (1000,), dtype=torch.int8)
    assert torch.equal(tcuscan_ops.run_scan_cpu(x), torch.cumsum(x, 0, dtype=torch.int32))
    xf = torch.randn(1000).half()
    assert tcuscan_ops.run_scan_cpu(xf).dtype == torch.float32
    assert tcuscan_ops.run_scan_cpu(torch.empty(0, dtype=torch.float32)).numel() == 0
    with pytest.raises(TypeError):
        tcuscan_ops.run_scan_cpu(torch.zeros(4, dtype=torch.float64))


def test_run_scan_cpu_matches_reference_fixtures(golden):
    """run_scan_cpu against the reference's own run_scan_cpu outputs (golden
    fixtures, made with the thread count they record): bit-exact for int8,
    fp16 and fp32 when the block count is the same."""
    import tcuscan_ops

    threads = int(golden["scan_threads"])
    keys = sorted({k[:-4] for k in golden.files if k.startswith("scan_") and k.endswith("_ref")
                   and k.split("_")[1] in ("i8", "f16", "f32")})
    assert keys
    old = torch.get_num_threads()
    try:
        torch.set_num_threads(threads)
        for b in keys:
            x, ref = golden[b + "_x"], golden[b + "_ref"]
            got = tcuscan_ops.run_scan_cpu(torch.from_numpy(x)).numpy()
            assert got.dtype == ref.dtype, b
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), b
    finally:
        torch.set_num_threads(old)


@pytest.mark.parametrize("threads", [1, 3, 16])
@pytest.mark.parametrize("dtype", [torch.int8, torch.float16, torch.float32])
def test_run_scan_cpu_blocked_order(threads, dtype):
    """Same rounding as the oracle's restatement of the reference's blocked
    scan for any block count, across the worker threshold (2^16 elements)."""
    import oracle
    import tcuscan_ops

    g = torch.Generator().manual_seed(threads)
    for n in (1, 5, 1000, (1 << 16) + 3):
        if dtype == torch.int8:
            x = torch.randint(-128, 128, (n,), dtype=torch.int8, generator=g)
            want = oracle.blocked_scan_like_reference(x.numpy().astype(np.int32), threads)
        else:
            x = (torch.randn(n, generator=g) * 100).to(dtype)
            want = oracle.blocked_scan_like_reference(x.numpy().astype(np.float32), threads)
        old = torch.get_num_threads()
        try:
            torch.set_num_threads(threads)
            got = tcuscan_ops.run_scan_cpu(x).numpy()
        finally:
            torch.set_num_threads(old)
        assert np.array_equal(got.view(np.uint32), np.asarray(want).view(np.uint32)), (n, threads)


def test_tcuscan_package_reexports():
    import tcuscan

    assert hasattr(tcuscan, "run_scan_multi_core") and hasattr(tcuscan, "run_row_scan")
