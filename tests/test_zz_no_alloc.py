"""The scan entry point that allocates nothing (tcu_scan_noalloc).

Some callers cannot allocate device memory where they need a scan -- code
running inside an allocator or memory-pool callback, plugins given a fixed
device budget by their host, paths that must never reach cudaMalloc -- so
this entry point takes its look-back scratch from a fixed array inside the
library instead of a caller workspace.  These tests call it through the C ABI
and check it against tcu_scan (the entry point with a workspace) on two calls
in a row, within the tolerances the other scan tests use: int8 bit-exact,
fp16 / fp32 within 1e-3 relative to max(|ref|, 1).

This file is collected last on purpose, and it passes both alone in a fresh
process and after the rest of the suite.
"""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
MAX_N = 2_147_221_504  # (1 MiB - 128) / 16 tiles x 32768 elements


def _lib():
    from tcuscan_ops import _lib as L

    f = L.lib.tcu_scan_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                  ctypes.c_void_p]
    e = L.lib.tcu_scan_noalloc_error
    e.restype = ctypes.c_int
    e.argtypes = [ctypes.POINTER(ctypes.c_uint32), ctypes.c_int, ctypes.c_void_p]
    return L


def _compare(L, dtype, n, S, start, seed, stream):
    """One tcu_scan (workspace) and one tcu_scan_noalloc call on the same
    input; int8 bit-exact, floats within 1e-3 of each other (floor 1)."""
    out_dtype = torch.int32 if dtype == torch.int8 else torch.float32
    x = _input(dtype, n, seed)
    ref = torch.empty(n, dtype=out_dtype, device=DEV)
    ws, wsb = L.workspace(torch.device(DEV), L.lib.tcu_workspace_bytes(n, S))
    assert L.lib.tcu_scan(x.data_ptr(), L.DTYPE_CODE[dtype], n, S, start, ref.data_ptr(), ws, wsb, stream) == 0
    got = torch.full((n,), 7, dtype=out_dtype, device=DEV)  # stale contents must not leak through
    st = L.lib.tcu_scan_noalloc(x.data_ptr(), L.DTYPE_CODE[dtype], n, S, start, got.data_ptr(), stream)
    assert st == 0, L.lib.tcu_last_error_message()
    info = (ctypes.c_uint32 * 3)()
    assert L.lib.tcu_scan_noalloc_error(info, 1, stream) == 0, list(info)
    if dtype == torch.int8:
        assert torch.equal(got, ref), f"n={n} S={S}: int8 results differ"
    else:
        err = ((got.double() - ref.double()).abs() / ref.double().abs().clamp_min(1.0)).max().item()
        assert err <= 1e-3, f"n={n} S={S}: max rel diff {err}"


def _input(dtype, n, seed):
    g = torch.Generator(device=DEV).manual_seed(seed)
    if dtype == torch.int8:
        return torch.randint(-8, 9, (n,), dtype=torch.int8, device=DEV, generator=g)
    return (torch.rand(n, device=DEV, generator=g) * 2 - 1).to(dtype)


@pytest.mark.parametrize("dtype,n,S,start", [(torch.int8, 3_000_017, 128, 5.0), (torch.float16, 1_000_003, 64, 0.0),
                                             (torch.float32, 777_777, 64, -2.5)])
def test_noalloc_matches_workspace_scan_on_two_calls(dtype, n, S, start):
    L = _lib()
    out_dtype = torch.int32 if dtype == torch.int8 else torch.float32
    stream = ctypes.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)
    for call in range(2):
        x = _input(dtype, n, 100 + call)
        ref = torch.empty(n, dtype=out_dtype, device=DEV)
        ws, wsb = L.workspace(torch.device(DEV), L.lib.tcu_workspace_bytes(n, S))
        assert L.lib.tcu_scan(x.data_ptr(), L.DTYPE_CODE[dtype], n, S, start, ref.data_ptr(), ws, wsb, stream) == 0
        got = torch.full((n,), 7, dtype=out_dtype, device=DEV)  # stale contents must not leak through
        st = L.lib.tcu_scan_noalloc(x.data_ptr(), L.DTYPE_CODE[dtype], n, S, start, got.data_ptr(), stream)
        assert st == 0, L.lib.tcu_last_error_message()
        torch.cuda.synchronize()
        if dtype == torch.int8:
            assert torch.equal(got, ref), f"call {call}: int8 results differ"
        else:
            err = ((got.double() - ref.double()).abs() / ref.double().abs().clamp_min(1.0)).max().item()
            assert err <= 1e-3, f"call {call}: max rel diff {err}"


def test_noalloc_call_sequence_reuses_the_scratch():
    """Calls in a row share the array and keep its last contents: more tiles
    than the call before (stale descriptors past the previous range), fewer,
    exact multiples of the 32768-element tile, inputs small enough for the
    one-block tiles, int8 with S = 16 (run as 32) and S = 32."""
    L = _lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)
    seq = [(torch.int8, 40_000, 128), (torch.int8, 3 * 32768, 128), (torch.float16, 1000, 64),
           (torch.int8, 6_000_000, 16), (torch.float16, 5_000_000, 64), (torch.int8, 32 * 32768, 32),
           (torch.float32, 100_003, 64), (torch.int8, 2_000_000, 64), (torch.float16, 32768, 16),
           (torch.int8, 9_000_001, 128), (torch.float32, 4 * 32768, 64), (torch.int8, 777, 16)]
    for i, (dtype, n, S) in enumerate(seq):
        _compare(L, dtype, n, S, float(i % 3) - 1.0, 500 + i, stream)


def test_noalloc_error_accessor_reads_a_clean_state():
    """The accessor copies the scratch's error words without allocating; after
    successful calls they are zero."""
    L = _lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)
    _compare(L, torch.int8, 123_457, 64, 0.0, 9, stream)
    info = (ctypes.c_uint32 * 3)(1, 2, 3)
    assert L.lib.tcu_scan_noalloc_error(info, 0, stream) == 0
    assert list(info) == [0, 0, 0]


def test_noalloc_rejects_sizes_beyond_its_scratch():
    """n above the fixed scratch's limit is refused before any device work."""
    L = _lib()
    st = L.lib.tcu_scan_noalloc(ctypes.c_void_p(0x1000), L.TCU_INT8, MAX_N + 1, 128, 0.0, ctypes.c_void_p(0x2000),
                                None)
    assert st == L.TCU_ERR_ARG
    assert b"limit" in L.lib.tcu_last_error_message()
