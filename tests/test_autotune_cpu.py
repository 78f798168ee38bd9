"""Autotuner host logic without a GPU: candidates per op and dtype, the
fastest (S, CTA count) kept, the JSON table written and read back, nearest-
size lookups, defaults without a table, and the CTA knob reaching the C ABI."""
import json

import pytest
import torch


@pytest.fixture
def at(tmp_path, monkeypatch):
    from tcuscan_b200 import autotune

    monkeypatch.setenv("TCU_AUTOTUNE", "1")
    autotune.reload(str(tmp_path / "tune.json"))
    yield autotune
    autotune.apply_ctas(0)
    autotune.reload(autotune.CACHE)


def _fake(costs):
    """workload/timer pair: the timed cost is costs(op, dtype, n, S, ctas)."""
    from tcuscan_ops import _lib

    def workload(op, dtype, n, device):
        return lambda S: (op, dtype, n, S)

    def timer(fn, steps, warmup):
        op, dtype, n, S = fn()
        return costs(op, dtype, n, S, _lib.lib.tcu_get_max_ctas())

    return workload, timer


def test_tune_picks_fastest_and_writes_table(at, tmp_path):
    # S = 64 fastest for scans at 2^20, S = 128 at 2^28; half the SMs best for compress
    def costs(op, dtype, n, S, ctas):
        if op == "scan":
            return abs(S - (64 if n == 1 << 20 else 128)) + 1.0
        if op == "compress":
            return 1.0 if ctas == 74 else 2.0
        return 1.0 + S / 100

    wl, tm = _fake(costs)
    table = at.tune(device="cpu", ops=("scan", "seg", "compress"), dtypes=(torch.int8, torch.float16),
                    log2_sizes=(20, 28), workload=wl, timer=tm, path=str(tmp_path / "tune.json"))
    e = table["entries"]
    assert e["scan/int8/20"]["S"] == 64 and e["scan/int8/28"]["S"] == 128
    assert e["scan/float16/20"]["S"] == 64
    assert e["seg/int8/28"]["S"] == 32
    assert e["compress/float16/20"]["ctas"] == 74
    on_disk = json.load(open(tmp_path / "tune.json"))
    assert on_disk["entries"] == e
    # lookups, including the nearest tuned size
    assert at.best("scan", torch.int8, 1 << 20) == (64, 0)
    assert at.best("scan", torch.int8, 1 << 27) == (128, 0)
    assert at.best("scan", torch.int8, 1 << 18) == (64, 0)
    assert at.best("compress", torch.float16, 1 << 21) == (64, 74)
    assert at.best("scan", torch.float32, 1 << 20) == (64, 0)  # not tuned: default


def test_defaults_without_table(at):
    assert at.best("scan", torch.int8, 1 << 28) == (128, 0)
    assert at.best("scan", torch.float16, 1 << 28) == (64, 0)
    assert at.best("seg", torch.float32, 1 << 20) == (64, 0)


def test_cta_knob_reaches_library(at):
    from tcuscan_ops import _lib

    at.apply_ctas(100)
    assert _lib.lib.tcu_get_max_ctas() == 100
    at.apply_ctas(0)
    assert _lib.lib.tcu_get_max_ctas() == 0


def test_pick_S_uses_table(at, tmp_path):
    import tcuscan_ops
    from tcuscan_ops import _lib

    tab = {"device": "x", "entries": {"scan/int8/24": {"S": 32, "ctas": 120}, "seg/float16/24": {"S": 32, "ctas": 0}}}
    p = tmp_path / "t2.json"
    p.write_text(json.dumps(tab))
    at.reload(str(p))
    assert tcuscan_ops._pick_S(None, torch.int8, 1 << 24) == 32
    assert _lib.lib.tcu_get_max_ctas() == 120
    assert tcuscan_ops._pick_S(64, torch.int8, 1 << 24) == 64  # explicit S: default CTAs
    assert _lib.lib.tcu_get_max_ctas() == 0
    assert tcuscan_ops._pick_S(0, torch.float16, 1 << 24, op="seg") == 32
    with pytest.raises(ValueError):
        tcuscan_ops._pick_S(48, torch.int8)


def test_lookup_cache_cleared_on_reload(at, tmp_path):
    p1, p2 = tmp_path / "a.json", tmp_path / "b.json"
    p1.write_text(json.dumps({"entries": {"scan/int8/24": {"S": 32, "ctas": 0}}}))
    p2.write_text(json.dumps({"entries": {"scan/int8/24": {"S": 64, "ctas": 0}}}))
    at.reload(str(p1))
    assert at.best("scan", torch.int8, 1 << 24) == (32, 0)
    assert at.best("scan", torch.int8, (1 << 24) + 5) == (32, 0)  # same size class, cached
    at.reload(str(p2))
    assert at.best("scan", torch.int8, 1 << 24) == (64, 0)


def test_segment_sum_dispatch_rule(monkeypatch):
    import tcuscan_ops

    monkeypatch.setattr(tcuscan_ops, "ROWS_MAX_MEAN", 32)
    monkeypatch.setattr(tcuscan_ops, "ROWS_FP32", True)
    assert tcuscan_ops._rows_for(torch.float16, 32 * 100, 100)  # mean 32: element-split
    assert not tcuscan_ops._rows_for(torch.float16, 33 * 100, 100)  # longer: tensor cores
    assert not tcuscan_ops._rows_for(torch.int8, 1 << 20, 16)
    assert tcuscan_ops._rows_for(torch.float32, 1 << 20, 16)  # fp32: always element-split
    assert not tcuscan_ops._rows_for(torch.float16, 10, 0)  # no segments
    monkeypatch.setattr(tcuscan_ops, "ROWS_FP32", False)
    assert not tcuscan_ops._rows_for(torch.float32, 1 << 20, 16)
    monkeypatch.setattr(tcuscan_ops, "ROWS_MAX_MEAN", 0)  # 0: every length element-split (the default)
    assert tcuscan_ops._rows_for(torch.float16, 1 << 20, 16)
    assert tcuscan_ops._rows_for(torch.int8, 1 << 20, 1)
    assert not tcuscan_ops._rows_for(torch.float16, 10, 0)
    monkeypatch.setattr(tcuscan_ops, "ROWS_MAX_MEAN", -1)  # negative: the tensor-core path for every length
    assert not tcuscan_ops._rows_for(torch.float16, 4 * 100, 100)
