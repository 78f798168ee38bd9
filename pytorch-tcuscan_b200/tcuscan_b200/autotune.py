"""Tile-parameter selection for the tensor-core scan family.

``best_S(op, dtype, n)`` returns the S used when a caller passes S=None/0.
Defaults below are the fastest measured choice per (op, dtype); a tuned table
written by ``tune()`` (JSON, keyed by op, dtype and log2(n) bucket) overrides
them when present.
"""
import json
import math
import os

import torch

# Fastest measured tile parameter per (op, dtype) on B200 at n = 2^28 (the
# autotune table refines this per size bucket when present).
_DEFAULTS = {
    ("scan", torch.int8): 128,
    ("scan", torch.float16): 64,
    ("scan", torch.float32): 64,
}
CACHE = os.environ.get("TCU_AUTOTUNE_CACHE", os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotune.json"))
_table = None


def _load():
    global _table
    if _table is None:
        _table = {}
        if os.path.exists(CACHE):
            try:
                with open(CACHE) as fh:
                    _table = json.load(fh)
            except (OSError, ValueError):
                _table = {}
    return _table


def _key(op, dtype, n):
    b = int(math.log2(max(int(n), 1))) if n else 0
    return f"{op}/{str(dtype).replace('torch.', '')}/{b}"


def best_S(op, dtype, n=None):
    if os.environ.get("TCU_AUTOTUNE", "1") != "0" and n is not None:
        v = _load().get(_key(op, dtype, n))
        if v:
            return int(v)
    return _DEFAULTS.get((op, dtype), 64)
