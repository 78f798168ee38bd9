"""Host logic of the serving loop, without a GPU: the packed-item layout
matches the C header, arrivals enter per-class queues in order, batches are
cut by request count and by the memory budget (oldest first), and the arena
allocator hands out disjoint blocks and coalesces freed ones."""
import collections
import os
import re
import time

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _server(budget, max_batch):
    from tcuscan_b200 import serve

    s = object.__new__(serve.Server)
    s._cap, s._n, s._next_arrival = 0, 0, 0
    s._alloc(8)
    s.queues = collections.defaultdict(collections.deque)
    s.budget, s.max_batch, s.max_batch_bytes = budget, max_batch, budget
    s.t0 = time.perf_counter()
    s._keepalive = {}
    return s


def test_pack_item_matches_header():
    from tcuscan_b200 import serve

    hdr = open(os.path.join(REPO, "include", "tcuscan.h")).read()
    body = re.search(r"typedef struct tcu_pack_item \{(.*?)\} tcu_pack_item_t;", hdr, re.S).group(1)
    fields = re.findall(r"(\w+);", body)
    assert fields == list(serve.PACK_ITEM.names)
    assert serve.PACK_ITEM.itemsize == 40


def test_arrivals_split_by_class_in_order():
    from tcuscan_b200 import serve

    s = _server(1 << 30, 100)
    k = 40
    rng = np.random.default_rng(0)
    op = rng.integers(0, 3, size=k).astype(np.int8)
    dt = rng.integers(0, 3, size=k).astype(np.int8)
    iw = np.where(op == serve.SEG_SUM, 4, 0).astype(np.int8)
    s.submit_many(op, dt, np.full(k, 5000), np.zeros(k, np.uint64), np.zeros(k, np.uint64),
                  np.where(op == serve.SEG_SUM, 70, 0), iw, np.zeros(k))
    s._arrivals()
    seen = []
    for cls, q in s.queues.items():
        ids = np.concatenate(list(q))
        assert np.all(np.diff(ids) > 0)
        assert len({(int(op[i]), int(dt[i])) for i in ids}) == 1
        seen.extend(ids.tolist())
    assert sorted(seen) == list(range(k))
    # future arrivals stay out of the queues
    s.submit_many(op[:3], dt[:3], np.full(3, 10), np.zeros(3, np.uint64), np.zeros(3, np.uint64),
                  np.zeros(3, np.int64), np.zeros(3, np.int8), np.full(3, 1e9))
    s._arrivals()
    assert s._next_arrival == k


def test_take_respects_budget_and_count():
    from tcuscan_b200 import serve

    s = _server(1 << 30, 4)
    k = 10
    s.submit_many(np.zeros(k, np.int8), np.ones(k, np.int8), np.full(k, 1 << 16), np.zeros(k, np.uint64),
                  np.zeros(k, np.uint64), np.zeros(k, np.int64), np.zeros(k, np.int8), np.zeros(k))
    s._arrivals()
    cls = next(iter(s.queues))
    per = int(s._bytes(np.array([0]))[0])
    slack = serve.BATCH_SLACK
    ids, used = s._take(cls, 1 << 30)
    assert list(ids) == [0, 1, 2, 3] and used == 4 * per + slack  # count cap
    ids, used = s._take(cls, int(2.5 * per) + slack)
    assert list(ids) == [4, 5] and used == 2 * per + slack  # memory cap
    ids, used = s._take(cls, per - 1 + slack)
    assert ids is None  # the head does not fit yet: nothing is skipped
    ids, _ = s._take(cls, 1 << 30)
    assert list(ids) == [6, 7, 8, 9]
    assert cls not in s.queues


def test_request_over_budget_is_refused():
    from tcuscan_b200 import serve

    s = _server(1 << 20, 4)
    s.submit_many(np.zeros(1, np.int8), np.full(1, 2, np.int8), np.array([1 << 20]), np.zeros(1, np.uint64),
                  np.zeros(1, np.uint64), np.zeros(1, np.int64), np.zeros(1, np.int8), np.zeros(1))
    s._arrivals()
    with pytest.raises(MemoryError):
        s._take(next(iter(s.queues)), 1 << 20)


def test_bytes_cover_outputs():
    from tcuscan_b200 import serve

    s = _server(1 << 30, 4)
    n = 100_000
    s.submit_many(np.array([0, 1, 2], np.int8), np.array([0, 1, 2], np.int8), np.full(3, n),
                  np.zeros(3, np.uint64), np.zeros(3, np.uint64), np.array([0, 1500, 0]), np.array([0, 4, 0], np.int8),
                  np.zeros(3))
    b = s._bytes(np.arange(3))
    npad = -(-n // 256) * 256
    assert b[0] >= npad * (1 + 4)          # int8 in, int32 out
    assert b[1] >= npad * 2 + 1501 * 12    # fp16 in, bounds + sums
    assert b[2] >= npad * (4 + 1 + 4) + 8  # fp32 in, mask, full-capacity out, output offset


def test_arena_first_fit_and_coalescing():
    from tcuscan_b200 import serve

    a = object.__new__(serve.Arena)
    a.size, a.base, a.free = 1 << 20, 0, [(0, 1 << 20)]
    blocks = [a.alloc(n) for n in (1000, 70_000, 256, 300_000)]
    offs = [o for o, _ in blocks]
    assert all(o % serve.BLOCK_ALIGN == 0 for o in offs)
    spans = sorted((o, o + sz) for o, sz in blocks)
    assert all(spans[i][1] <= spans[i + 1][0] for i in range(len(spans) - 1))
    a.release(*blocks[1])
    o, sz = a.alloc(60_000)  # first fit reuses the hole
    assert o == blocks[1][0]
    a.release(o, sz)
    for b in (blocks[0], blocks[2], blocks[3]):
        a.release(*b)
    assert a.free == [(0, 1 << 20)] and a.largest() == 1 << 20
    assert a.alloc(2 << 20) == (None, 0)
