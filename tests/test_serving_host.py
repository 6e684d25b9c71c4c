"""Host logic of the scan server: the pool range allocator and request footprints."""

import numpy as np


def test_range_allocator_first_fit_and_coalesce(rb):
    a = rb.RangeAllocator(100, align=4)
    assert a.capacity == 100
    x = a.alloc(10)  # rounds to 12
    y = a.alloc(40)
    z = a.alloc(40)
    assert (x, y, z) == (0, 12, 52)
    assert a.alloc(16) is None  # 8 left
    a.release(y, 40)
    assert a.largest_free == 40
    assert a.alloc(20) == 12  # first fit into the hole
    a.release(x, 10)
    a.release(12, 20)
    a.release(z, 40)
    assert a.free == [[0, 100]] and a.used == 0


def test_range_allocator_random_never_overlaps(rb):
    rng = np.random.default_rng(3)
    a = rb.RangeAllocator(4096, align=4)
    live = {}
    for _ in range(2000):
        if live and rng.random() < 0.45:
            off = list(live)[rng.integers(len(live))]
            a.release(off, live.pop(off))
        else:
            n = int(rng.integers(1, 300))
            off = a.alloc(n)
            if off is not None:
                assert off % 4 == 0
                for o, m in live.items():
                    assert off + n <= o or o + m <= off
                live[off] = n
    for off, n in list(live.items()):
        a.release(off, n)
    assert a.free == [[0, 4096]] and a.used == 0


def test_request_footprint(rb):
    fp = rb.request_footprint(64, 8, 4, 10)
    nw = rb.packing.words_for(64)
    assert fp == {"words": 32 * nw + 4 * 2 * nw, "rows": 320, "chains": 32}
