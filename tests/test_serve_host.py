"""Host-side tests of the serving loop: the device-memory arena allocator
(first fit, coalescing, shrink), run on the CPU through mans_debug_arena."""
import ctypes as C

import numpy as np
import mans_b200 as mb


def run(size, ops):
    flat = np.array([v for op in ops for v in op], dtype=np.uint64)
    res = np.zeros(len(ops), dtype=np.uint64)
    used = mb.load().mans_debug_arena(size, flat.ctypes.data_as(C.c_void_p), len(ops),
                                      res.ctypes.data_as(C.c_void_p))
    return int(used), [int(r) for r in res]


NONE = (1 << 64) - 1


def test_arena_first_fit_and_exhaustion():
    used, r = run(4096, [(0, 1000, 0), (0, 1000, 0), (0, 1000, 0), (0, 1000, 0), (0, 1, 0)])
    assert r[:4] == [0, 1024, 2048, 3072]
    assert r[4] == NONE and used == 4096


def test_arena_release_coalesces():
    # free the middle two blocks: one 2048-byte hole must serve a 2048 request
    used, r = run(4096, [(0, 1024, 0), (0, 1024, 0), (0, 1024, 0), (0, 1024, 0),
                         (1, 1024, 1024), (1, 2048, 1024), (0, 2048, 0)])
    assert r[6] == 1024 and used == 4096


def test_arena_shrink_returns_tail():
    used, r = run(8192, [(0, 4096, 0), (2, 0, 300), (0, 3000, 0), (0, 4096, 0)])
    assert r[2] == 512  # 300 rounds up to 512; the freed tail joins the free space after it
    assert r[3] == 512 + 3072  # [3584, 8192) is one free block
    assert used == 512 + 3072 + 4096


def test_arena_full_cycle_returns_to_empty():
    rng = np.random.default_rng(0)
    size = 1 << 20
    # allocate, free in random order, then the whole arena must be one block
    _, offs = run(size, [(0, 4096 * (i + 1), 0) for i in range(10)])
    frees = [(1, offs[i], 4096 * (i + 1)) for i in rng.permutation(10)]
    used2, _ = run(size, [(0, 4096 * (i + 1), 0) for i in range(10)] + frees + [(0, size, 0)])
    assert used2 == size  # everything coalesced back into one block, then fully used
