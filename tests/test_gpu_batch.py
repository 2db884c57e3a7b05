"""GPU tests of the batched codec (mans_batch_* in include/mans.h).

Every buffer's stream must be byte-identical to the single-buffer path (and
to the oracle for the small cases), decode back losslessly, and keep its own
status when another buffer of the batch fails."""
import numpy as np
import pytest

import mans_b200 as mb
from mans_b200 import workloads as W
from mans_b200.batch import Batch
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu

NP2T = {}
KIND = {np.uint8: "u8", np.uint16: "u16", np.uint32: "u32"}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    NP2T.update({np.uint8: torch.uint8, np.uint16: torch.uint16, np.uint32: torch.uint32})
    return torch


@pytest.fixture(scope="module")
def ws(torch_cuda):
    w = mb.Workspace(64 << 20)
    yield w
    w.close()


@pytest.fixture(scope="module")
def batch(torch_cuda):
    b = Batch(512, 256 << 20)
    yield b
    b.close()


def gen(kind: str, n: int, seed: int) -> np.ndarray:
    if kind == "u8":
        return W.random_bytes(n, seed, ("skewed", "uniform", "two", "sparse")[seed % 4])
    if kind == "u16":
        return (W.gradient_u16, W.laplace_u16, W.volume_u16)[seed % 3](n, seed)
    return (W.quant_u32, W.detector_u32)[seed % 2](n, seed)


EDGE = [0, 1, 31, 511, 512, 513, 4095, 4096, 4097, 16384, 70_001]


def mixed(seed: int, sizes) -> list[np.ndarray]:
    kinds = ("u8", "u16", "u32")
    return [gen(kinds[(i + seed) % 3], int(n), seed * 1000 + i) for i, n in enumerate(sizes)]


def single_stream(ws, x: np.ndarray, p: int) -> np.ndarray:
    return to_host(mb.compress(to_dev(x), p, ws=ws))


def run_compress(batch, xs, ps, caps=None):
    import torch
    dx = [to_dev(x) for x in xs]
    outs = []
    for i, x in enumerate(xs):
        cap = caps[i] if caps else mb.max_compressed_size(mb.dtype_code(dx[i]), x.size)
        outs.append(torch.empty(cap, dtype=torch.uint8, device="cuda"))
    sizes = torch.zeros(len(xs), dtype=torch.int64, device="cuda")
    items = batch.compress_items(dx, outs, sizes, ps)
    batch.compress_async(items)
    first, st, det = batch.status(len(xs))
    streams = [to_host(o[: int(n)]) for o, n in zip(outs, sizes.tolist())]
    return first, st, streams


def run_decompress(batch, streams, xs, in_bytes=None):
    import torch
    ds = [to_dev(s) if s.size else torch.zeros(16, dtype=torch.uint8, device="cuda")
          for s in streams]
    outs = [torch.empty(x.size, dtype=NP2T[x.dtype.type], device="cuda") for x in xs]
    sz = in_bytes if in_bytes is not None else [s.size for s in streams]
    items = batch.decompress_items(ds, sz, outs)
    batch.decompress_async(items)
    first, st, det = batch.status(len(xs))
    return first, st, [to_host(o, x.dtype) for o, x in zip(outs, xs)]


# ---------------------------------------------------------------- parity
def test_batch_edge_sizes_match_single_and_oracle(ws, batch, oracle):
    xs = mixed(1, EDGE * 3)
    ps = [9 + i % 3 for i in range(len(xs))]
    first, st, streams = run_compress(batch, xs, ps)
    assert first == 0 and not any(st), st
    for i, (x, p, s) in enumerate(zip(xs, ps, streams)):
        ref = oracle.compress(x, p) if x.dtype != np.uint8 else oracle.ans_encode(x, p)
        np.testing.assert_array_equal(s, ref, err_msg=f"item {i} {x.dtype} n={x.size} p={p}")
        np.testing.assert_array_equal(s, single_stream(ws, x, p), err_msg=f"item {i}")
    first, st, back = run_decompress(batch, streams, xs)
    assert first == 0 and not any(st), st
    for i, (x, y) in enumerate(zip(xs, back)):
        np.testing.assert_array_equal(y, x, err_msg=f"item {i}")


def test_batch_mixed_sizes_match_single(ws, batch, oracle):
    sizes_b = W.mixed_sizes(96, seed=11, lo=4 << 10, hi=2 << 20)
    kinds = ("u16", "u32", "u8")
    xs = []
    for i, nb in enumerate(sizes_b):
        k = kinds[i % 3]
        xs.append(gen(k, int(nb) // {"u8": 1, "u16": 2, "u32": 4}[k], 7000 + i))
    ps = [10] * len(xs)
    first, st, streams = run_compress(batch, xs, ps)
    assert first == 0 and not any(st)
    for i, (x, s) in enumerate(zip(xs, streams)):
        ref = oracle.compress_par(x, 10) if x.dtype != np.uint8 else oracle.ans_encode(x, 10)
        np.testing.assert_array_equal(s, ref, err_msg=f"item {i} against the oracle")
        np.testing.assert_array_equal(s, single_stream(ws, x, 10), err_msg=f"item {i}")
    first, st, back = run_decompress(batch, streams, xs)
    assert first == 0 and not any(st)
    for x, y in zip(xs, back):
        np.testing.assert_array_equal(y, x)


def test_batch_single_item_and_repeated_calls(ws, batch):
    # consecutive calls of different shapes reuse the workspace (device epoch)
    a = mixed(3, [100_000, 5_000, 0, 777])
    b = mixed(4, [1])
    for xs in (a, b, a, b, a):
        first, st, streams = run_compress(batch, xs, [11] * len(xs))
        assert first == 0
        for x, s in zip(xs, streams):
            np.testing.assert_array_equal(s, single_stream(ws, x, 11))
        first, st, back = run_decompress(batch, streams, xs)
        assert first == 0
        for x, y in zip(xs, back):
            np.testing.assert_array_equal(y, x)


# ---------------------------------------------------------------- errors stay per buffer
def test_batch_output_overflow_is_per_item(ws, batch):
    xs = mixed(5, [50_000, 60_000, 70_000, 80_000])
    caps = [mb.max_compressed_size({np.uint8: 1, np.uint16: 2, np.uint32: 4}[x.dtype.type], x.size)
            for x in xs]
    caps[2] = 1024  # far too small
    first, st, streams = run_compress(batch, xs, [10] * 4, caps)
    assert first == 8 and st[2] == 8
    for i in (0, 1, 3):
        assert st[i] == 0
        np.testing.assert_array_equal(streams[i], single_stream(ws, xs[i], 10))


def test_batch_bad_streams_are_per_item(batch, oracle):
    xs = mixed(6, [40_000, 40_000, 40_000, 40_000, 40_000])
    first, st, streams = run_compress(batch, xs, [10] * 5)
    assert first == 0
    bad = [s.copy() for s in streams]
    bad[1][0] ^= 0xFF            # magic
    bad[3][16] ^= 0x0F           # precision field
    sizes = [s.size for s in bad]
    sizes[4] = 100               # truncated
    first, st, back = run_decompress(batch, bad, xs, sizes)
    assert first == 7
    assert st[1] == 7 and st[3] == 7 and st[4] == 7
    for i in (0, 2):
        assert st[i] == 0
        np.testing.assert_array_equal(back[i], xs[i])


def test_batch_host_argument_errors(torch_cuda):
    import torch
    b = Batch(4, 1 << 20)
    try:
        x = torch.zeros(1000, dtype=torch.uint8, device="cuda")
        out = torch.empty(1 << 16, dtype=torch.uint8, device="cuda")
        sizes = torch.zeros(4, dtype=torch.int64, device="cuda")
        items = b.compress_items([x[1:]], [out], sizes, 10)
        with pytest.raises(mb.MansError) as e:
            b.compress_async(items)
        assert e.value.code == 3
        items = b.compress_items([x], [out], sizes, 8)
        with pytest.raises(mb.MansError) as e:
            b.compress_async(items)
        assert e.value.code == 2
        items = b.compress_items([x] * 5, [out] * 5, sizes, 10)
        with pytest.raises(mb.MansError) as e:
            b.compress_async(items)
        assert e.value.code == 4
        big = torch.zeros(2 << 20, dtype=torch.uint8, device="cuda")
        items = b.compress_items([big], [out], sizes, 10)
        with pytest.raises(mb.MansError) as e:
            b.compress_async(items)
        assert e.value.code == 4
    finally:
        b.close()


# ---------------------------------------------------------------- graph capture and schedules
def test_batch_cuda_graph_replay(ws, batch):
    import torch
    xs = mixed(8, [30_000, 4096, 123_457, 0, 9_999, 65_536])
    dx = [to_dev(x) for x in xs]
    outs = [torch.empty(mb.max_compressed_size(mb.dtype_code(d), d.numel()), dtype=torch.uint8,
                        device="cuda") for d in dx]
    sizes = torch.zeros(len(xs), dtype=torch.int64, device="cuda")
    items = Batch.compress_items(dx, outs, sizes, 10)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        batch.compress_async(items)  # warm-up outside capture
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        batch.compress_async(items)
    torch.cuda.synchronize()
    for rep in range(3):
        new = [gen(KIND[x.dtype.type], x.size, 900 + 10 * rep + i) for i, x in enumerate(xs)]
        for d, n in zip(dx, new):
            if n.size:
                d.copy_(to_dev(n))
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
        first, st, _ = batch.status(len(xs))
        assert first == 0
        for i, (n, o, sz) in enumerate(zip(new, outs, sizes.tolist())):
            np.testing.assert_array_equal(to_host(o[: int(sz)]), single_stream(ws, n, 10),
                                          err_msg=f"replay {rep} item {i}")
    del g


def test_batch_schedule_and_autotune_keep_bytes(ws, torch_cuda):
    import torch
    b = Batch(64, 64 << 20)
    try:
        xs = mixed(9, list(W.mixed_sizes(24, seed=9, lo=4 << 10, hi=1 << 20) // 4))
        ref = [single_stream(ws, x, 10) for x in xs]
        cur, mx = b.schedule()
        assert all(1 <= c <= m for c, m in zip(cur, mx))
        for sched in ([1] * 6, mx, [max(1, m // 2) for m in mx]):
            b.set_schedule(sched)
            first, st, streams = run_compress(b, xs, [10] * len(xs))
            assert first == 0
            for r, s in zip(ref, streams):
                np.testing.assert_array_equal(s, r)
        with pytest.raises(mb.MansError):
            b.set_schedule([0] * 6)
        dx = [to_dev(x) for x in xs]
        outs = [torch.empty(mb.max_compressed_size(mb.dtype_code(d), d.numel()),
                            dtype=torch.uint8, device="cuda") for d in dx]
        sizes = torch.zeros(len(xs), dtype=torch.int64, device="cuda")
        items = Batch.compress_items(dx, outs, sizes, 10)
        ms = b.autotune(items)
        assert ms > 0
        for r, o, n in zip(ref, outs, sizes.tolist()):
            np.testing.assert_array_equal(to_host(o[: int(n)]), r)
        cur, _ = b.schedule()
        first, st, streams = run_compress(b, xs, [10] * len(xs))
        for r, s in zip(ref, streams):
            np.testing.assert_array_equal(s, r)
    finally:
        b.close()


def test_batch_full_schedule_keeps_bytes(ws, torch_cuda):
    """Warps per CTA of the map stage (4 or 8) and the L2 prefetch distance of
    the map and encode stages change the schedule only: every stream equals
    the single-buffer path's and decodes back."""
    b = Batch(64, 64 << 20)
    try:
        xs = mixed(11, list(W.mixed_sizes(30, seed=11, lo=4 << 10, hi=2 << 20) // 4) + EDGE)
        ref = [single_stream(ws, x, 10) for x in xs]
        cur, lim = b.schedule_ex()
        assert cur["warps_per_cta"] == [8] * 6
        assert lim["prefetch_grids"][0] == 2 and lim["prefetch_grids"][2] == 2
        for warps, pf_map, pf_enc, frac in ((4, 0, 0, 1), (4, 2, 1, 2), (8, 0, 2, 1), (4, 1, 2, 4)):
            sch = {k: list(v) for k, v in cur.items()}
            sch["warps_per_cta"][0] = warps
            sch["prefetch_grids"][0] = pf_map
            sch["prefetch_grids"][2] = pf_enc
            sch["ctas_per_sm"] = [max(1, m // frac) for m in lim["ctas_per_sm"]]
            b.set_schedule_ex(sch)
            assert b.schedule_ex()[0] == sch
            first, st, streams = run_compress(b, xs, [10] * len(xs))
            assert first == 0, (sch, st)
            for i, (r, s) in enumerate(zip(ref, streams)):
                np.testing.assert_array_equal(s, r, err_msg=f"{sch} item {i}")
            first, st, back = run_decompress(b, streams, xs)
            assert first == 0
            for x, y in zip(xs, back):
                np.testing.assert_array_equal(y, x)
        for bad in ({"warps_per_cta": [6, 8, 8, 8, 8, 8]}, {"warps_per_cta": [8, 4, 8, 8, 8, 8]},
                    {"prefetch_grids": [3, 0, 0, 0, 0, 0]}, {"prefetch_grids": [0, 1, 0, 0, 0, 0]}):
            sch = {k: list(v) for k, v in cur.items()}
            sch.update(bad)
            with pytest.raises(mb.MansError):
                b.set_schedule_ex(sch)
    finally:
        b.close()
