"""GPU tests of the serving loop (mans_server_* in include/mans.h): every
result is byte-identical to the single-buffer call of that request alone,
errors stay with their request, and admission waits for memory."""
import numpy as np
import pytest

import mans_b200 as mb
from mans_b200 import serve
from mans_b200 import workloads as W
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu
CODE = {np.uint8: 1, np.uint16: 2, np.uint32: 4}


@pytest.fixture(scope="module")
def ws():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    w = mb.Workspace(64 << 20)
    yield w
    w.close()


def gen(i: int, n: int) -> np.ndarray:
    k = i % 3
    if k == 0:
        return W.random_bytes(n, 100 + i, ("skewed", "two", "uniform")[(i // 3) % 3])
    if k == 1:
        return (W.gradient_u16, W.laplace_u16)[i % 2](n, 200 + i)
    return (W.quant_u32, W.detector_u32)[i % 2](n, 300 + i)


def host_bytes(ptr: int, nbytes: int) -> np.ndarray:
    return serve.view_device(ptr, nbytes).cpu().numpy()


def drain(srv, want: int, release: bool = True, timeout_s: float = 60.0):
    import time
    done = {}
    t0 = time.time()
    while len(done) < want:
        for c in srv.poll(timeout_us=20_000):
            done[c.ticket] = (c, host_bytes(c.d_out, c.out_bytes) if c.status == 0 and c.d_out else None)
            if release and c.status == 0 and c.d_out:
                srv.release(c.ticket)
        assert time.time() - t0 < timeout_s, f"only {len(done)} of {want} completed"
    return done


SIZES = [0, 1, 511, 4097, 30_000, 70_001, 200_000, 1 << 20]


@pytest.mark.parametrize("plain", [False, True])
def test_server_results_identical_to_single_calls(ws, plain):
    xs = [gen(i, n) for i, n in enumerate(SIZES * 2)]
    ref = [to_host(mb.compress(to_dev(x), 10, ws=ws)) for x in xs]
    srv = serve.Server(2 << 30, max_batch_bytes=64 << 20, plain=plain)
    try:
        dx = [to_dev(x) for x in xs]
        ds = [to_dev(s) for s in ref]
        tickets = {}
        for i, (x, d, s) in enumerate(zip(xs, dx, ds)):
            t = srv.submit(serve.COMPRESS, CODE[x.dtype.type], x.size, d.data_ptr() if x.size else None,
                           precision=10, tag=i)
            tickets[t] = ("c", i)
            t = srv.submit(serve.DECOMPRESS, CODE[x.dtype.type], x.size, s.data_ptr(),
                           in_bytes=ref[i].size, tag=i)
            tickets[t] = ("d", i)
        done = drain(srv, len(tickets))
        for t, (c, data) in done.items():
            kind, i = tickets[t]
            assert c.status == 0, (kind, i, c.status)
            if kind == "c":
                np.testing.assert_array_equal(data, ref[i], err_msg=f"compress {i}")
            else:
                np.testing.assert_array_equal(data, xs[i].view(np.uint8), err_msg=f"decompress {i}")
        st = srv.stats()
        assert st["completed"] == len(tickets) and st["arena_used"] == 0
        if plain:
            assert st["launches"] == len(tickets)
    finally:
        srv.close()


def test_server_errors_stay_with_their_request(ws):
    xs = [gen(i, 50_000) for i in range(6)]
    ref = [to_host(mb.compress(to_dev(x), 10, ws=ws)) for x in xs]
    bad = ref[2].copy()
    bad[0] ^= 0xFF
    streams = [to_dev(s) for s in ref[:2]] + [to_dev(bad)] + [to_dev(s) for s in ref[3:]]
    srv = serve.Server(1 << 30, max_batch_bytes=16 << 20)
    try:
        tick = [srv.submit(serve.DECOMPRESS, CODE[x.dtype.type], x.size, s.data_ptr(),
                           in_bytes=r.size, tag=i) for i, (x, s, r) in enumerate(zip(xs, streams, ref))]
        done = drain(srv, len(tick))
        for i, t in enumerate(tick):
            c, data = done[t]
            if i == 2:
                assert c.status == 7 and data is None
            else:
                assert c.status == 0
                np.testing.assert_array_equal(data.view(xs[i].dtype), xs[i])
    finally:
        srv.close()


def test_server_admission_waits_for_memory(ws):
    # the arena holds only a few worst-case outputs: requests wait in the
    # queue until earlier results are released, and all complete
    xs = [gen(3 * i + 1, 2 << 20) for i in range(24)]  # 4 MiB of uint16 each
    ref = [to_host(mb.compress(to_dev(x), 10, ws=ws)) for x in xs]
    srv = serve.Server(256 << 20, max_batch_bytes=8 << 20, max_batch_items=8, lanes=1)
    try:
        st = srv.stats()
        assert st["device_bytes"] <= 256 << 20
        # fewer worst-case outputs fit in the arena than there are requests
        assert st["arena_bytes"] < 24 * (4 << 20) * 2
        dx = [to_dev(x) for x in xs]
        tick = [srv.submit(serve.COMPRESS, 2, x.size, d.data_ptr(), precision=10)
                for x, d in zip(xs, dx)]
        done = drain(srv, len(tick))
        for i, t in enumerate(tick):
            c, data = done[t]
            assert c.status == 0
            np.testing.assert_array_equal(data, ref[i])
        assert srv.stats()["arena_peak"] <= srv.stats()["arena_bytes"]
    finally:
        srv.close()


def test_server_rejects_what_can_never_fit(ws):
    import torch
    srv = serve.Server(512 << 20, max_batch_bytes=8 << 20, lanes=1)
    try:
        x = torch.zeros(16 << 20, dtype=torch.uint8, device="cuda")
        with pytest.raises(mb.MansError) as e:
            srv.submit(serve.COMPRESS, 1, x.numel(), x.data_ptr(), precision=10)
        assert e.value.code == 4
        with pytest.raises(mb.MansError) as e:
            srv.submit(serve.COMPRESS, 1, 100, x.data_ptr() + 1, precision=10)
        assert e.value.code == 3
        with pytest.raises(mb.MansError) as e:
            srv.submit(serve.COMPRESS, 1, 100, x.data_ptr(), precision=12)
        assert e.value.code == 2
    finally:
        srv.close()


def test_server_caller_owned_outputs(ws):
    import torch
    xs = [gen(3 * i + 2, 100_000 + 17 * i) for i in range(5)]
    ref = [to_host(mb.compress(to_dev(x), 11, ws=ws)) for x in xs]
    outs = [torch.zeros(mb.max_compressed_size(4, x.size), dtype=torch.uint8, device="cuda") for x in xs]
    srv = serve.Server(1 << 30, max_batch_bytes=16 << 20)
    try:
        dx = [to_dev(x) for x in xs]
        tick = [srv.submit(serve.COMPRESS, 4, x.size, d.data_ptr(), precision=11, d_out=o.data_ptr(),
                           out_capacity=o.numel()) for x, d, o in zip(xs, dx, outs)]
        done = drain(srv, len(tick), release=False)
        for i, t in enumerate(tick):
            c, _ = done[t]
            assert c.status == 0 and c.d_out == outs[i].data_ptr()
            np.testing.assert_array_equal(to_host(outs[i][: c.out_bytes]), ref[i])
        assert srv.stats()["arena_used"] == 0
    finally:
        srv.close()


def test_server_admits_requests_while_a_batch_runs(ws, oracle):
    """Continuous batching: with one lane per direction, a 1 GiB compress
    request occupies the compress lane for milliseconds; 16 small requests
    submitted meanwhile (while it is in flight) are admitted, wait for the
    lane, and then run together in one batch of more than one item. Every
    small result equals the oracle's stream of that request alone."""
    import torch
    big = W.gen_device("volume_u16", 1 << 29, 31)
    smalls = [W.gradient_u16(65_536 + 512 * i, 400 + i) for i in range(16)]
    ds = [to_dev(x) for x in smalls]
    srv = serve.Server(8 << 30, max_batch_bytes=(1 << 30) + (64 << 20), max_batch_items=64, lanes=1)
    try:
        torch.cuda.synchronize()
        t_big = srv.submit(serve.COMPRESS, 2, big.numel(), big.data_ptr(), precision=10, tag=999)
        import time
        t0 = time.time()
        while srv.stats()["in_flight"] == 0 and srv.stats()["completed"] == 0:
            assert time.time() - t0 < 10, "the large request was never dispatched"
        in_flight_before = srv.stats()["in_flight"]
        tick = [srv.submit(serve.COMPRESS, 2, x.size, d.data_ptr(), precision=10, tag=i)
                for i, (x, d) in enumerate(zip(smalls, ds))]
        still_running = srv.stats()["completed"] == 0
        done = drain(srv, len(tick) + 1)
        assert in_flight_before >= 1 and still_running, "the large request finished too early"
        assert done[t_big][0].status == 0 and done[t_big][0].batch_items == 1
        items = [done[t][0].batch_items for t in tick]
        assert max(items) > 1, items
        for i, t in enumerate(tick):
            c, data = done[t]
            assert c.status == 0
            np.testing.assert_array_equal(data, oracle.compress(smalls[i], 10), err_msg=f"request {i}")
    finally:
        srv.close()
