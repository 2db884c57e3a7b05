"""GPU parity tests: the CUDA path (through the C ABI) against the oracle.

Bit-exact for every stream byte and every decoded value."""
import numpy as np
import pytest

import mans_b200 as mb
from mans_b200 import workloads as W
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def ws(torch_cuda):
    w = mb.Workspace(64 << 20)
    yield w
    w.close()


def gpu_compress(ws, x: np.ndarray, p: int) -> np.ndarray:
    import torch
    d = to_dev(x)
    code = mb.dtype_code(d)
    cap = mb.max_compressed_size(code, x.size)
    out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    mb.compress_into(ws, d, out, size, p)
    ws.check(what="compress")
    return to_host(out[: int(size.item())])


def gpu_decompress(ws, s: np.ndarray, n: int, dtype) -> np.ndarray:
    import torch
    tdt = {np.uint8: torch.uint8, np.uint16: torch.uint16, np.uint32: torch.uint32}[dtype]
    out = torch.empty(max(n, 1) * np.dtype(dtype).itemsize, dtype=torch.uint8,
                      device="cuda").view(tdt)[:n]
    sd = to_dev(s) if s.size else torch.zeros(16, dtype=torch.uint8, device="cuda")
    mb.decompress_into(ws, sd, s.size, out)
    ws.check(what="decompress")
    return to_host(out, dtype)


# ---------------------------------------------------------------- rANS over bytes
@pytest.mark.parametrize("p", [9, 10, 11])
@pytest.mark.parametrize("kind", ["skewed", "uniform", "single", "two", "sparse"])
def test_ans_bytes_parity(ws, oracle, p, kind):
    for i, n in enumerate([0, 1, 31, 32, 33, 4095, 4096, 4097, 100_000, 1 << 20]):
        x = W.random_bytes(n, 1000 + i, kind)
        s = gpu_compress(ws, x, p)
        ref = oracle.ans_encode(x, p)
        assert s.size == ref.size, (n, kind)
        np.testing.assert_array_equal(s, ref, err_msg=f"n={n} kind={kind} p={p}")
        np.testing.assert_array_equal(gpu_decompress(ws, s, n, np.uint8), x)


def test_ans_blocks_near_the_word_bound(ws, oracle):
    """Blocks of rare symbols at p = 11: each symbol has frequency 1 and costs
    11 bits, so a block takes about 2,816 words -- past the point where the
    encoder checks its word buffer step by step. Streams stay bit-exact."""
    n = 1 << 20
    x = np.zeros(n, np.uint8)
    for blk in (3, 100, 255):  # whole 4 KiB blocks of symbols 1..255
        x[blk * 4096:(blk + 1) * 4096] = 1 + np.arange(4096) % 255
    ref, bw = oracle.ans_encode(x, 11, with_block_words=True)
    assert int(bw.max()) > 2632  # the guarded tail runs
    s = gpu_compress(ws, x, 11)
    np.testing.assert_array_equal(s, ref)
    y = mb.decompress(to_dev(s), n, __import__("torch").uint8, ws=ws)
    np.testing.assert_array_equal(to_host(y), x)


def test_ans_decode_of_oracle_stream(ws, oracle):
    x = W.random_bytes(300_000, 5, "skewed")
    s = oracle.ans_encode(x, 11)
    np.testing.assert_array_equal(gpu_decompress(ws, s, x.size, np.uint8), x)


# ---------------------------------------------------------------- uint16 (ADM V15 + rANS)
U16_SIZES = [1, 7, 8, 15, 16, 17, 511, 512, 513, 4095, 4096, 4097, 32768, 100_003]


@pytest.mark.parametrize("gen", ["laplace", "volume", "gradient", "wide"])
def test_u16_parity(ws, oracle, gen):
    for i, n in enumerate(U16_SIZES):
        x = {"laplace": lambda: W.laplace_u16(n, 50 + i),
             "volume": lambda: W.volume_u16(n, 60 + i),
             "gradient": lambda: W.gradient_u16(n, 70 + i),
             "wide": lambda: W.laplace_u16(n, 80 + i, b=3000.0)}[gen]()
        p = (9, 10, 11)[i % 3]
        s = gpu_compress(ws, x, p)
        ref = oracle.compress(x, p)
        assert s.size == ref.size, (gen, n)
        np.testing.assert_array_equal(s, ref, err_msg=f"{gen} n={n}")
        np.testing.assert_array_equal(gpu_decompress(ws, s, n, np.uint16), x)


def test_u16_long_lanes(ws, oracle):
    """Lanes beyond 64 and beyond 256 bits (the reference's own lane buffer):
    the byte-wise paths of map and unmap."""
    rng = np.random.default_rng(3)
    x = np.tile(np.array([0, 65535], np.uint16), 4096)
    y = np.clip(np.round(30000 + rng.laplace(0, 5000, 9000)), 0, 65535).astype(np.uint16)
    for v in (x, y):
        s = gpu_compress(ws, v, 10)
        np.testing.assert_array_equal(s, oracle.compress(v, 10))
        np.testing.assert_array_equal(gpu_decompress(ws, s, v.size, np.uint16), v)


def test_u16_config1_full(ws, oracle):
    x = W.laplace_u16(W.C1_N, 1)
    s = gpu_compress(ws, x, 10)
    np.testing.assert_array_equal(s, oracle.compress(x, 10))
    np.testing.assert_array_equal(gpu_decompress(ws, s, x.size, np.uint16), x)


# ---------------------------------------------------------------- uint32 (ADM V9 + rANS)
@pytest.mark.parametrize("gen", ["detector", "quant", "random"])
def test_u32_parity(ws, oracle, gen):
    for i, n in enumerate([1, 15, 16, 17, 512, 513, 4096, 4097, 65_537, 300_000]):
        x = {"detector": lambda: W.detector_u32(n, 90 + i),
             "quant": lambda: W.quant_u32(n, 100 + i),
             "random": lambda: np.random.default_rng(110 + i).integers(0, 2**32, n, dtype=np.uint32)}[gen]()
        p = (9, 10, 11)[i % 3]
        s = gpu_compress(ws, x, p)
        ref = oracle.compress(x, p)
        assert s.size == ref.size, (gen, n)
        np.testing.assert_array_equal(s, ref, err_msg=f"{gen} n={n}")
        np.testing.assert_array_equal(gpu_decompress(ws, s, n, np.uint32), x)


# ---------------------------------------------------------------- reference-named entry points
def test_reference_entry_points(torch_cuda, oracle):
    import torch
    for n in [0, 100, 4096, 123_457]:
        x = W.random_bytes(n, 9, "skewed")
        d = to_dev(x) if n else torch.zeros(16, dtype=torch.uint8, device="cuda")
        cap = mb.getMaxCompressedSize(n)
        out = torch.empty(cap, dtype=torch.uint8, device="cuda")
        size = torch.zeros(1, dtype=torch.int32, device="cuda")
        mb.ansEncode(10, d, n, out, size)
        assert mb.ans_last_status()[0] == 0
        s = to_host(out[: int(size.item())])
        np.testing.assert_array_equal(s, oracle.ans_encode(x, 10))
        dec = torch.empty(max(n, 16), dtype=torch.uint8, device="cuda")
        mb.ansDecode(10, out, dec)
        assert mb.ans_last_status()[0] == 0
        np.testing.assert_array_equal(to_host(dec[:n]), x)
    # precision mismatch against the header is a bad stream, not a device assert
    mb.ansDecode(9, out, dec)
    assert mb.STATUS[mb.ans_last_status()[0]] == "MANS_ERR_BAD_STREAM"


# ---------------------------------------------------------------- errors without faults
def test_bad_streams_report_status(ws, oracle):
    import torch
    x = W.laplace_u16(20_000, 3)
    s = oracle.compress(x, 10)
    out = torch.empty(x.size, dtype=torch.uint16, device="cuda")

    def dec(buf, size=None):
        mb.decompress_into(ws, to_dev(buf), buf.size if size is None else size, out)
        return ws.status()[0]

    bad = s.copy()
    bad[3] ^= 0x40  # magic
    assert mb.STATUS[dec(bad)] == "MANS_ERR_BAD_STREAM"
    assert mb.STATUS[dec(s, size=600)] == "MANS_ERR_BAD_STREAM"  # truncated
    bad = s.copy()
    bad[16] = 12  # precision 12
    assert mb.STATUS[dec(bad)] == "MANS_ERR_BAD_STREAM"
    bad = s.copy()
    bad[-64:] ^= 0x5A  # payload corruption: detected by the per-block checks
    st = dec(bad)
    assert mb.STATUS[st] in ("MANS_ERR_CORRUPT", "MANS_OK")
    assert dec(s) == 0
    np.testing.assert_array_equal(to_host(out, np.uint16), x)


def test_output_overflow_reports_status(ws):
    import torch
    x = to_dev(W.random_bytes(50_000, 4, "uniform"))
    out = torch.empty(1024, dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    mb.compress_into(ws, x, out, size, 10)
    st, need = ws.status()
    assert mb.STATUS[st] == "MANS_ERR_OUTPUT_OVERFLOW" and need > 1024


def test_workspace_overflow_reports_status(torch_cuda, oracle):
    import torch
    small = mb.Workspace(1 << 16, merged_capacity=40_000)
    x = np.tile(np.array([0, 65535], np.uint16), 8192)  # maps to ~65 bytes per element
    d = to_dev(x)
    out = torch.empty(mb.max_compressed_size(mb.MANS_U16, x.size), dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    mb.compress_into(small, d, out, size, 10)
    st, need = small.status()
    assert mb.STATUS[st] == "MANS_ERR_WORKSPACE_OVERFLOW"
    assert need == oracle.adm_u16_map(x).size
    # after reading the status the workspace is usable again
    y = W.laplace_u16(8192, 1)
    mb.compress_into(small, to_dev(y), out, size, 10)
    assert small.status()[0] == 0
    np.testing.assert_array_equal(to_host(out[: int(size.item())]), oracle.compress(y, 10))
    small.close()


def test_worst_case_bounds_size_the_widest_uint16_data(torch_cuda, oracle):
    """Sized only by the library's worst-case bounds -- mans_max_mapped_size
    for the workspace's mapped capacity, mans_max_compressed_size for the
    output -- the widest uint16 data (alternating 0 / 65535, about 65 mapped
    bytes per element; one lane of 65535 per group over zeros) compresses to
    the oracle's stream and decodes back."""
    import torch
    n = 65_536
    one_lane = np.zeros(n, np.uint16)
    one_lane.reshape(-1, 512)[:, :16] = 65535
    for x in (np.tile(np.array([0, 65535], np.uint16), n // 2), one_lane):
        w = mb.Workspace(2 * n, merged_capacity=mb.max_mapped_size(mb.MANS_U16, n))
        out = torch.empty(mb.max_compressed_size(mb.MANS_U16, n), dtype=torch.uint8, device="cuda")
        size = torch.zeros(1, dtype=torch.int64, device="cuda")
        d = to_dev(x)
        mb.compress_into(w, d, out, size, 10)
        w.check(None, "compress")
        got = to_host(out[: int(size.item())])
        want = oracle.compress(x, 10)
        assert oracle.adm_u16_map(x).size > 2.1 * 2 * n  # beyond the default workspace
        np.testing.assert_array_equal(got, want)
        back = torch.empty_like(d)
        mb.decompress_into(w, out, got.size, back)
        w.check(None, "decompress")
        np.testing.assert_array_equal(to_host(back, np.uint16), x)
        w.close()


def test_repeated_calls_identical(ws):
    x = W.detector_u32(200_000, 8)
    a = gpu_compress(ws, x, 10)
    b = gpu_compress(ws, x, 10)
    np.testing.assert_array_equal(a, b)


def test_single_path_cuda_graph_replay(ws, oracle):
    """mans_compress / mans_decompress captured in a CUDA graph and replayed
    with new input: every stream and value matches (the look-back epoch and
    all bounds live on the device)."""
    import torch
    n = 300_001
    x0 = W.laplace_u16(n, 41)
    dx = to_dev(x0)
    cap = mb.max_compressed_size(2, n)
    out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    back = torch.empty(n, dtype=torch.uint16, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        mb.compress_into(ws, dx, out, size, 10, s)
        mb.decompress_into(ws, out, cap, back, s)
    torch.cuda.synchronize()
    ws.check(what="warm-up")
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        mb.compress_into(ws, dx, out, size, 10, s)
        mb.decompress_into(ws, out, cap, back, s)
    torch.cuda.synchronize()
    for rep in range(3):
        x = (W.laplace_u16, W.gradient_u16, W.volume_u16)[rep](n, 50 + rep)
        dx.copy_(to_dev(x))
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
        ws.check(what=f"replay {rep}")
        np.testing.assert_array_equal(to_host(out[: int(size.item())]), oracle.compress(x, 10))
        np.testing.assert_array_equal(to_host(back, np.uint16), x)
    del g


# ---------------------------------------------------------------- maximum sizes
def _free_gib():
    import torch
    free, _ = torch.cuda.mem_get_info()
    return free / (1 << 30)


def test_max_size_u32_round_trip(torch_cuda):
    """2^30 uint32 values (4 GiB; the reference's uint32 mapper is limited to
    2^27 per call): bit-exact round trip and a stream that the decoder
    accepts; the mapped size stays below the 32-bit stream field."""
    import torch

    import bench
    if _free_gib() < 40:
        pytest.skip("needs ~40 GiB free")
    n = 1 << 30
    x = bench.gen_device("detector_u32", n, 12)
    w = mb.Workspace(n * 4)
    try:
        s = mb.compress(x, 10, ws=w)
        hdr = to_host(s[:32]).view(np.uint32)
        assert hdr[0] == 0xD00D0001 and hdr[2] < (1 << 32) - 16
        y = mb.decompress(s, n, torch.uint32, ws=w)
        assert torch.equal(y, x)
    finally:
        w.close()


def test_max_size_u8_round_trip(torch_cuda):
    """4.0e9 raw bytes, just below the stream's 32-bit byte count."""
    import torch
    if _free_gib() < 30:
        pytest.skip("needs ~30 GiB free")
    n = 4_000_000_000
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    x = (torch.randint(0, 16, (n,), device="cuda", dtype=torch.uint8, generator=g) *
         torch.randint(0, 2, (n,), device="cuda", dtype=torch.uint8, generator=g))
    w = mb.Workspace(n)
    try:
        s = mb.compress(x, 11, ws=w)
        hdr = to_host(s[:32]).view(np.uint32)
        assert int(hdr[2]) == n and int(hdr[1]) == -(-n // 4096)
        y = mb.decompress(s, n, torch.uint8, ws=w)
        assert torch.equal(y, x)
    finally:
        w.close()
