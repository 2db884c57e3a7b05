"""The allocation-free rANS encode entry point (mans_ans_encode_noalloc).

Some callers cannot allocate device memory on their call path (a real-time
loop that cannot absorb cudaMalloc's latency or implicit synchronisation, a
process whose device memory is reserved up front by another allocator);
this entry point keeps its scratch in a fixed array inside the library. The
test calls it through the C ABI, several calls in a row on the shared
scratch, and checks each stream byte for byte against the oracle's encoder
and against the existing entry point (mans_ans_encode), reads the device
status through mans_ans_noalloc_status, and decodes the stream back through
mans_ans_decode. Sizes cover the empty input, ragged and multi-megabyte
inputs, and the 64 MiB maximum (the last look-back flag slots). This file is
collected last so that a failure here stops a run only after every other
test has run."""

import numpy as np
import pytest

import mans_b200 as mb
from mans_b200 import workloads as W
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu

MAX_BYTES = 64 << 20


def _encode(fn, x: np.ndarray, p: int) -> np.ndarray:
    import torch
    d = to_dev(x)
    cap = mb.getMaxCompressedSize(x.size)
    out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(p, d.data_ptr() if x.size else None, x.size, out.data_ptr(), size.data_ptr(), stream)
    assert rc == 0, mb.STATUS[rc]
    torch.cuda.synchronize()
    return to_host(out[: int(size.item())])


def _noalloc_status() -> int:
    import ctypes as C

    import torch
    detail = C.c_uint64(0)
    return mb.load().mans_ans_noalloc_status(torch.cuda.current_stream().cuda_stream,
                                             C.byref(detail))


def _decode(s: np.ndarray, n: int, p: int) -> np.ndarray:
    import torch
    d = to_dev(s)
    out = torch.empty(max(n, 16), dtype=torch.uint8, device="cuda")
    rc = mb.load().mans_ans_decode(p, d.data_ptr(), out.data_ptr(),
                                   torch.cuda.current_stream().cuda_stream)
    assert rc == 0, mb.STATUS[rc]
    st, det = mb.ans_last_status()
    assert st == 0, (mb.STATUS[st], det)
    return to_host(out[:n])


def test_noalloc_encode_matches_oracle_and_existing_entry_point(oracle):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = mb.load()
    cases = [(W.random_bytes(1_000_003, 21, "skewed"), 10),
             (W.random_bytes(3 << 20, 22, "uniform"), 11),
             (np.zeros(0, np.uint8), 10),
             (W.random_bytes(4095, 23, "sparse"), 9),
             (W.random_bytes(MAX_BYTES, 24, "skewed"), 10),
             (W.random_bytes(1_000_003, 21, "skewed"), 10)]
    for x, p in cases:  # calls in a row on the shared scratch
        got = _encode(lib.mans_ans_encode_noalloc, x, p)
        assert _noalloc_status() == 0
        want = oracle.ans_encode(x, p)
        assert got.size == want.size, (x.size, got.size, want.size)
        np.testing.assert_array_equal(got, want)
        np.testing.assert_array_equal(got, _encode(lib.mans_ans_encode, x, p))
        if x.size:
            np.testing.assert_array_equal(_decode(got, x.size, p), x)


def test_noalloc_encode_rejects_sizes_beyond_its_maximum():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = mb.load()
    d = to_dev(np.zeros(16, np.uint8))
    out = torch.empty(1024, dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.mans_ans_encode_noalloc(10, d.data_ptr(), MAX_BYTES + 1, out.data_ptr(),
                                     size.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert mb.STATUS[rc] == "MANS_ERR_TOO_LARGE"
