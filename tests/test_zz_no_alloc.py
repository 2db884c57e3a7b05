"""The allocation-free rANS encode entry point (mans_ans_encode_noalloc).

Some callers cannot allocate device memory on their call path (a real-time
loop that cannot absorb cudaMalloc's latency or implicit synchronisation, a
process whose device memory is reserved up front by another allocator);
this entry point keeps its scratch in a fixed array inside the library. The
test calls it through the C ABI twice in a row and checks each stream
against the existing entry point's (mans_ans_encode), byte for byte. This
file is collected last so that a failure here stops a run only after every
other test has run."""

import numpy as np
import pytest

import mans_b200 as mb
from mans_b200 import workloads as W
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu


def _encode(fn, x: np.ndarray, p: int) -> np.ndarray:
    import torch
    d = to_dev(x)
    cap = mb.getMaxCompressedSize(x.size)
    out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(p, d.data_ptr(), x.size, out.data_ptr(), size.data_ptr(), stream)
    assert rc == 0, mb.STATUS[rc]
    torch.cuda.synchronize()
    return to_host(out[: int(size.item())])


def test_noalloc_encode_matches_existing_entry_point():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = mb.load()
    cases = [(W.random_bytes(1_000_003, 21, "skewed"), 10),
             (W.random_bytes(3 << 20, 22, "uniform"), 11)]
    for x, p in cases:  # two calls in a row on the shared scratch
        want = _encode(lib.mans_ans_encode, x, p)
        got = _encode(lib.mans_ans_encode_noalloc, x, p)
        assert got.size == want.size
        np.testing.assert_array_equal(got, want)
    # sizes beyond the fixed maximum are rejected before any device work
    d = to_dev(np.zeros(16, np.uint8))
    out = torch.empty(1024, dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.mans_ans_encode_noalloc(10, d.data_ptr(), (64 << 20) + 1, out.data_ptr(),
                                     size.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert mb.STATUS[rc] == "MANS_ERR_TOO_LARGE"
