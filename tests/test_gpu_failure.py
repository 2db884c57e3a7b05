"""Failure path on the GPU without a fault: a bounded device wait that
nothing satisfies must end with MANS_ERR_TIMEOUT and leave the context
usable (the next codec call works)."""
import ctypes as C

import numpy as np
import pytest

import mans_b200 as mb
from mans_b200 import workloads as W
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives(oracle):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    st, ms = C.c_uint32(0), C.c_float(0)
    assert mb.load().mans_debug_bounded_wait(C.byref(st), C.byref(ms)) == 0
    assert st.value == 11  # MANS_ERR_TIMEOUT
    assert 10.0 < ms.value < 30_000.0
    x = W.laplace_u16(100_000, 3)
    s = to_host(mb.compress(to_dev(x), 10))
    np.testing.assert_array_equal(s, oracle.compress(x, 10))
    y = mb.decompress(to_dev(s), x.size, torch.uint16)
    np.testing.assert_array_equal(to_host(y, np.uint16), x)
