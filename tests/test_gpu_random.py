"""Seeded randomized parity sweep of the whole codec: random element type,
size (0 to 2 M elements), value distribution, precision and (uint16) file
layout per case. Every stream byte must equal the oracle's and every
decompressed value the input."""
import numpy as np
import pytest

import mans_b200 as mb
from mans_b200 import workloads as W
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu

CASES = 48


@pytest.fixture(scope="module")
def ws():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    w = mb.Workspace(64 << 20)
    yield w
    w.close()


def _u16(rng, n: int) -> np.ndarray:
    fam = int(rng.integers(0, 6))
    seed = int(rng.integers(1 << 30))
    if fam == 0:
        b = float(rng.choice([2.0, 40.0, 400.0, 4000.0]))
        return W.laplace_u16(n, seed, b=b, center=float(rng.integers(0, 65536)))
    if fam == 1:
        return W.gradient_u16(n, seed)
    if fam == 2:
        return W.volume_u16(n, seed)
    if fam == 3:  # full range: long lanes (the byte-by-byte path)
        return rng.integers(0, 65536, min(n, 100_000), dtype=np.uint16)
    if fam == 4:
        return np.full(n, rng.integers(0, 65536), np.uint16)
    return (rng.integers(0, 4, n) * int(rng.integers(1, 16_000))).astype(np.uint16)


def _u32(rng, n: int) -> np.ndarray:
    fam = int(rng.integers(0, 6))
    seed = int(rng.integers(1 << 30))
    if fam == 0:
        return W.detector_u32(n, seed, peak_frac=float(rng.choice([0.0, 0.001, 0.2])))
    if fam == 1:
        return W.quant_u32(n, seed, b=float(rng.choice([3.0, 300.0, 30_000.0])))
    if fam == 2:  # escapes everywhere
        return rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    if fam == 3:
        return np.full(n, rng.integers(0, 1 << 32), np.uint32)
    if fam == 4:  # just below 2^32: 64-bit center sums and no wrap
        return (np.uint64(0xFFFFFFFF) - rng.integers(0, 1000, n).astype(np.uint64)).astype(np.uint32)
    v = np.zeros(n, np.uint32)
    m = rng.random(n) < 0.01
    v[m] = rng.integers(0, 1 << 32, int(m.sum()), dtype=np.uint64).astype(np.uint32)
    return v


@pytest.mark.parametrize("case", range(CASES))
def test_random_case_matches_oracle(ws, oracle, case):
    import torch
    rng = np.random.default_rng(7000 + case)
    kind = ("u8", "u16", "u32")[case % 3]
    n = int(np.exp(rng.uniform(0.0, np.log(2e6))))
    if case % 7 == 0:
        n = int(rng.integers(0, 600))
    elif case % 4 == 1:
        n = int(rng.integers(1 << 18, 2_000_000))
    p = int(rng.integers(9, 12))
    layout = mb.LAYOUT_NATIVE
    if kind == "u8":
        x = W.random_bytes(n, int(rng.integers(1 << 30)),
                           str(rng.choice(["skewed", "uniform", "single", "two", "sparse"])))
        ref = oracle.ans_encode(x, p)
    elif kind == "u16":
        x = _u16(rng, n)
        layout = int(rng.choice([mb.LAYOUT_NATIVE, mb.LAYOUT_V12, mb.LAYOUT_CPUV2]))
        ref = oracle.compress(x, p, layout)
    else:
        x = _u32(rng, n)
        ref = oracle.compress(x, p)
    what = f"case {case}: {kind} n={x.size} p={p} layout={layout}"
    s = to_host(mb.compress(to_dev(x), p, ws=ws, layout=layout))
    np.testing.assert_array_equal(s, ref, err_msg=what)
    tdt = {np.uint8: torch.uint8, np.uint16: torch.uint16, np.uint32: torch.uint32}[x.dtype.type]
    y = mb.decompress(to_dev(s), x.size, tdt, ws=ws, layout=layout)
    np.testing.assert_array_equal(to_host(y, x.dtype), x, err_msg=what)
