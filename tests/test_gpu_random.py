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


def _u16(rng, n: int, full_range: bool = True) -> np.ndarray:
    fam = int(rng.integers(0, 6))
    if fam == 3 and not full_range:
        fam = 0
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


@pytest.mark.parametrize("seed", range(3))
def test_random_batch_matches_oracle(ws, oracle, seed):
    """40 random buffers of mixed type in one batched call per direction."""
    import torch

    from mans_b200.batch import Batch
    rng = np.random.default_rng(9100 + seed)
    xs, ps = [], []
    for i in range(40):
        kind = ("u8", "u16", "u32")[int(rng.integers(0, 3))]
        n = int(np.exp(rng.uniform(0.0, np.log(600_000))))
        if kind == "u8":
            xs.append(W.random_bytes(n, int(rng.integers(1 << 30)),
                                     str(rng.choice(["skewed", "uniform", "two", "sparse"]))))
        elif kind == "u16":
            # no full-range uint16: a small one maps to up to ~33x its bytes, past
            # the per-buffer room of any fixed ratio (it then fails alone)
            xs.append(_u16(rng, n, full_range=False))
        else:
            xs.append(_u32(rng, n))
        ps.append(int(rng.integers(9, 12)))
    refs = [oracle.ans_encode(x, p) if x.dtype == np.uint8 else oracle.compress(x, p)
            for x, p in zip(xs, ps)]
    tdt = {np.uint8: torch.uint8, np.uint16: torch.uint16, np.uint32: torch.uint32}
    # wide uint16 spreads map to up to ~8x their bytes here; the default room
    # (210%) would fail those buffers alone with MANS_ERR_WORKSPACE_OVERFLOW
    b = Batch(64, 64 << 20, 1000)
    try:
        dx = [to_dev(x) for x in xs]
        outs = [torch.empty(mb.max_compressed_size(mb.dtype_code(d), d.numel()),
                            dtype=torch.uint8, device="cuda") for d in dx]
        sizes = torch.zeros(len(xs), dtype=torch.int64, device="cuda")
        b.compress_async(Batch.compress_items(dx, outs, sizes, ps))
        b.check(len(xs), what="random batch compress")
        streams = [to_host(o[: int(n)]) for o, n in zip(outs, sizes.tolist())]
        for i, (s, r) in enumerate(zip(streams, refs)):
            np.testing.assert_array_equal(s, r, err_msg=f"seed {seed} item {i} {xs[i].dtype} n={xs[i].size}")
        ds = [to_dev(s) for s in streams]
        backs = [torch.empty(x.size, dtype=tdt[x.dtype.type], device="cuda") for x in xs]
        b.decompress_async(Batch.decompress_items(ds, [s.size for s in streams], backs))
        b.check(len(xs), what="random batch decompress")
        for i, (x, y) in enumerate(zip(xs, backs)):
            np.testing.assert_array_equal(to_host(y, x.dtype), x, err_msg=f"seed {seed} item {i}")
    finally:
        b.close()
