"""GPU tests of self-describing frames: header fields, the body equal to the
plain stream (and the oracle's), and decoding from the frame alone."""
import numpy as np
import pytest

import mans_b200 as mb
from mans_b200 import workloads as W
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ws():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    w = mb.Workspace(64 << 20)
    yield w
    w.close()


CASES = [("u8", 0), ("u16", 0), ("u16", 1), ("u16", 2), ("u32", 0)]


@pytest.mark.parametrize("kind,layout", CASES)
def test_frame_round_trip(ws, oracle, kind, layout):
    for i, n in enumerate([0, 1, 513, 70001, 1 << 20]):
        x = {"u8": lambda: W.random_bytes(n, 30 + i, "skewed"),
             "u16": lambda: W.gradient_u16(n, 30 + i),
             "u32": lambda: W.quant_u32(n, 30 + i)}[kind]()
        p = 9 + i % 3
        fr = mb.frame_compress(to_dev(x), p, layout, ws=ws)
        h = to_host(fr)
        info = mb.frame_parse(h.tobytes())
        assert info.dtype == {"u8": 1, "u16": 2, "u32": 4}[kind]
        assert (info.layout, info.precision, info.n_elems) == (layout, p, n)
        body = h[64:]
        assert info.stream_bytes == body.size
        ref = oracle.ans_encode(x, p) if kind == "u8" else oracle.compress(x, p, layout)
        np.testing.assert_array_equal(body, ref)
        assert info.mapped_bytes == int(ref[8:12].view(np.uint32)[0])
        y = mb.frame_decompress(fr, ws=ws)
        np.testing.assert_array_equal(to_host(y, x.dtype), x)


def test_frame_overflow_records_no_stream(ws):
    import torch
    x = to_dev(W.random_bytes(100_000, 3, "uniform"))
    out = torch.zeros(4096, dtype=torch.uint8, device="cuda")
    size = torch.zeros(1, dtype=torch.int64, device="cuda")
    mb.load().mans_frame_compress(ws.h, 1, 0, x.data_ptr(), x.numel(), out.data_ptr(), out.numel(),
                                  size.data_ptr(), 10, mb._stream_handle(None))
    st, _ = ws.status()
    assert st == 8  # MANS_ERR_OUTPUT_OVERFLOW
    # the header records no stream, and a reader rejects the frame
    assert int(size.item()) == 64
    assert int(to_host(out[32:40]).view(np.uint64)[0]) == 0
    with pytest.raises(mb.MansError) as e:
        mb.frame_parse(to_host(out[:64]).tobytes())
    assert e.value.code == 7


def test_cli_frame_files(oracle, tmp_path):
    """mans_cli --compress / --decompress: separate runs through a frame file."""
    import subprocess

    from mans_b200 import build as B
    cli = B.build_cli()
    x = W.quant_u32(123_457, 4)
    fi, ff, fo = tmp_path / "in.u4", tmp_path / "x.mans", tmp_path / "out.u4"
    x.tofile(fi)
    r = subprocess.run([cli, "--compress", str(fi), str(ff), "--dtype", "u32"], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    f = np.fromfile(ff, np.uint8)
    info = mb.frame_parse(f.tobytes())
    assert info.n_elems == x.size and info.dtype == 4
    np.testing.assert_array_equal(f[64:], oracle.compress(x, 10))
    r = subprocess.run([cli, "--decompress", str(ff), str(fo)], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    np.testing.assert_array_equal(np.fromfile(fo, np.uint32), x)
