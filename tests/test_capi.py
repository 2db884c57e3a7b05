"""CPU tests of the C ABI: the library loads, exports every function that
include/*.h declares, and rejects bad arguments on the host without touching
a GPU."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

import mans_b200 as mb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(mans_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_loads_and_exports_declared_symbols():
    lib = mb.load()
    decl = declared_functions()
    assert len(decl) >= 15
    for name in decl:
        assert hasattr(lib, name), name
        assert name in mb.SIGNATURES, name
    assert mb.version().startswith("mans_b200")


def test_host_side_argument_checks():
    lib = mb.load()
    # precision outside {9,10,11}: rejected before any CUDA call
    assert lib.mans_ans_encode(8, 16, 10, 32, 48, None) == 2
    assert lib.mans_ans_encode(12, 16, 10, 32, 48, None) == 2
    assert lib.mans_ans_decode(13, 16, 32, None) == 2
    # unaligned device pointers
    assert lib.mans_ans_encode(10, 17, 10, 32, 48, None) == 3
    assert lib.mans_ans_decode(10, 16, 33, None) == 3
    # null arguments
    assert lib.mans_ans_encode(10, 16, 10, None, 48, None) == 1
    assert lib.mans_compress(None, 2, 16, 10, 32, 100, 48, 10, None) == 1
    assert lib.mans_decompress(None, 2, 16, 100, 32, 10, None) == 1
    assert lib.mans_workspace_destroy(None) == 1


@pytest.mark.parametrize("n", [0, 1, 4096, 4097, 10 ** 7])
def test_max_compressed_size_is_a_bound(n, oracle):
    assert mb.getMaxCompressedSize(n) >= oracle.max_compressed_size(n)
    assert mb.max_compressed_size(mb.MANS_U8, n) >= oracle.max_compressed_size(n)
    for dt in (mb.MANS_U16, mb.MANS_U32):
        m = min(mb.max_mapped_size(dt, n), 0xFFFFFFF0)
        assert mb.max_compressed_size(dt, n) == mb.stream_bound(m) >= oracle.max_compressed_size(m)


def _wide_u16_patterns(n):
    """uint16 inputs that map to the most bytes: alternating extremes, one
    lane of 65535 per group over zeros (and the reverse), uniform noise."""
    rng = np.random.default_rng(5)
    one_lane = np.zeros(n, np.uint16)
    one_lane.reshape(-1, 512)[:, :16] = 65535
    return [np.tile(np.array([0, 65535], np.uint16), n // 2), one_lane, 65535 - one_lane,
            rng.integers(0, 65536, n, dtype=np.uint16)]


@pytest.mark.parametrize("n", [512, 8192, 65_536])
def test_max_mapped_size_covers_the_widest_uint16_data(n, oracle):
    """The worst-case bounds hold for the uint16 inputs that map widest (up to
    about 65 mapped bytes per element) in every layout, and for uint32 data
    of only escapes and of only 8-byte elements."""
    for x in _wide_u16_patterns(n):
        for layout in (0, 1, 2):
            m = oracle.adm_u16_map(x, layout)
            assert m.size <= mb.max_mapped_size(mb.MANS_U16, n)
        assert oracle.compress(x, 9).size <= mb.max_compressed_size(mb.MANS_U16, n)
    for x in (np.tile(np.array([0, 1 << 31], np.uint32), n // 2),
              np.tile(np.array([0, 8 * 126 * 2], np.uint32), n // 2)):
        assert oracle.adm_u32_map(x).size <= mb.max_mapped_size(mb.MANS_U32, n)
        assert oracle.compress(x, 9).size <= mb.max_compressed_size(mb.MANS_U32, n)


def test_division_table_is_exact():
    """x / pdf through the encoder's reciprocal table equals exact division for
    every pdf and p, on all states the encoder can hold (x < pdf << (31-p))."""
    lib = mb.load()
    out = (C.c_uint32 * 2)()
    rng = np.random.default_rng(0)
    for p in (9, 10, 11):
        M = 1 << p
        for pdf in range(1, M + 1):
            cdf = int(rng.integers(0, M - pdf + 1))
            lib.mans_debug_enc_entry(pdf, cdf, p, out)
            rcp, y = int(out[0]), int(out[1])
            sh, bias, cmpl = y & 0x1F, (y >> 5) & 0x1FFF, y >> 20
            assert cmpl == M - pdf
            hi = pdf << (31 - p)
            x = np.concatenate([rng.integers(1, hi, 2000, dtype=np.uint64),
                                np.array([1, 2, pdf - 1, pdf, pdf + 1, hi - 1], np.uint64)])
            x = x[(x >= 1) & (x < hi)]
            q = ((x * np.uint64(rcp)) >> np.uint64(32)) >> np.uint64(sh)
            got = x + np.uint64(bias) + q * np.uint64(cmpl)
            want = (x // np.uint64(pdf)) * np.uint64(M) + x % np.uint64(pdf) + np.uint64(cdf)
            np.testing.assert_array_equal(got, want, err_msg=f"p={p} pdf={pdf}")


def test_cli_usage_without_gpu():
    """The command-line driver (argv of the reference's examples/compress.cu) builds and prints usage."""
    import subprocess

    from mans_b200 import build as B
    cli = B.build_cli()
    r = subprocess.run([cli, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0
    assert "<input.img> <temp.ans> <output.img>" in r.stderr
