"""GPU tests of the on-disk compatibility layouts (mans_compress_ex,
mans_adm_map / mans_adm_unmap): every mapped byte and stream byte equals the
oracle's, which is pinned against the reference's V12 and CPU mappers."""
import numpy as np
import pytest

import mans_b200 as mb
from mans_b200 import workloads as W
from tests.helpers import to_dev, to_host

pytestmark = pytest.mark.gpu

SIZES = [0, 1, 16, 511, 512, 513, 1040, 4097, 70001, 1 << 20]


@pytest.fixture(scope="module")
def ws():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    w = mb.Workspace(64 << 20)
    yield w
    w.close()


@pytest.mark.parametrize("layout", [mb.LAYOUT_NATIVE, mb.LAYOUT_V12, mb.LAYOUT_CPUV2])
def test_u16_layouts_match_oracle(ws, oracle, layout):
    import torch
    for i, n in enumerate(SIZES):
        x = (W.gradient_u16, W.laplace_u16, W.volume_u16)[i % 3](n, 600 + i)
        dx = to_dev(x)
        m = to_host(mb.adm_map(dx, layout, ws=ws))
        ref_m = oracle.adm_u16_map(x, layout)
        np.testing.assert_array_equal(m, ref_m, err_msg=f"map n={n} layout={layout}")
        back = mb.adm_unmap(to_dev(ref_m), n, torch.uint16, layout, ws=ws)
        np.testing.assert_array_equal(to_host(back, np.uint16), x, err_msg=f"unmap n={n}")
        p = 9 + i % 3
        s = to_host(mb.compress(dx, p, ws=ws, layout=layout))
        np.testing.assert_array_equal(s, oracle.compress(x, p, layout), err_msg=f"stream n={n}")
        y = mb.decompress(to_dev(s), n, torch.uint16, ws=ws, layout=layout)
        np.testing.assert_array_equal(to_host(y, np.uint16), x, err_msg=f"decompress n={n}")


def test_u32_native_mapping_matches_oracle(ws, oracle):
    import torch
    for i, n in enumerate([1, 511, 513, 70001, 1 << 18]):
        x = (W.quant_u32, W.detector_u32)[i % 2](n, 700 + i)
        m = to_host(mb.adm_map(to_dev(x), ws=ws))
        np.testing.assert_array_equal(m, oracle.adm_u32_map(x))
        back = mb.adm_unmap(to_dev(m), n, torch.uint32, ws=ws)
        np.testing.assert_array_equal(to_host(back, np.uint32), x)


@pytest.mark.parametrize("dtype", ["u16", "u32"])
def test_map_only_calls_in_a_row_with_new_data(ws, oracle, dtype):
    """Consecutive map-only calls (and a compress after them) on one workspace
    with different data of the same size: the look-back flags of one call
    must never be read as valid by the next, whatever the data."""
    n = 300_000
    gens = (W.gradient_u16, W.volume_u16, W.laplace_u16) if dtype == "u16" else \
        (W.quant_u32, W.detector_u32, W.quant_u32)
    for i, gen in enumerate(gens):
        x = gen(n, 900 + i)
        dx = to_dev(x)
        ref = oracle.adm_u16_map(x) if dtype == "u16" else oracle.adm_u32_map(x)
        np.testing.assert_array_equal(to_host(mb.adm_map(dx, ws=ws)), ref, err_msg=f"call {i}")
    y = gens[0](n, 990)
    np.testing.assert_array_equal(to_host(mb.compress(to_dev(y), 10, ws=ws)), oracle.compress(y, 10))


def test_layout_header_corruption_is_reported(ws, oracle):
    import torch
    n = 70001
    x = W.gradient_u16(n, 5)
    g = -(-n // 512)
    m = oracle.adm_u16_map(x, mb.LAYOUT_CPUV2)
    m[4 * g] ^= 1  # the final prefix word no longer matches the bit section
    with pytest.raises(mb.MansError) as e:
        mb.adm_unmap(to_dev(m), n, torch.uint16, mb.LAYOUT_CPUV2, ws=ws)
    assert e.value.code == 10
    m = oracle.adm_u16_map(x, mb.LAYOUT_V12)
    m[0] ^= 1  # group lengths no longer add up to the bit section
    with pytest.raises(mb.MansError) as e:
        mb.adm_unmap(to_dev(m), n, torch.uint16, mb.LAYOUT_V12, ws=ws)
    assert e.value.code == 10


def test_u16_malformed_lane_streams_are_reported(ws, oracle):
    """Lane bit streams that cannot be decoded are reported as corrupt (status
    10): a lane whose stream does not start with a 1, and a lane whose
    elements run past its bytes. The faults are planted in the oracle's
    mapped buffer on the CPU, in a group whose lanes take at most 4 bytes
    (decoded on 32-bit words) and in one whose lanes take 5 to 8 (64 bits);
    the untouched buffers decode to the input."""
    import torch
    n = 512 * 16
    g = n // 512
    for gen, seed, lo, hi in ((W.laplace_u16, 11, 1, 4), (W.volume_u16, 12, 5, 8)):
        x = gen(n, seed)
        m0 = oracle.adm_u16_map(x)
        pre = m0[:4 * g].copy().view(np.int32)  # exclusive prefix, 32-byte units
        bits = 6 * g + n
        tot = (m0.size - bits) // 32
        lens = np.diff(np.append(pre, tot))
        grps = np.nonzero((lens >= lo) & (lens <= hi))[0]
        assert grps.size, (gen.__name__, lens)
        grp = int(grps[0])
        L = int(lens[grp])
        base = bits + 32 * int(pre[grp])
        back = mb.adm_unmap(to_dev(m0), n, torch.uint16, ws=ws)
        np.testing.assert_array_equal(to_host(back, np.uint16), x)
        m = m0.copy()
        m[base + 5 * L] &= 0x7F  # lane 5 no longer starts with a 1
        with pytest.raises(mb.MansError) as e:
            mb.adm_unmap(to_dev(m), n, torch.uint16, ws=ws)
        assert e.value.code == 10
        m = m0.copy()
        m[base + 7 * L] = 0x80  # lane 7: one leading 1, then zeros to its end
        m[base + 7 * L + 1:base + 8 * L] = 0
        with pytest.raises(mb.MansError) as e:
            mb.adm_unmap(to_dev(m), n, torch.uint16, ws=ws)
        assert e.value.code == 10


def _u32_lane_record(m, n, grp, lane):
    """Offset and length of one lane's record in a uint32 mapped buffer:
    [i32 group offset x g][u32 center x g][u8 length / 8 x 32 g][records]."""
    g = -(-n // 512)
    goff = int(m[4 * grp:4 * grp + 4].view(np.uint32)[0])
    lens = 8 * m[8 * g + 32 * grp:8 * g + 32 * grp + 32].astype(np.int64)
    return 40 * g + goff + int(lens[:lane].sum()), int(lens[lane])


def test_u32_malformed_records_are_reported(ws, oracle):
    """uint32 records that cannot be parsed are reported as corrupt (status
    10): a lane record of zero bytes only, and a padding byte (255) where a
    code byte belongs. Planted in the oracle's mapped buffer on the CPU; the
    oracle rejects both too."""
    import torch
    n = 512 * 8
    x = W.quant_u32(n, 21)
    m0 = oracle.adm_u32_map(x)
    np.testing.assert_array_equal(to_host(mb.adm_unmap(to_dev(m0), n, torch.uint32, ws=ws),
                                          np.uint32), x)
    start, ln = _u32_lane_record(m0, n, 3, 9)
    m = m0.copy()
    m[start:start + ln] = 0
    m2 = m0.copy()
    first = start + int(np.nonzero(m0[start:start + ln])[0][0])  # the lane's first nonzero byte
    m2[first] = 255
    for bad in (m, m2):
        with pytest.raises(ValueError):
            oracle.adm_u32_unmap(bad, n)
        with pytest.raises(mb.MansError) as e:
            mb.adm_unmap(to_dev(bad), n, torch.uint32, ws=ws)
        assert e.value.code == 10


def test_layout_argument_checks(ws):
    import torch
    x = torch.zeros(1024, dtype=torch.uint32, device="cuda")
    with pytest.raises(mb.MansError) as e:
        mb.compress(x, 10, ws=ws, layout=mb.LAYOUT_V12)
    assert e.value.code == 1
    with pytest.raises(mb.MansError) as e:
        mb.adm_map(torch.zeros(16, dtype=torch.uint8, device="cuda"), ws=ws)
    assert e.value.code == 1


@pytest.mark.parametrize("dtype,layout", [("u8", "native"), ("u16", "native"), ("u16", "v12"),
                                          ("u16", "cpuv2"), ("u32", "native")])
def test_cli_round_trip(oracle, tmp_path, dtype, layout):
    """mans_cli <input> <temp> <output>: the temp file is the oracle's stream and
    the output equals the input, as with the reference's example driver."""
    import subprocess

    from mans_b200 import build as B
    cli = B.build_cli()
    n = 300_001
    x = {"u8": lambda: W.random_bytes(n, 9, "skewed"), "u16": lambda: W.laplace_u16(n, 9),
         "u32": lambda: W.detector_u32(n, 9)}[dtype]()
    fi, ft, fo = tmp_path / "in.img", tmp_path / "t.ans", tmp_path / "out.img"
    x.tofile(fi)
    r = subprocess.run([cli, str(fi), str(ft), str(fo), "--dtype", dtype, "--precision", "11",
                        "--layout", layout], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Compression completed successfully." in r.stdout
    s = np.fromfile(ft, np.uint8)
    lay = {"native": 0, "v12": 1, "cpuv2": 2}[layout]
    ref = oracle.ans_encode(x, 11) if dtype == "u8" else oracle.compress(x, 11, lay)
    np.testing.assert_array_equal(s, ref)
    np.testing.assert_array_equal(np.fromfile(fo, x.dtype), x)
