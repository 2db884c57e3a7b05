"""CPU tests of the oracle: pinned against the reference's own code and its
recorded outputs, plus the algorithmic properties the GPU path relies on."""
import json
import os

import numpy as np
import pytest

from mans_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
MANIFEST = os.path.join(GOLDEN, "manifest.json")


def _manifest():
    if not os.path.exists(MANIFEST):
        return []
    with open(MANIFEST) as f:
        return json.load(f)


def _gen(spec, O):
    from tests.golden.make_golden import gen
    return gen(spec)


def _sha(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8).tobytes()).hexdigest()


# ---------------------------------------------------------------- golden pins
@pytest.mark.parametrize("case", [c for c in _manifest() if c["kind"] == "adm_u16_cpu"],
                         ids=lambda c: c["name"])
def test_golden_cpu_mapping(case, oracle):
    """Oracle uint16 mapping == reference CPU mapping (mappingcpuV2.cpp) output.

    Cases outside the reference's defined domain (lanes longer than its
    32-byte lane buffer, where it fails its own round trip) only require the
    oracle to round-trip."""
    x = _gen(case["input"], oracle)
    m = oracle.adm_u16_map(x)
    if not case.get("ref_defined", True):
        assert not case["ref_roundtrip"]
        np.testing.assert_array_equal(oracle.adm_u16_unmap(m, x.size), x)
        return
    assert case["ref_roundtrip"]
    assert m.size == case["ref_size"]
    assert _sha(m) == case["ref_sha256"]
    if "ref_file" in case:
        ref = np.fromfile(os.path.join(GOLDEN, case["ref_file"]), np.uint8)
        np.testing.assert_array_equal(m, ref)


@pytest.mark.parametrize("case", [c for c in _manifest() if c["kind"] == "adm_u16_gpu"],
                         ids=lambda c: c["name"])
def test_golden_gpu_mapping_u16(case, oracle):
    """Oracle uint16 mapping == reference GPU mapping (mappingV15) output file."""
    assert case.get("ref_log_pass", False)
    x = _gen(case["input"], oracle)
    m = oracle.adm_u16_map(x)
    assert m.size == case["ref_size"]
    assert _sha(m) == case["ref_sha256"]


@pytest.mark.parametrize("case", [c for c in _manifest() if c["kind"] == "adm_u32_gpu"],
                         ids=lambda c: c["name"])
def test_golden_gpu_mapping_u32(case, oracle):
    """Records section of the oracle's uint32 mapping == reference V9 output file."""
    assert case.get("ref_log_pass", False)
    x = _gen(case["input"], oracle)
    m = oracle.adm_u32_map(x)
    g = -(-x.size // 512)
    recs = m[40 * g:]
    assert recs.size == case["ref_size"]
    assert _sha(recs) == case["ref_sha256"]


@pytest.mark.parametrize("case", [c for c in _manifest() if c["kind"] == "ans" and "skipped" not in c],
                         ids=lambda c: c["name"])
def test_golden_ans(case, oracle):
    """Oracle rANS stream == reference GPU ansEncode stream (uninitialised bytes masked)."""
    assert case.get("ref_roundtrip", False)
    x = _gen(case["input"], oracle)
    assert _sha(x) == case["input_sha256"]
    s = oracle.ans_encode(x, case["prob_bits"])
    assert s.size == case["ref_size"]
    sm = oracle.ans_mask(s)
    np.testing.assert_array_equal(sm, s)  # the oracle writes zeros where the reference is undefined
    assert _sha(sm) == case["ref_sha256"]
    if "ref_file" in case:
        ref = np.fromfile(os.path.join(GOLDEN, case["ref_file"]), np.uint8)
        np.testing.assert_array_equal(sm, ref)
    np.testing.assert_array_equal(oracle.ans_decode(s), x)


def _check_layout_case(case, oracle, layout):
    x = _gen(case["input"], oracle)
    m = oracle.adm_u16_map(x, layout)
    assert m.size == case["ref_size"]
    assert _sha(m) == case["ref_sha256"]
    if "ref_file" in case:
        ref = np.fromfile(os.path.join(GOLDEN, case["ref_file"]), np.uint8)
        np.testing.assert_array_equal(m, ref)
    np.testing.assert_array_equal(oracle.adm_u16_unmap(m, x.size, layout), x)


@pytest.mark.parametrize("case", [c for c in _manifest() if c["kind"] == "adm_u16_cpu_native"],
                         ids=lambda c: c["name"])
def test_golden_cpu_native_layout(case, oracle):
    """Oracle CPU-V2 layout (g + 1 prefix words) == the reference CPU mapping's own merged file."""
    assert case["ref_roundtrip"]
    _check_layout_case(case, oracle, oracle.LAYOUT_CPUV2)


@pytest.mark.parametrize("case", [c for c in _manifest() if c["kind"] == "adm_u16_v12_gpu"],
                         ids=lambda c: c["name"])
def test_golden_v12_layout(case, oracle):
    """Oracle V12 layout (u16 group lengths) == the reference mappingV12 output file."""
    assert case.get("ref_log_pass", False)
    _check_layout_case(case, oracle, oracle.LAYOUT_V12)


def test_layouts_round_trip_and_differ_only_in_header(oracle):
    """All three uint16 layouts round-trip; they share codes and bits except
    that V12 fills lanes past n with 0xFF."""
    for n in [16, 512, 1040, 5000, 70001]:
        x = W.gradient_u16(n, 11)
        g = -(-n // 512)
        ms = {lay: oracle.adm_u16_map(x, lay) for lay in (0, 1, 2)}
        for lay, m in ms.items():
            np.testing.assert_array_equal(oracle.adm_u16_unmap(m, n, lay), x)
        body15 = ms[0][6 * g:]
        np.testing.assert_array_equal(ms[2][6 * g + 4:], body15)
        np.testing.assert_array_equal(ms[1][4 * g:4 * g + n], body15[:n])  # codes
        if n % 16 == 0 and n % 512 == 0:
            np.testing.assert_array_equal(ms[1][4 * g:], body15)


def test_golden_manifest_present():
    m = _manifest()
    kinds = {c["kind"] for c in m}
    assert {"adm_u16_cpu", "adm_u16_cpu_native", "adm_u16_gpu", "adm_u16_v12_gpu", "adm_u32_gpu",
            "ans"} <= kinds, kinds


# ---------------------------------------------------------------- live reference CPU mapping
def test_live_reference_cpu_mapping(oracle):
    """Oracle == reference CPU mapping run here (one OpenMP thread), ragged sizes."""
    if oracle.ref_lib() is None:
        pytest.skip("reference CPU mapping not built (oracle/_ref)")
    rng = np.random.default_rng(5)
    for n in [1, 2, 15, 16, 17, 255, 511, 512, 513, 777, 1023, 1024, 1025, 9999]:
        x = np.clip(np.round(30000 + rng.laplace(0, 500, n)), 0, 65535).astype(np.uint16)
        r = oracle.RefAdmCpu(x)
        r.compress()
        np.testing.assert_array_equal(oracle.adm_u16_map(x), r.merged(True))
        r.decompress()
        np.testing.assert_array_equal(r.recovered(), x)
        r.close()


# ---------------------------------------------------------------- oracle properties
@pytest.mark.parametrize("n", [0, 1, 17, 512, 513, 4096, 70001])
def test_oracle_u16_roundtrip(n, oracle):
    x = W.laplace_u16(n, 11, b=2000.0)
    m = oracle.adm_u16_map(x)
    np.testing.assert_array_equal(oracle.adm_u16_unmap(m, n), x)
    s = oracle.compress(x, 10)
    np.testing.assert_array_equal(oracle.decompress(s, n, np.uint16), x)


def test_oracle_u16_extreme_values(oracle):
    """Alternating 0 / 65535: k up to 261 per element, lanes far beyond 256 bits."""
    x = np.tile(np.array([0, 65535], np.uint16), 2048)
    m = oracle.adm_u16_map(x)
    np.testing.assert_array_equal(oracle.adm_u16_unmap(m, x.size), x)


def test_oracle_u16_rejects_malformed_lane_streams(oracle):
    """The reference's restore (mappingcpuV2.cpp:161-197, restated by the
    oracle) rejects a lane stream that does not start with a 1 and one that
    holds fewer elements than the lane: the two faults the GPU unmap must
    report as corrupt (tests/test_gpu_layouts.py plants the same ones)."""
    n = 512 * 16
    g = n // 512
    for gen, seed in ((W.laplace_u16, 11), (W.volume_u16, 12)):
        x = gen(n, seed)
        m0 = oracle.adm_u16_map(x)
        pre = m0[:4 * g].copy().view(np.int32)
        bits = 6 * g + n
        lens = np.diff(np.append(pre, (m0.size - bits) // 32))
        for grp in (0, int(np.argmax(lens))):
            L = int(lens[grp])
            base = bits + 32 * int(pre[grp])
            m = m0.copy()
            m[base + 5 * L] &= 0x7F  # lane 5: no leading 1
            with pytest.raises(ValueError, match="-4"):
                oracle.adm_u16_unmap(m, n)
            m = m0.copy()
            m[base + 7 * L] = 0x80  # lane 7: one element, then zeros to its end
            m[base + 7 * L + 1:base + 8 * L] = 0
            with pytest.raises(ValueError, match="-5"):
                oracle.adm_u16_unmap(m, n)
        np.testing.assert_array_equal(oracle.adm_u16_unmap(m0, n), x)


@pytest.mark.parametrize("n", [0, 1, 16, 513, 4096, 70001])
def test_oracle_u32_roundtrip(n, oracle):
    for x in (W.detector_u32(n, 12), W.quant_u32(n, 13),
              np.random.default_rng(14).integers(0, 2**32, n, dtype=np.uint32)):
        m = oracle.adm_u32_map(x)
        np.testing.assert_array_equal(oracle.adm_u32_unmap(m, n), x)
        s = oracle.compress(x, 11)
        np.testing.assert_array_equal(oracle.decompress(s, n, np.uint32), x)


@pytest.mark.parametrize("p", [9, 10, 11])
def test_normalize_sums_and_presence(p, oracle):
    rng = np.random.default_rng(p)
    for _ in range(50):
        h = (rng.geometric(0.02, 256) * (rng.random(256) < 0.7)).astype(np.uint32)
        tot = int(h.sum())
        if tot == 0:
            continue
        pdf, cdf = oracle.normalize(h, tot, p)
        assert int(pdf.sum()) == 1 << p
        assert np.all(pdf[h > 0] >= 1)
        np.testing.assert_array_equal(cdf, np.concatenate([[0], np.cumsum(pdf)[:-1]]))


def test_normalize_adds_to_low_symbol_ids(oracle):
    """The under-allocation fix-up adds 1 by symbol id, absent symbols included
    (GpuANSStatistics.h:271-283)."""
    h = np.zeros(256, np.uint32)
    h[200] = 3
    h[201] = 3
    h[202] = 3  # each quantises to floor(1024/3) = 341 -> sum 1023, diff 1
    pdf, _ = oracle.normalize(h, 9, 10)
    assert pdf[0] == 1 and pdf[200] == 341 and pdf[201] == 341 and pdf[202] == 341
    assert int(pdf.sum()) == 1024


def test_normalize_float32_rounding(oracle):
    """The first pass is IEEE float32 division and multiply, truncated."""
    h = np.zeros(256, np.uint32)
    h[0] = 16777217  # not representable in float32
    h[1] = 3
    tot = int(h.sum())
    pdf, _ = oracle.normalize(h, tot, 11)
    q = np.float32(2048) * (np.float32(h[0]) / np.float32(tot))
    q1 = np.float32(2048) * (np.float32(h[1]) / np.float32(tot))
    assert int(pdf.sum()) == 2048
    assert pdf[1] == max(1, int(q1))
    assert pdf[0] == 2048 - pdf[1] or pdf[0] == int(q)


def test_ans_roundtrip_sizes(oracle):
    rng = np.random.default_rng(7)
    for n in [0, 1, 31, 32, 33, 4095, 4096, 4097, 12345]:
        for kind in ["uniform", "skewed", "single", "two", "sparse"]:
            x = W.random_bytes(n, int(rng.integers(1 << 30)), kind)
            for p in (9, 10, 11):
                s = oracle.ans_encode(x, p)
                np.testing.assert_array_equal(oracle.ans_decode(s), x)


def test_ans_decode_rejects_bad_header(oracle):
    x = W.random_bytes(5000, 1)
    s = oracle.ans_encode(x, 10)
    bad = s.copy()
    bad[2] ^= 0xFF  # magic
    with pytest.raises(ValueError):
        oracle.ans_decode(bad)
    with pytest.raises(ValueError):
        oracle.ans_decode(s[:600])  # truncated


def test_ans_worst_case_bound(oracle):
    """The true bound holds where the reference's 1.25x estimate does not."""
    # frequent symbol everywhere except one block of rare symbols
    x = np.zeros(64 * 4096, np.uint8)
    x[:4096] = np.arange(4096) % 255 + 1
    s, bw = oracle.ans_encode(x, 11, with_block_words=True)
    assert int(bw[0]) * 2 > 5120  # the reference's per-block slot would overflow
    assert s.size <= oracle.max_compressed_size(x.size)
    np.testing.assert_array_equal(oracle.ans_decode(s), x)


def test_div126_magic():
    """floor(a/126) == (a * 512 * 66577) >> 32 for every a the mappers use."""
    a = np.arange(0, 65661 + 1009, dtype=np.uint64)
    np.testing.assert_array_equal((a * 512 * 66577) >> 32, a // 126)


@pytest.mark.parametrize("layout", [0, 1, 2])
@pytest.mark.parametrize("n", [0, 1, 511, 512, 513, 4097, 70_001, 1 << 18])
def test_parallel_oracle_equals_serial_u16(n, layout, oracle):
    """The group- and block-parallel oracle (the judge of the full-size GPU
    streams) gives exactly the serial oracle's bytes, which the golden
    vectors pin to the reference."""
    from mans_b200 import workloads as W
    rng = np.random.default_rng(n + layout)
    for x in (W.volume_u16(n, 4), rng.integers(0, 65536, n, dtype=np.uint16)):
        np.testing.assert_array_equal(oracle.compress_par(x, 10, layout, threads=4),
                                      oracle.compress(x, 10, layout))


@pytest.mark.parametrize("n", [0, 1, 511, 513, 70_001, 1 << 18])
def test_parallel_oracle_equals_serial_u32(n, oracle):
    from mans_b200 import workloads as W
    for x in (W.detector_u32(n, 2), W.quant_u32(n, 3)):
        np.testing.assert_array_equal(oracle.compress_par(x, 11, threads=4), oracle.compress(x, 11))
