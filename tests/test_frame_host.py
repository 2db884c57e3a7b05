"""Host-side tests of the self-describing frame header (mans_frame_parse, no GPU)."""
import struct

import pytest

import mans_b200 as mb


def header(magic=0x534E414D, ver=1, dtype=2, layout=0, p=10, hb=64, n=1000, mapped=1200,
           stream=700):
    h = struct.pack("<IHBBBBHI", magic, ver, dtype, layout, p, 0, hb, 0)
    h += struct.pack("<QQQ", n, mapped, stream) + bytes(24)
    assert len(h) == 64
    return h


def test_frame_parse_fields():
    f = mb.frame_parse(header() + bytes(700))
    assert (f.dtype, f.layout, f.precision, f.header_bytes) == (2, 0, 10, 64)
    assert (f.n_elems, f.mapped_bytes, f.stream_bytes) == (1000, 1200, 700)


@pytest.mark.parametrize("kw", [dict(magic=0x12345678), dict(ver=2), dict(hb=32), dict(dtype=3),
                                dict(layout=3), dict(dtype=4, layout=1), dict(p=8), dict(p=12),
                                dict(dtype=1, n=10, mapped=11), dict(stream=543)])
def test_frame_parse_rejects(kw):
    with pytest.raises(mb.MansError) as e:
        mb.frame_parse(header(**kw) + bytes(700))
    assert e.value.code == 7


def test_frame_parse_checks_the_available_size():
    with pytest.raises(mb.MansError):
        mb.frame_parse(header(stream=701) + bytes(700))
    mb.frame_parse(header(stream=701))  # header alone: size unknown, accepted


@pytest.mark.parametrize("stream", [2 ** 64 - 1, 2 ** 64 - 63, 2 ** 64 - 64, 2 ** 63])
def test_frame_parse_rejects_wrapping_stream_sizes(stream):
    """A stream size near 2^64 must not wrap the available-size check, and a
    stream larger than any stream of its mapped bytes is rejected even when
    the available size is unknown."""
    for avail in (64 + 700, 2 ** 64 - 2, None):
        with pytest.raises(mb.MansError) as e:
            blob = header(stream=stream) + bytes(700)
            mb.frame_parse(blob) if avail is None else mb.frame_parse(blob, avail)
        assert e.value.code == 7


def test_frame_parse_bounds_sizes_by_the_element_count():
    # mapped bytes beyond the worst case of 1000 uint16 values
    with pytest.raises(mb.MansError):
        mb.frame_parse(header(mapped=mb.max_mapped_size(mb.MANS_U16, 1000) + 1))
    # a stream beyond the worst case of its mapped bytes
    with pytest.raises(mb.MansError):
        mb.frame_parse(header(mapped=1200, stream=mb.stream_bound(1200) + 16))
    f = mb.frame_parse(header(mapped=1200, stream=mb.stream_bound(1200)))
    assert f.stream_bytes == mb.stream_bound(1200)
