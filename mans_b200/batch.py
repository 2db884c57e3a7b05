"""Batched MANS over many device buffers (``mans_batch_*`` in include/mans.h).

One call compresses (or decompresses) thousands of buffers of uneven size and
element type with one persistent launch per stage. Each buffer's stream is
byte-identical to ``mans_b200.compress`` of that buffer alone, and errors are
reported per buffer.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

from . import MansError, _check, _stream_handle, dtype_code, load, max_compressed_size

STAGES = ("map", "plan", "encode", "decode_plan", "decode", "unmap")


class BatchItem(C.Structure):
    """mans_batch_item (include/mans.h)."""
    _fields_ = [
        ("dtype", C.c_int),
        ("precision", C.c_int),
        ("n_elems", C.c_uint64),
        ("d_in", C.c_void_p),
        ("d_out", C.c_void_p),
        ("d_out_size", C.c_void_p),
        ("in_bytes", C.c_uint64),
        ("out_capacity", C.c_uint64),
    ]


def _ptr(t) -> int | None:
    return t.data_ptr() if t is not None and t.numel() else None


class Batch:
    """A batch workspace (mans_batch_create) on the current device."""

    def __init__(self, max_items: int, max_total_bytes: int, merged_ratio_pct: int = 0):
        h = C.c_void_p()
        _check(load().mans_batch_create(C.byref(h), max_items, max_total_bytes, merged_ratio_pct),
               "mans_batch_create")
        self.h = h
        self.max_items = max_items
        self.max_total_bytes = max_total_bytes

    @property
    def device_bytes(self) -> int:
        return int(load().mans_batch_device_bytes(self.h))

    # ---- descriptor builders ----
    @staticmethod
    def compress_items(xs: Sequence, outs: Sequence, sizes, precision: int | Sequence[int] = 10):
        """Descriptors for compressing xs[i] into outs[i]; sizes: int64 device tensor [len(xs)]."""
        arr = (BatchItem * len(xs))()
        base = sizes.data_ptr() if sizes is not None else 0
        for i, (x, o) in enumerate(zip(xs, outs)):
            p = precision if isinstance(precision, int) else precision[i]
            arr[i] = BatchItem(dtype_code(x), p, x.numel(), _ptr(x), _ptr(o),
                               base + 8 * i if base else None, 0, o.numel())
        return arr

    @staticmethod
    def decompress_items(streams: Sequence, stream_sizes: Sequence[int], outs: Sequence):
        arr = (BatchItem * len(streams))()
        for i, (s, sz, o) in enumerate(zip(streams, stream_sizes, outs)):
            arr[i] = BatchItem(dtype_code(o), 0, o.numel(), _ptr(s), _ptr(o), None, int(sz), 0)
        return arr

    # ---- calls ----
    def compress_async(self, items, stream=None) -> None:
        _check(load().mans_batch_compress(self.h, C.cast(items, C.c_void_p), len(items),
                                          _stream_handle(stream)), "mans_batch_compress")

    def decompress_async(self, items, stream=None) -> None:
        _check(load().mans_batch_decompress(self.h, C.cast(items, C.c_void_p), len(items),
                                            _stream_handle(stream)), "mans_batch_decompress")

    def status(self, count: int, stream=None) -> tuple[int, list[int], list[int]]:
        """(first error, per-buffer statuses, per-buffer details); synchronises the stream."""
        st = (C.c_uint32 * max(count, 1))()
        det = (C.c_uint64 * max(count, 1))()
        first = load().mans_batch_status(self.h, _stream_handle(stream), st, det, count)
        return int(first), [int(v) for v in st[:count]], [int(v) for v in det[:count]]

    def check(self, count: int, stream=None, what: str = "batch") -> None:
        first, st, det = self.status(count, stream)
        if first != 0:
            bad = [i for i, v in enumerate(st) if v]
            raise MansError(first, f"{what}: buffers {bad[:8]} (detail {det[bad[0]] if bad else 0})")

    def set_timing(self, enable: bool = True) -> None:
        _check(load().mans_batch_set_timing(self.h, int(enable)), "mans_batch_set_timing")

    def stage_times(self) -> dict:
        """Summed stage milliseconds and call counts recorded since the last read."""
        ms = (C.c_float * 6)()
        calls = (C.c_int * 2)()
        _check(load().mans_batch_stage_times(self.h, ms, calls), "mans_batch_stage_times")
        d = {name: ms[i] for i, name in enumerate(STAGES)}
        d["compress_calls"], d["decompress_calls"] = calls[0], calls[1]
        return d

    def schedule(self) -> tuple[list[int], list[int]]:
        cur = (C.c_int * 6)()
        mx = (C.c_int * 6)()
        _check(load().mans_batch_get_schedule(self.h, cur, mx), "mans_batch_get_schedule")
        return list(cur), list(mx)

    def set_schedule(self, ctas_per_sm: Sequence[int]) -> None:
        arr = (C.c_int * 6)(*ctas_per_sm)
        _check(load().mans_batch_set_schedule(self.h, arr), "mans_batch_set_schedule")

    def schedule_ex(self) -> tuple[dict, dict]:
        """The full schedule and its limits, each as {"ctas_per_sm": [...],
        "warps_per_cta": [...], "prefetch_grids": [...]} over the six stages."""
        from . import BatchSchedule
        cur, lim = BatchSchedule(), BatchSchedule()
        _check(load().mans_batch_get_schedule_ex(self.h, C.byref(cur), C.byref(lim)),
               "mans_batch_get_schedule_ex")

        def as_dict(x):
            return {f: list(getattr(x, f)) for f, _ in BatchSchedule._fields_}
        return as_dict(cur), as_dict(lim)

    def set_schedule_ex(self, sch: dict) -> None:
        from . import BatchSchedule
        x = BatchSchedule()
        for f, _ in BatchSchedule._fields_:
            getattr(x, f)[:] = list(sch[f])
        _check(load().mans_batch_set_schedule_ex(self.h, C.byref(x)), "mans_batch_set_schedule_ex")

    def autotune(self, items, stream=None) -> float:
        ms = C.c_float(0)
        _check(load().mans_batch_autotune(self.h, C.cast(items, C.c_void_p), len(items),
                                          _stream_handle(stream), C.byref(ms)), "mans_batch_autotune")
        return float(ms.value)

    # ---- convenience ----
    def compress(self, xs: Sequence, precision: int | Sequence[int] = 10, stream=None):
        """Compress every tensor of xs; returns a list of uint8 tensors (synchronises)."""
        import torch
        dev = xs[0].device
        outs = [torch.empty(max_compressed_size(dtype_code(x), x.numel()), dtype=torch.uint8,
                            device=dev) for x in xs]
        sizes = torch.zeros(len(xs), dtype=torch.int64, device=dev)
        items = self.compress_items(xs, outs, sizes, precision)
        self.compress_async(items, stream)
        self.check(len(xs), stream, "mans_batch_compress")
        return [o[:int(n)].clone() for o, n in zip(outs, sizes.tolist())]

    def decompress(self, streams: Sequence, shapes: Sequence[tuple[int, object]], stream=None):
        """Decompress streams[i] into a new tensor of shapes[i] = (n_elems, dtype) (synchronises)."""
        import torch
        dev = streams[0].device
        outs = [torch.empty(n, dtype=dt, device=dev) for n, dt in shapes]
        items = self.decompress_items(streams, [s.numel() for s in streams], outs)
        self.decompress_async(items, stream)
        self.check(len(streams), stream, "mans_batch_decompress")
        return outs

    def close(self) -> None:
        if getattr(self, "h", None):
            load().mans_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
