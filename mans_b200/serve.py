"""Serving loop over the batched codec (``mans_server_*`` in include/mans.h).

A scheduler thread inside the library admits compress / decompress requests
against an HBM budget and folds whatever is queued into the next batched
launch; several launches per direction are in flight at once on their own
streams. Results are byte-identical to the single-buffer calls.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import MansError, _check, dtype_code, load

COMPRESS, DECOMPRESS = 0, 1


class ServerConfig(C.Structure):
    _fields_ = [
        ("hbm_budget_bytes", C.c_uint64),
        ("max_batch_bytes", C.c_uint64),
        ("max_batch_items", C.c_uint32),
        ("lanes", C.c_uint32),
        ("merged_ratio_pct", C.c_uint32),
        ("plain", C.c_int),
    ]


class Request(C.Structure):
    _fields_ = [
        ("op", C.c_int),
        ("dtype", C.c_int),
        ("precision", C.c_int),
        ("pad", C.c_uint32),
        ("n_elems", C.c_uint64),
        ("d_in", C.c_void_p),
        ("in_bytes", C.c_uint64),
        ("d_out", C.c_void_p),
        ("out_capacity", C.c_uint64),
        ("tag", C.c_uint64),
        ("arrival_ns", C.c_uint64),
    ]


class Completion(C.Structure):
    _fields_ = [
        ("ticket", C.c_uint64),
        ("tag", C.c_uint64),
        ("status", C.c_int),
        ("batch_items", C.c_uint32),
        ("detail", C.c_uint64),
        ("d_out", C.c_void_p),
        ("out_bytes", C.c_uint64),
        ("queued_ns", C.c_uint64),
        ("latency_ns", C.c_uint64),
    ]


class Stats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("submitted", "completed", "launches", "in_flight", "queued",
                                          "arena_bytes", "arena_used", "arena_peak", "device_bytes")]


@dataclass
class Done:
    ticket: int
    tag: int
    status: int
    batch_items: int
    detail: int
    d_out: int
    out_bytes: int
    queued_ns: int
    latency_ns: int


def clock_ns() -> int:
    return int(load().mans_clock_ns())


class Server:
    """mans_server on the current device."""

    def __init__(self, hbm_budget_bytes: int, max_batch_bytes: int = 0, max_batch_items: int = 0,
                 lanes: int = 0, merged_ratio_pct: int = 0, plain: bool = False):
        cfg = ServerConfig(hbm_budget_bytes, max_batch_bytes, max_batch_items, lanes,
                           merged_ratio_pct, int(plain))
        h = C.c_void_p()
        _check(load().mans_server_create(C.byref(h), C.byref(cfg)), "mans_server_create")
        self.h = h
        self._buf = (Completion * 256)()

    def submit(self, op: int, dtype: int, n_elems: int, d_in: int | None, in_bytes: int = 0,
               precision: int = 10, d_out: int | None = None, out_capacity: int = 0, tag: int = 0,
               arrival_ns: int = 0) -> int:
        r = Request(op, dtype, precision, 0, n_elems, d_in, in_bytes, d_out, out_capacity, tag,
                    arrival_ns)
        t = C.c_uint64(0)
        _check(load().mans_server_submit(self.h, C.byref(r), C.byref(t)), "mans_server_submit")
        return int(t.value)

    def submit_tensor(self, op: int, x, precision: int = 10, tag: int = 0, out_dtype=None,
                      n_elems: int = 0, arrival_ns: int = 0) -> int:
        """compress: x is the values; decompress: x is the stream and out_dtype / n_elems describe the result."""
        if op == COMPRESS:
            return self.submit(op, dtype_code(x), x.numel(), x.data_ptr() if x.numel() else None,
                               0, precision, tag=tag, arrival_ns=arrival_ns)
        code = {"torch.uint8": 1, "torch.uint16": 2, "torch.uint32": 4}[str(out_dtype)]
        return self.submit(op, code, n_elems, x.data_ptr(), x.numel(), tag=tag, arrival_ns=arrival_ns)

    def poll(self, timeout_us: int = 0, max_n: int = 256) -> list[Done]:
        n = C.c_uint32(0)
        _check(load().mans_server_poll(self.h, self._buf, min(max_n, 256), C.byref(n), timeout_us),
               "mans_server_poll")
        out = []
        for i in range(n.value):
            c = self._buf[i]
            out.append(Done(int(c.ticket), int(c.tag), int(c.status), int(c.batch_items), int(c.detail),
                            int(c.d_out or 0), int(c.out_bytes), int(c.queued_ns), int(c.latency_ns)))
        return out

    def release(self, ticket: int) -> None:
        _check(load().mans_server_release(self.h, ticket), "mans_server_release")

    def stats(self) -> dict:
        st = Stats()
        _check(load().mans_server_get_stats(self.h, C.byref(st)), "mans_server_get_stats")
        return {k: int(getattr(st, k)) for k, _ in Stats._fields_}

    def close(self) -> None:
        if getattr(self, "h", None):
            load().mans_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def view_device(ptr: int, nbytes: int, device=None):
    """A uint8 tensor over device memory owned by the server (valid until released)."""
    import torch
    if nbytes == 0:
        return torch.empty(0, dtype=torch.uint8, device=device or "cuda")
    dev = torch.device(device or "cuda")
    # wrap the pointer without copying, through the CUDA array interface
    class _A:
        __cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                    "version": 3, "strides": None}
    return torch.as_tensor(_A(), device=dev)


__all__ = ["Server", "COMPRESS", "DECOMPRESS", "clock_ns", "view_device", "Done", "MansError"]
