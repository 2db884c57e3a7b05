"""mans_b200 -- B200-native MANS codec (ADM byte mapping + byte rANS).

The product is ``libmans_b200.so`` (C ABI declared in ``include/mans.h``,
kernels in ``csrc/``). This module loads it with ctypes and offers a thin
host layer over device tensors. Names follow the reference interface
(``ansEncode``/``ansDecode``/``getMaxCompressedSize`` of include/ans) plus the
MANS entry points that add the ADM mapping for uint16/uint32 arrays.

There is no CPU fallback: if the library is missing or no GPU is present the
calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmans_b200.so")

# mans_status (include/mans.h)
STATUS = {
    0: "MANS_OK",
    1: "MANS_ERR_INVALID_ARG",
    2: "MANS_ERR_UNSUPPORTED_PRECISION",
    3: "MANS_ERR_ALIGNMENT",
    4: "MANS_ERR_TOO_LARGE",
    5: "MANS_ERR_CUDA",
    6: "MANS_ERR_OUT_OF_MEMORY",
    7: "MANS_ERR_BAD_STREAM",
    8: "MANS_ERR_OUTPUT_OVERFLOW",
    9: "MANS_ERR_WORKSPACE_OVERFLOW",
    10: "MANS_ERR_CORRUPT",
    11: "MANS_ERR_TIMEOUT",
}
MANS_U8, MANS_U16, MANS_U32 = 1, 2, 4

# Every symbol include/mans.h declares, with (restype, argtypes).
_vp, _u64, _u32, _i32 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int
class BatchSchedule(C.Structure):
    """mans_batch_schedule (include/mans.h): per stage (map, plan, encode,
    decode plan, decode, unmap) resident CTAs per SM, warps per CTA and L2
    prefetch distance in grids of units ahead."""
    _fields_ = [("ctas_per_sm", C.c_int * 6), ("warps_per_cta", C.c_int * 6),
                ("prefetch_grids", C.c_int * 6)]


SIGNATURES = {
    "mans_workspace_create": (_i32, [C.POINTER(_vp), _u64, _u64]),
    "mans_workspace_destroy": (_i32, [_vp]),
    "mans_workspace_device_bytes": (_u64, [_vp]),
    "mans_workspace_status": (_i32, [_vp, _vp, C.POINTER(_u64)]),
    "mans_workspace_set_timing": (_i32, [_vp, _i32]),
    "mans_workspace_kernel_times": (_i32, [_vp, C.POINTER(C.c_float), C.POINTER(C.c_int)]),
    "mans_max_compressed_size": (_u64, [_i32, _u64]),
    "mans_max_mapped_size": (_u64, [_i32, _u64]),
    "mans_stream_bound": (_u64, [_u64]),
    "mans_compress": (_i32, [_vp, _i32, _vp, _u64, _vp, _u64, _vp, _i32, _vp]),
    "mans_decompress": (_i32, [_vp, _i32, _vp, _u64, _vp, _u64, _vp]),
    "mans_compress_ex": (_i32, [_vp, _i32, _i32, _vp, _u64, _vp, _u64, _vp, _i32, _vp]),
    "mans_decompress_ex": (_i32, [_vp, _i32, _i32, _vp, _u64, _vp, _u64, _vp]),
    "mans_adm_map": (_i32, [_vp, _i32, _i32, _vp, _u64, _vp, _u64, _vp, _vp]),
    "mans_adm_unmap": (_i32, [_vp, _i32, _i32, _vp, _u64, _vp, _u64, _vp]),
    "mans_frame_max_size": (_u64, [_i32, _u64]),
    "mans_frame_compress": (_i32, [_vp, _i32, _i32, _vp, _u64, _vp, _u64, _vp, _i32, _vp]),
    "mans_frame_parse": (_i32, [_vp, _u64, _vp]),
    "mans_frame_decompress": (_i32, [_vp, _vp, _vp, _vp, _u64, _vp]),
    "mans_ans_encode": (_i32, [_i32, _vp, _u32, _vp, _vp, _vp]),
    "mans_ans_decode": (_i32, [_i32, _vp, _vp, _vp]),
    "mans_ans_encode_batch": (_i32, [_i32, _vp, _u32, _vp, _vp, _vp]),
    "mans_ans_decode_batch": (_i32, [_i32, _vp, _vp, _vp]),
    "mans_ans_max_compressed_size": (_u32, [_u32]),
    "mans_ans_last_status": (_i32, [_vp, C.POINTER(_u64)]),
    "mans_ans_encode_noalloc": (_i32, [_i32, _vp, _u32, _vp, _vp, _vp]),
    "mans_ans_noalloc_status": (_i32, [_vp, C.POINTER(_u64)]),
    "mans_batch_create": (_i32, [C.POINTER(_vp), _u32, _u64, _u32]),
    "mans_batch_destroy": (_i32, [_vp]),
    "mans_batch_device_bytes": (_u64, [_vp]),
    "mans_batch_compress": (_i32, [_vp, _vp, _u32, _vp]),
    "mans_batch_decompress": (_i32, [_vp, _vp, _u32, _vp]),
    "mans_batch_status": (_i32, [_vp, _vp, C.POINTER(_u32), C.POINTER(_u64), _u32]),
    "mans_batch_set_timing": (_i32, [_vp, _i32]),
    "mans_batch_stage_times": (_i32, [_vp, C.POINTER(C.c_float), C.POINTER(C.c_int)]),
    "mans_batch_get_schedule": (_i32, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "mans_batch_set_schedule": (_i32, [_vp, C.POINTER(C.c_int)]),
    "mans_batch_get_schedule_ex": (_i32, [_vp, C.POINTER(BatchSchedule), C.POINTER(BatchSchedule)]),
    "mans_batch_set_schedule_ex": (_i32, [_vp, C.POINTER(BatchSchedule)]),
    "mans_batch_autotune": (_i32, [_vp, _vp, _u32, _vp, C.POINTER(C.c_float)]),
    "mans_clock_ns": (_u64, []),
    "mans_server_create": (_i32, [C.POINTER(_vp), _vp]),
    "mans_server_destroy": (_i32, [_vp]),
    "mans_server_submit": (_i32, [_vp, _vp, C.POINTER(_u64)]),
    "mans_server_poll": (_i32, [_vp, _vp, _u32, C.POINTER(_u32), _u32]),
    "mans_server_release": (_i32, [_vp, _u64]),
    "mans_server_get_stats": (_i32, [_vp, _vp]),
    "mans_debug_arena": (_u64, [_u64, _vp, _u32, _vp]),
    "mans_version": (C.c_char_p, []),
    "mans_debug_enc_entry": (None, [_u32, _u32, _i32, C.POINTER(_u32)]),
    "mans_debug_bounded_wait": (_i32, [C.POINTER(_u32), C.POINTER(C.c_float)]),
}

_LIB: Optional[C.CDLL] = None


class MansError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        super().__init__(f"{what}: {STATUS.get(code, code)}" if what else STATUS.get(code, str(code)))


def load(build_if_missing: bool = False) -> C.CDLL:
    """Load libmans_b200.so (raise if it is absent)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise RuntimeError(f"{LIB_PATH} not built; run `python -m mans_b200.build`")
        from . import build as _b
        _b.build()
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _LIB = lib
    return lib


def _check(code: int, what: str) -> None:
    if code != 0:
        raise MansError(code, what)


def _torch():
    import torch
    return torch


def _stream_handle(stream) -> int:
    torch = _torch()
    if stream is None:
        stream = torch.cuda.current_stream()
    return int(stream.cuda_stream)


_DTYPE_CODE = {"uint8": MANS_U8, "uint16": MANS_U16, "uint32": MANS_U32}


def dtype_code(t) -> int:
    name = str(t.dtype).replace("torch.", "")
    if name not in _DTYPE_CODE:
        raise TypeError(f"unsupported dtype {t.dtype}; use uint8, uint16 or uint32")
    return _DTYPE_CODE[name]


def max_compressed_size(dtype: int, n_elems: int) -> int:
    return int(load().mans_max_compressed_size(dtype, n_elems))


def max_mapped_size(dtype: int, n_elems: int) -> int:
    """Worst-case mapped bytes of n elements (mans_max_mapped_size)."""
    return int(load().mans_max_mapped_size(dtype, n_elems))


def stream_bound(mapped_bytes: int) -> int:
    """Worst-case stream bytes for mapped_bytes of rANS input (mans_stream_bound)."""
    return int(load().mans_stream_bound(mapped_bytes))


def getMaxCompressedSize(in_size: int) -> int:  # noqa: N802 (reference name)
    """multibyte_ans::getMaxCompressedSize (include/ans/GpuANSCodec.h:237)."""
    return int(load().mans_ans_max_compressed_size(in_size))


class Workspace:
    """Device scratch reused across calls (mans_workspace_create)."""

    def __init__(self, max_input_bytes: int, merged_capacity: int = 0):
        lib = load()
        h = C.c_void_p()
        _check(lib.mans_workspace_create(C.byref(h), max_input_bytes, merged_capacity),
               "mans_workspace_create")
        self.h = h
        self.max_input_bytes = max_input_bytes

    @property
    def device_bytes(self) -> int:
        return int(load().mans_workspace_device_bytes(self.h))

    def status(self, stream=None) -> tuple[int, int]:
        d = C.c_uint64(0)
        st = load().mans_workspace_status(self.h, _stream_handle(stream), C.byref(d))
        return int(st), int(d.value)

    def check(self, stream=None, what: str = "device") -> None:
        st, det = self.status(stream)
        if st != 0:
            raise MansError(st, f"{what} (detail {det})")

    def set_timing(self, enable: bool = True) -> None:
        _check(load().mans_workspace_set_timing(self.h, int(enable)), "mans_workspace_set_timing")

    def kernel_times(self) -> dict:
        """Summed kernel milliseconds and call counts recorded since the last read."""
        ms = (C.c_float * 4)()
        calls = (C.c_int * 2)()
        _check(load().mans_workspace_kernel_times(self.h, ms, calls), "mans_workspace_kernel_times")
        return {"map": ms[0], "encode": ms[1], "decode": ms[2], "unmap": ms[3],
                "compress_calls": calls[0], "decompress_calls": calls[1]}

    def close(self) -> None:
        if getattr(self, "h", None):
            load().mans_workspace_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# mans_layout: mapped-buffer layouts (uint16 compatibility modes)
LAYOUT_NATIVE, LAYOUT_V12, LAYOUT_CPUV2 = 0, 1, 2


def compress_into(ws: Workspace, x, out, out_size, precision: int = 10, stream=None,
                  layout: int = LAYOUT_NATIVE) -> None:
    """Enqueue MANS compress of device tensor x into out (uint8) and out_size (int64[1])."""
    n = x.numel()
    code = dtype_code(x)
    _check(load().mans_compress_ex(ws.h, code, layout, x.data_ptr() if n else None, n,
                                   out.data_ptr(), out.numel(), out_size.data_ptr(), precision,
                                   _stream_handle(stream)), "mans_compress")


def decompress_into(ws: Workspace, stream_bytes, in_size: int, out, stream=None,
                    layout: int = LAYOUT_NATIVE) -> None:
    """Enqueue MANS decompress of stream_bytes[:in_size] into out (dtype decides the mapping)."""
    n = out.numel()
    code = dtype_code(out)
    _check(load().mans_decompress_ex(ws.h, code, layout, stream_bytes.data_ptr(), in_size,
                                     out.data_ptr() if n else None, n, _stream_handle(stream)),
           "mans_decompress")


def adm_map(x, layout: int = LAYOUT_NATIVE, ws: Optional[Workspace] = None, stream=None):
    """The mapped buffer of device tensor x (uint16/uint32) as the reference's mappers write it."""
    torch = _torch()
    n = x.numel()
    own = ws is None
    if own:
        ws = Workspace(max(n * x.element_size(), 1))
    cap = n * x.element_size() * 3 + 65536
    out = torch.empty(cap, dtype=torch.uint8, device=x.device)
    size = torch.zeros(1, dtype=torch.int64, device=x.device)
    _check(load().mans_adm_map(ws.h, dtype_code(x), layout, x.data_ptr() if n else None, n,
                               out.data_ptr(), cap, size.data_ptr(), _stream_handle(stream)),
           "mans_adm_map")
    ws.check(stream, "mans_adm_map")
    res = out[: int(size.item())].clone()
    if own:
        ws.close()
    return res


def adm_unmap(m, n: int, dtype, layout: int = LAYOUT_NATIVE, ws: Optional[Workspace] = None,
              stream=None):
    """Inverse of adm_map: n values of dtype from the mapped buffer m (device uint8)."""
    torch = _torch()
    out = torch.empty(n, dtype=dtype, device=m.device)
    own = ws is None
    if own:
        ws = Workspace(max(n * out.element_size(), 1))
    _check(load().mans_adm_unmap(ws.h, dtype_code(out), layout, m.data_ptr() if m.numel() else None,
                                 m.numel(),
                                 out.data_ptr() if n else None, n, _stream_handle(stream)),
           "mans_adm_unmap")
    ws.check(stream, "mans_adm_unmap")
    if own:
        ws.close()
    return out


def compress(x, precision: int = 10, ws: Optional[Workspace] = None, stream=None,
             layout: int = LAYOUT_NATIVE):
    """Compress device tensor x (uint8/uint16/uint32); returns a uint8 tensor (synchronises)."""
    torch = _torch()
    n = x.numel()
    code = dtype_code(x)
    own = ws is None
    if own:
        ws = Workspace(max(n * x.element_size(), 1))
    cap = max_compressed_size(code, n)
    out = torch.empty(cap, dtype=torch.uint8, device=x.device)
    size = torch.zeros(1, dtype=torch.int64, device=x.device)
    compress_into(ws, x, out, size, precision, stream, layout)
    ws.check(stream, "mans_compress")
    nbytes = int(size.item())
    res = out[:nbytes].clone()
    if own:
        ws.close()
    return res


def decompress(s, n: int, dtype, ws: Optional[Workspace] = None, stream=None,
               layout: int = LAYOUT_NATIVE):
    """Decompress a stream (device uint8 tensor) of n elements of dtype (synchronises)."""
    torch = _torch()
    out = torch.empty(n, dtype=dtype, device=s.device)
    own = ws is None
    if own:
        ws = Workspace(max(n * out.element_size(), 1))
    decompress_into(ws, s, s.numel(), out, stream, layout)
    ws.check(stream, "mans_decompress")
    if own:
        ws.close()
    return out


# ---- self-describing frames ----
class FrameInfo(C.Structure):
    """mans_frame_info (include/mans.h)."""
    _fields_ = [("dtype", C.c_int), ("layout", C.c_int), ("precision", C.c_int),
                ("header_bytes", C.c_uint32), ("n_elems", C.c_uint64),
                ("mapped_bytes", C.c_uint64), ("stream_bytes", C.c_uint64)]


FRAME_HEADER_BYTES = 64
_CODE_DTYPE = {MANS_U8: "uint8", MANS_U16: "uint16", MANS_U32: "uint32"}


def frame_parse(header: bytes, avail: Optional[int] = None) -> FrameInfo:
    """Parse a frame header from host bytes (the whole frame, or at least its
    64-byte header). avail: bytes of the frame available (default: len(header)
    when more than the header is given, else unknown)."""
    buf = (C.c_uint8 * max(len(header), 1)).from_buffer_copy(bytes(header) or b"\0")
    info = FrameInfo()
    if avail is None:
        avail = len(header) if len(header) > FRAME_HEADER_BYTES else (1 << 64) - 1
    _check(load().mans_frame_parse(C.cast(buf, C.c_void_p), avail, C.byref(info)), "mans_frame_parse")
    return info


def frame_compress(x, precision: int = 10, layout: int = LAYOUT_NATIVE,
                   ws: Optional[Workspace] = None, stream=None):
    """Compress device tensor x into a self-describing frame (uint8 tensor; synchronises)."""
    torch = _torch()
    n = x.numel()
    code = dtype_code(x)
    own = ws is None
    if own:
        ws = Workspace(max(n * x.element_size(), 1))
    cap = int(load().mans_frame_max_size(code, n))
    out = torch.empty(cap, dtype=torch.uint8, device=x.device)
    size = torch.zeros(1, dtype=torch.int64, device=x.device)
    _check(load().mans_frame_compress(ws.h, code, layout, x.data_ptr() if n else None, n,
                                      out.data_ptr(), cap, size.data_ptr(), precision,
                                      _stream_handle(stream)), "mans_frame_compress")
    ws.check(stream, "mans_frame_compress")
    res = out[: int(size.item())].clone()
    if own:
        ws.close()
    return res


def frame_decompress(frame, ws: Optional[Workspace] = None, stream=None):
    """Decompress a frame (device uint8 tensor); the element type and count come from its header."""
    torch = _torch()
    info = frame_parse(frame[:FRAME_HEADER_BYTES].cpu().numpy().tobytes())
    if FRAME_HEADER_BYTES + info.stream_bytes > frame.numel():
        raise MansError(7, "frame_decompress: truncated frame")
    dt = getattr(torch, _CODE_DTYPE[info.dtype])
    out = torch.empty(info.n_elems, dtype=dt, device=frame.device)
    own = ws is None
    if own:
        ws = Workspace(max(out.numel() * out.element_size(), 1))
    _check(load().mans_frame_decompress(ws.h, C.byref(info), frame.data_ptr(),
                                        out.data_ptr() if out.numel() else None,
                                        out.numel() * out.element_size(), _stream_handle(stream)),
           "mans_frame_decompress")
    ws.check(stream, "mans_frame_decompress")
    if own:
        ws.close()
    return out


# ---- reference-named rANS entry points (include/ans, src/GpuANS.cu) ----
def ansEncode(precision: int, d_in, in_size: int, d_out, d_out_size, stream=None) -> None:  # noqa: N802
    """multibyte_ans::ansEncode (include/ans/GpuANSEncode.h:286); d_out_size is a device uint32/int32[1]."""
    _check(load().mans_ans_encode(precision, d_in.data_ptr(), in_size, d_out.data_ptr(),
                                  d_out_size.data_ptr(), _stream_handle(stream)), "ansEncode")


def ansDecode(precision: int, d_in, d_out, stream=None) -> None:  # noqa: N802
    """multibyte_ans::ansDecode (include/ans/GpuANSDecode.h:379)."""
    _check(load().mans_ans_decode(precision, d_in.data_ptr(), d_out.data_ptr(),
                                  _stream_handle(stream)), "ansDecode")


ansEncodeBatch = ansEncode  # src/GpuANS.cu:16 forwards to ansEncode
ansDecodeBatch = ansDecode  # src/GpuANS.cu:33 forwards to ansDecode


def ans_last_status(stream=None) -> tuple[int, int]:
    d = C.c_uint64(0)
    st = load().mans_ans_last_status(_stream_handle(stream), C.byref(d))
    return int(st), int(d.value)


def version() -> str:
    return load().mans_version().decode()
