"""ctypes bindings of the C oracle and of the reference code compiled as a checker.

TEST INFRASTRUCTURE: imported by tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` only.

* ``libmans_oracle.so`` -- the C restatement (``oracle/mans_oracle.c``).
* ``_ref/libref_adm_cpu.so`` -- the reference's own CPU ADM mapping
  (mapping/cpu/mappingcpuV2.cpp) behind a small C shim, present when the
  reference tree was available at build time.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

u8p = C.POINTER(C.c_uint8)
u16p = C.POINTER(C.c_uint16)
u32p = C.POINTER(C.c_uint32)


def build(ref: bool = False) -> None:
    """Compile the oracle (and with ref=True the reference checkers)."""
    subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", _HERE, "ref"], check=True)


def _ptr(a: np.ndarray, t=u8p):
    return a.ctypes.data_as(t)


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libmans_oracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        i64, u64, i32 = C.c_int64, C.c_uint64, C.c_int
        sig = {
            "mo_adm_u16_merged_size": (u64, [u16p, u64]),
            "mo_adm_u16_map": (i64, [u16p, u64, u8p, u64]),
            "mo_adm_u16_unmap": (i32, [u8p, u64, u64, u16p]),
            "mo_adm_u16_header_bytes": (u64, [u64, i32]),
            "mo_adm_u16_map_layout": (i64, [u16p, u64, i32, u8p, u64]),
            "mo_adm_u16_unmap_layout": (i32, [u8p, u64, u64, i32, u16p]),
            "mo_adm_u32_max_merged_size": (u64, [u64]),
            "mo_adm_u32_map": (i64, [u32p, u64, u8p, u64]),
            "mo_adm_u32_unmap": (i32, [u8p, u64, u64, u32p]),
            "mo_ans_histogram": (None, [u8p, u64, u32p]),
            "mo_ans_normalize": (i32, [u32p, C.c_uint32, i32, u32p, u32p]),
            "mo_ans_max_compressed_size": (u64, [u64]),
            "mo_ans_encode": (i64, [i32, u8p, u64, u8p, u64]),
            "mo_ans_encode_ex": (i64, [i32, u8p, u64, u8p, u64, u32p]),
            "mo_ans_decode": (i32, [u8p, u64, u8p, u64, C.POINTER(u64)]),
            "mo_ans_stream_uncompressed_size": (u64, [u8p, u64]),
            "mo_ans_mask": (None, [u8p, u64]),
            "mo_mans_compress_u16": (i64, [i32, u16p, u64, u8p, u64]),
            "mo_mans_decompress_u16": (i32, [u8p, u64, u64, u16p]),
            "mo_mans_compress_u32": (i64, [i32, u32p, u64, u8p, u64]),
            "mo_mans_decompress_u32": (i32, [u8p, u64, u64, u32p]),
            "mo_set_threads": (None, [i32]),
            "mo_ans_histogram_par": (None, [u8p, u64, u32p]),
            "mo_ans_par_scratch_words": (u64, [u64]),
            "mo_ans_encode_par": (i64, [i32, u8p, u64, u8p, u64, u16p, u32p, u32p]),
            "mo_ans_decode_par": (i32, [u8p, u64, u8p, u64]),
            "mo_adm_u16_map_layout_par": (i64, [u16p, u64, i32, u8p, u64]),
            "mo_adm_u32_map_par": (i64, [u32p, u64, u8p, u64]),
            "mo_adm_u32_unmap_par": (i32, [u8p, u64, u64, u32p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


# ---------------------------------------------------------------- ADM u16
# uint16 merged layouts: V15 (canonical), V12 (u16 lengths), CPU-V2 (g + 1 prefix words)
LAYOUT_V15, LAYOUT_V12, LAYOUT_CPUV2 = 0, 1, 2


def adm_u16_map(x: np.ndarray, layout: int = LAYOUT_V15) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.uint16)
    L = lib()
    n = x.size
    size = L.mo_adm_u16_merged_size(_ptr(x, u16p), n) - L.mo_adm_u16_header_bytes(n, 0) + \
        L.mo_adm_u16_header_bytes(n, layout)
    out = np.zeros(max(size, 1), np.uint8)
    r = L.mo_adm_u16_map_layout(_ptr(x, u16p), n, layout, _ptr(out), size)
    assert r == size, (r, size)
    return out[:size]


def adm_u16_unmap(m: np.ndarray, n: int, layout: int = LAYOUT_V15) -> np.ndarray:
    m = np.ascontiguousarray(m, dtype=np.uint8)
    out = np.zeros(max(n, 1), np.uint16)
    rc = lib().mo_adm_u16_unmap_layout(_ptr(m), m.size, n, layout, _ptr(out, u16p))
    if rc != 0:
        raise ValueError(f"adm_u16_unmap failed: {rc}")
    return out[:n]


# ---------------------------------------------------------------- ADM u32
def adm_u32_map(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.uint32)
    L = lib()
    cap = L.mo_adm_u32_max_merged_size(x.size)
    out = np.zeros(max(cap, 1), np.uint8)
    r = L.mo_adm_u32_map(_ptr(x, u32p), x.size, _ptr(out), cap)
    assert r >= 0
    return out[:r]


def adm_u32_unmap(m: np.ndarray, n: int) -> np.ndarray:
    m = np.ascontiguousarray(m, dtype=np.uint8)
    out = np.zeros(max(n, 1), np.uint32)
    rc = lib().mo_adm_u32_unmap(_ptr(m), m.size, n, _ptr(out, u32p))
    if rc != 0:
        raise ValueError(f"adm_u32_unmap failed: {rc}")
    return out[:n]


# ---------------------------------------------------------------- rANS
def histogram(b: np.ndarray) -> np.ndarray:
    b = np.ascontiguousarray(b, dtype=np.uint8)
    h = np.zeros(256, np.uint32)
    lib().mo_ans_histogram(_ptr(b), b.size, _ptr(h, u32p))
    return h


def normalize(hist: np.ndarray, total: int, prob_bits: int):
    hist = np.ascontiguousarray(hist, dtype=np.uint32)
    pdf = np.zeros(256, np.uint32)
    cdf = np.zeros(256, np.uint32)
    rc = lib().mo_ans_normalize(_ptr(hist, u32p), total, prob_bits, _ptr(pdf, u32p), _ptr(cdf, u32p))
    assert rc == 0
    return pdf, cdf


def max_compressed_size(n: int) -> int:
    return int(lib().mo_ans_max_compressed_size(n))


def ans_encode(b: np.ndarray, prob_bits: int = 10, with_block_words: bool = False):
    b = np.ascontiguousarray(b, dtype=np.uint8)
    cap = max_compressed_size(b.size)
    out = np.zeros(cap, np.uint8)
    nb = (b.size + 4095) // 4096
    bw = np.zeros(max(nb, 1), np.uint32)
    r = lib().mo_ans_encode_ex(prob_bits, _ptr(b), b.size, _ptr(out), cap, _ptr(bw, u32p))
    if r < 0:
        raise ValueError(f"ans_encode failed: {r}")
    if with_block_words:
        return out[:r], bw[:nb]
    return out[:r]


def ans_decode(s: np.ndarray) -> np.ndarray:
    s = np.ascontiguousarray(s, dtype=np.uint8)
    L = lib()
    n = L.mo_ans_stream_uncompressed_size(_ptr(s), s.size)
    out = np.zeros(max(n, 1), np.uint8)
    got = C.c_uint64(0)
    rc = L.mo_ans_decode(_ptr(s), s.size, _ptr(out), n, C.byref(got))
    if rc != 0:
        raise ValueError(f"ans_decode failed: {rc}")
    return out[: got.value]


def ans_mask(s: np.ndarray) -> np.ndarray:
    s = np.array(s, dtype=np.uint8, copy=True)
    lib().mo_ans_mask(_ptr(s), s.size)
    return s


# ---------------------------------------------------------------- MANS
def compress(x: np.ndarray, prob_bits: int = 10, layout: int = LAYOUT_V15) -> np.ndarray:
    if x.dtype == np.uint16:
        m = adm_u16_map(x, layout)
    elif x.dtype == np.uint32:
        m = adm_u32_map(x)
    else:
        raise TypeError(x.dtype)
    return ans_encode(m, prob_bits)


def decompress(s: np.ndarray, n: int, dtype, layout: int = LAYOUT_V15) -> np.ndarray:
    m = ans_decode(s)
    if np.dtype(dtype) == np.uint16:
        return adm_u16_unmap(m, n, layout)
    return adm_u32_unmap(m, n)


def compress_par(x: np.ndarray, prob_bits: int = 10, layout: int = LAYOUT_V15,
                 threads: int = 0) -> np.ndarray:
    """compress() with the group- and block-parallel (OpenMP) variants: the
    same bytes, fast enough for inputs of several GiB."""
    L = lib()
    if threads:
        L.mo_set_threads(threads)
    n = x.size
    if x.dtype == np.uint16:
        x = np.ascontiguousarray(x)
        cap = L.mo_adm_u16_map_layout_par(_ptr(x, u16p), n, layout, None, 0)
        m = np.empty(max(cap, 1), np.uint8)
        ms = L.mo_adm_u16_map_layout_par(_ptr(x, u16p), n, layout, _ptr(m), cap)
    elif x.dtype == np.uint32:
        x = np.ascontiguousarray(x)
        cap = L.mo_adm_u32_max_merged_size(n)
        m = np.empty(max(cap, 1), np.uint8)
        ms = L.mo_adm_u32_map_par(_ptr(x, u32p), n, _ptr(m), cap)
    else:
        raise TypeError(x.dtype)
    if ms < 0:
        raise ValueError(f"mapping failed: {ms}")
    scap = max_compressed_size(ms)
    out = np.empty(scap, np.uint8)
    nb = (ms + 4095) // 4096
    scr = np.empty(max(L.mo_ans_par_scratch_words(ms), 1), np.uint16)
    sst = np.empty(max(32 * nb, 1), np.uint32)
    snw = np.empty(max(nb, 1), np.uint32)
    r = L.mo_ans_encode_par(prob_bits, _ptr(m), ms, _ptr(out), scap, _ptr(scr, u16p),
                            _ptr(sst, u32p), _ptr(snw, u32p))
    if r < 0:
        raise ValueError(f"ans_encode_par failed: {r}")
    return out[:r]


# ---------------------------------------------------------------- reference CPU ADM
def ref_lib():
    """The reference's own CPU ADM mapping, or None if it was not built."""
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libref_adm_cpu.so")
        if not os.path.exists(path):
            return None
        R = C.CDLL(path)
        R.ref_adm_cpu_create.restype = C.c_void_p
        R.ref_adm_cpu_create.argtypes = [u16p, C.c_uint64]
        R.ref_adm_cpu_destroy.argtypes = [C.c_void_p]
        R.ref_adm_cpu_compress.argtypes = [C.c_void_p]
        R.ref_adm_cpu_decompress.argtypes = [C.c_void_p]
        R.ref_adm_cpu_merged_size.restype = C.c_uint64
        R.ref_adm_cpu_merged_size.argtypes = [C.c_void_p, C.c_int]
        R.ref_adm_cpu_merged.restype = C.c_uint64
        R.ref_adm_cpu_merged.argtypes = [C.c_void_p, C.c_int, u8p]
        R.ref_adm_cpu_recovered.restype = C.c_uint64
        R.ref_adm_cpu_recovered.argtypes = [C.c_void_p, u16p]
        R.ref_adm_cpu_set_threads.argtypes = [C.c_int]
        R.ref_adm_cpu_get_threads.restype = C.c_int
        _REF = R
    return _REF


class RefAdmCpu:
    """Handle over the reference CPU mapping (mappingcpuV2.cpp compress/decompress)."""

    def __init__(self, x: np.ndarray, threads: int = 1):
        self.R = ref_lib()
        if self.R is None:
            raise RuntimeError("reference CPU mapping not built (oracle/_ref)")
        self.R.ref_adm_cpu_set_threads(threads)
        self.x = np.ascontiguousarray(x, dtype=np.uint16)
        self.h = self.R.ref_adm_cpu_create(_ptr(self.x, u16p), self.x.size)

    def compress(self):
        self.R.ref_adm_cpu_compress(self.h)

    def decompress(self):
        self.R.ref_adm_cpu_decompress(self.h)

    def merged(self, v15_layout: bool = True) -> np.ndarray:
        sz = self.R.ref_adm_cpu_merged_size(self.h, int(v15_layout))
        out = np.zeros(max(sz, 1), np.uint8)
        self.R.ref_adm_cpu_merged(self.h, int(v15_layout), _ptr(out))
        return out[:sz]

    def recovered(self) -> np.ndarray:
        out = np.zeros(max(self.x.size, 1), np.uint16)
        n = self.R.ref_adm_cpu_recovered(self.h, _ptr(out, u16p))
        return out[:n]

    def close(self):
        if self.h:
            self.R.ref_adm_cpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
