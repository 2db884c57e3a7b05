"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark configurations (the reference's datasets are not available, so
these generators stand in for them).

* ``laplace_u16``   -- single uint16 buffer: round(32768 + Laplace(0, 40)),
                       clipped; 4,194,304 values (tomography-like).
* ``detector_u32``  -- uint32 detector frames: round(Gamma(k=0.5, theta=20))
                       background with 0.1% of pixels replaced by uniform
                       integer peaks in [1e4, 1e6].
* ``gradient_u16``  -- smooth 2-D gradient plus Gaussian noise (mean 8000,
                       sigma 200) on rows of 1024.
* ``quant_u32``     -- Laplace(0, 300) quantisation codes offset by 2^31.
* ``volume_u16``    -- per-row N(20000, 3000) offsets plus per-pixel N(0, 150)
                       noise on rows of 2048, rounded and clipped.
* ``mixed_sizes``   -- buffer sizes log-uniform in [4 KiB, 64 MiB], rounded
                       down to a multiple of 1 KiB.

``gen_device`` / ``gen_mixed_device`` draw the same distributions with torch
on the GPU (different random streams), for the full-size workloads.
"""
from __future__ import annotations

import numpy as np

C1_N = 4_194_304               # 8 MiB of uint16
C2_N = 16 * 4096 * 4096        # 1 GiB of uint32
C4_N = 2048 * 2048 * 256       # 2 GiB of uint16


def laplace_u16(n: int, seed: int = 1, b: float = 40.0, center: float = 32768.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    x = np.round(center + rng.laplace(0.0, b, n))
    return np.clip(x, 0, 65535).astype(np.uint16)


def detector_u32(n: int, seed: int = 2, peak_frac: float = 0.001) -> np.ndarray:
    rng = np.random.default_rng(seed)
    x = np.round(rng.gamma(0.5, 20.0, n)).astype(np.uint32)
    m = rng.random(n) < peak_frac
    x[m] = rng.integers(10_000, 1_000_001, int(m.sum()), dtype=np.uint32)
    return x


def gradient_u16(n: int, seed: int = 3, width: int = 1024) -> np.ndarray:
    rng = np.random.default_rng(seed)
    h = max(1, -(-n // width))
    a, b = rng.uniform(-1000, 1000, 2)
    yy, xx = np.meshgrid(np.arange(h, dtype=np.float64), np.arange(width, dtype=np.float64),
                         indexing="ij")
    v = 8000.0 + a * xx / width + b * yy / h + rng.normal(0, 200, (h, width))
    return np.clip(np.round(v), 0, 65535).astype(np.uint16).ravel()[:n]


def quant_u32(n: int, seed: int = 3, b: float = 300.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = np.round(rng.laplace(0.0, b, n)).astype(np.int64) + (1 << 31)
    return np.clip(v, 0, 0xFFFFFFFF).astype(np.uint32)


def volume_u16(n: int, seed: int = 4, width: int = 2048) -> np.ndarray:
    rng = np.random.default_rng(seed)
    rows = -(-n // width)
    off = rng.normal(20000.0, 3000.0, rows)
    v = off[:, None] + rng.normal(0.0, 150.0, (rows, width))
    return np.clip(np.round(v), 0, 65535).astype(np.uint16).ravel()[:n]


def mixed_sizes(count: int, seed: int = 3, lo: int = 4 << 10, hi: int = 64 << 20) -> np.ndarray:
    rng = np.random.default_rng(seed)
    s = np.exp(rng.uniform(np.log(lo), np.log(hi), count))
    return (np.floor(s / 1024) * 1024).astype(np.int64)


def random_bytes(n: int, seed: int, kind: str = "skewed") -> np.ndarray:
    """Byte buffers for rANS-only tests: uniform, skewed (geometric), single, two-symbol."""
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        return rng.integers(0, 256, n, dtype=np.uint8)
    if kind == "single":
        return np.full(n, 7, np.uint8)
    if kind == "two":
        return np.where(rng.random(n) < 0.9, 3, 250).astype(np.uint8)
    if kind == "sparse":  # few symbols, most of them rare
        v = rng.geometric(0.3, n) - 1
        return np.minimum(v, 255).astype(np.uint8)
    v = np.minimum(rng.geometric(0.05, n) - 1, 255)
    return v.astype(np.uint8)


# ---- the same distributions generated on the GPU (fast at 1-2 GiB) ----
def gen_device(workload: str, n: int, seed: int):
    """Seeded synthetic input generated on the GPU (same distributions as
    mans_b200.workloads, which makes the CPU samples)."""
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    chunk = 1 << 26
    if workload == "detector_u32":
        out = torch.empty(n, dtype=torch.int64, device="cuda")
        for s in range(0, n, chunk):
            m = min(chunk, n - s)
            alpha = torch.full((m,), 0.5, device="cuda")
            v = torch.round(torch._standard_gamma(alpha, generator=g) * 20.0).to(torch.int64)
            peak = torch.rand(m, device="cuda", generator=g) < 0.001
            pv = torch.randint(10_000, 1_000_001, (m,), device="cuda", generator=g)
            out[s:s + m] = torch.where(peak, pv, v)
        return out.to(torch.int32).view(torch.uint32)
    if workload == "laplace_u16":
        x = laplace_u16(n, seed)
        return torch.from_numpy(x.view(np.uint8).copy()).cuda().view(torch.uint16)
    if workload in ("gradient_u16", "quant_u32"):
        it = {"elem": 2 if workload == "gradient_u16" else 4, "n": n, "off": 0, "a": 613.0, "b": -287.0}
        it["bytes"] = n * it["elem"]
        pool = gen_mixed_device([it], it["bytes"], seed)
        return pool.view(torch.uint16 if it["elem"] == 2 else torch.uint32)
    if workload == "volume_u16":
        width = 2048
        rows = n // width
        out = torch.empty(n, dtype=torch.int32, device="cuda")
        rs = 1 << 14
        for r0 in range(0, rows, rs):
            r = min(rs, rows - r0)
            off = torch.randn(r, 1, device="cuda", generator=g) * 3000.0 + 20000.0
            v = off + torch.randn(r, width, device="cuda", generator=g) * 150.0
            out[r0 * width:(r0 + r) * width] = torch.clamp(torch.round(v), 0, 65535).to(torch.int32).view(-1)
        return out.to(torch.int16).view(torch.uint16)
    raise ValueError(workload)


def gen_mixed_device(items, total: int, seed: int):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    pool = torch.zeros(total, dtype=torch.uint8, device="cuda")
    for it in items:
        n = it["n"]
        if it["elem"] == 2:
            idx = torch.arange(n, device="cuda", dtype=torch.int64)
            h = -(-n // 1024)
            v = (8000.0 + it["a"] * (idx % 1024).to(torch.float32) / 1024.0
                 + it["b"] * (idx // 1024).to(torch.float32) / h
                 + torch.randn(n, device="cuda", generator=g) * 200.0)
            v = torch.clamp(torch.round(v), 0, 65535).to(torch.int32).to(torch.int16)
        else:
            u = torch.rand(n, device="cuda", generator=g, dtype=torch.float64) - 0.5
            lap = -300.0 * torch.sign(u) * torch.log(torch.clamp(1.0 - 2.0 * u.abs(), min=1e-300))
            v = torch.clamp(torch.round(lap).to(torch.int64) + (1 << 31), 0, (1 << 32) - 1)
            v = torch.where(v >= (1 << 31), v - (1 << 32), v).to(torch.int32)
        pool[it["off"]:it["off"] + it["bytes"]].copy_(v.view(torch.uint8))
    return pool
