"""Shared helpers for the GPU tests: host<->device moves of numpy arrays."""
import numpy as np


def to_dev(x: np.ndarray):
    import torch
    tdt = {np.dtype(np.uint8): torch.uint8, np.dtype(np.uint16): torch.uint16,
           np.dtype(np.uint32): torch.uint32}[x.dtype]
    if x.size == 0:
        return torch.empty(0, dtype=tdt, device="cuda")
    b = torch.from_numpy(np.ascontiguousarray(x).view(np.uint8).copy()).cuda()
    if x.dtype == np.uint8:
        return b
    return b.view({np.dtype(np.uint16): torch.uint16, np.dtype(np.uint32): torch.uint32}[x.dtype])


def to_host(t, dtype=np.uint8) -> np.ndarray:
    import torch
    b = t.contiguous().view(torch.uint8).cpu().numpy()
    return b.view(dtype)
