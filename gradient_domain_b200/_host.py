"""Host <-> device transfers of the NumPy entry points.

The reference's functions take and return NumPy arrays, so every call moves
its images across PCIe.  From pageable NumPy memory the driver copies through
its own bounce buffers (about 10 GB/s up and, into freshly allocated result
arrays that are still being faulted in, about 2 GB/s down).  Larger arrays go
through page-locked memory from torch's pinned-memory cache instead: the input
is copied into a pinned buffer by a multi-threaded host copy and then moved by
DMA at PCIe speed, and results are copied by DMA straight into a pinned buffer
that the returned array wraps (the buffer returns to torch's cache when the
array is released).
"""

from __future__ import annotations

import numpy as np
import torch

_STAGE_MIN_BYTES = 1 << 20  # smaller arrays take the direct path


def upload(a, dev: torch.device, dtype=None) -> torch.Tensor:
    """A NumPy array (or anything ``np.asarray`` takes) as a tensor on ``dev``."""
    arr = np.ascontiguousarray(a, dtype=dtype)
    src = torch.from_numpy(arr)
    if arr.nbytes < _STAGE_MIN_BYTES:
        return src.to(dev)
    stage = torch.empty(src.shape, dtype=src.dtype, pin_memory=True)
    stage.copy_(src)
    return stage.to(dev, non_blocking=True)


def download(t: torch.Tensor) -> np.ndarray:
    """A device tensor as a NumPy array (contiguous, in page-locked memory when large)."""
    if t.numel() * t.element_size() < _STAGE_MIN_BYTES:
        return t.cpu().numpy()
    out = torch.empty(tuple(t.shape), dtype=t.dtype, pin_memory=True)
    out.copy_(t, non_blocking=True)
    torch.cuda.current_stream(t.device).synchronize()
    return out.numpy()
