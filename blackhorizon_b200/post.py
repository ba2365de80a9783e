"""HDR development of offline frames on the b200 backend.

Mirrors blackhorizon/offline/post.py:15-106: ``develop`` applies the exposure,
bloom (a bright pass above the threshold, blurred by a separable Gaussian with
edge padding and added back), the ACES filmic curve (Narkowicz 2015 fit) and
sRGB encoding to 8 bits, in float32 as NumPy computes it.  The per-pixel work
runs in ``bh_develop``; only the blur weights (``gaussian_kernel``) are made on
the host.
"""

from __future__ import annotations

import numpy
import torch

from . import _lib
from .backend import ptr, stream_handle


def gaussian_kernel(sigma: float) -> numpy.ndarray:
    """Normalised 1-D Gaussian truncated at three sigma (post.py:15-20)."""
    radius = max(1, int(numpy.ceil(3.0 * sigma)))
    x = numpy.arange(-radius, radius + 1, dtype=float)
    weights = numpy.exp(-0.5 * (x / sigma) ** 2)
    return weights / weights.sum()


def develop(hdr, exposure: float = 1.0, bloom_threshold: float = 1.0,
            bloom_strength: float = 0.35, bloom_sigma: float = 6.0):
    """Display-ready uint8 image (h, w, 3) from a linear HDR image (h, w, 3)
    (post.py:88-106).  A device tensor gives a device tensor; a NumPy array
    is developed on the device and returned as a NumPy array."""
    host = not isinstance(hdr, torch.Tensor)
    dev = torch.device("cuda", torch.cuda.current_device())
    img = torch.as_tensor(numpy.asarray(hdr), device=dev) if host else hdr
    if img.dim() != 3 or img.shape[2] != 3:
        raise ValueError("hdr must have shape (height, width, 3)")
    img = img.to(torch.float32).contiguous()
    height, width = int(img.shape[0]), int(img.shape[1])
    out = torch.empty((height, width, 3), dtype=torch.uint8, device=img.device)
    lib = _lib.load()
    weights = None
    radius = 0
    ws = None
    if bloom_strength > 0.0:
        k = gaussian_kernel(bloom_sigma)
        radius = k.size // 2
        weights = torch.as_tensor(k, device=img.device)
        ws = torch.empty(lib.bh_develop_workspace_bytes(width, height), dtype=torch.uint8,
                         device=img.device)
    _lib.check(lib.bh_develop(ptr(img), width, height, float(exposure), float(bloom_threshold),
                              float(bloom_strength),
                              ptr(weights) if weights is not None else None, radius, ptr(out),
                              ptr(ws) if ws is not None else None,
                              ws.numel() if ws is not None else 0, stream_handle()),
               "develop")
    return out.cpu().numpy() if host else out
