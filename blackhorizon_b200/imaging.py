"""Shading traced rays into images, b200 backend.

Mirrors blackhorizon/imaging.py: ``celestial_checkerboard`` (imaging.py:27-50),
``render_image`` (imaging.py:53-91) and ``save_png`` (imaging.py:94-96).  The
shading runs on the device (libbh_b200 ``bh_render_image``), where the traced
states are, so only the 3-byte pixels cross to the host.  ``render_image``
returns a NumPy array like the reference; ``render_image_device`` keeps the
image on the device.
"""

from __future__ import annotations

import numpy
import torch

from . import _lib
from .backend import Array, ptr, stream_handle, to_device_f64
from .kerr import KerrSpacetime


def celestial_checkerboard(directions: Array, cells: int = 12) -> Array:
    """Checkerboard colours (n, 3) uint8 of unit directions (n, 3) on the
    celestial sphere; NumPy in, NumPy out, device tensor in, device out."""
    d, host = to_device_f64(directions, "directions")
    if d.dim() != 2 or d.shape[1] != 3:
        raise ValueError("directions must have shape (n, 3)")
    n = d.shape[0]
    out = torch.empty((n, 3), dtype=torch.uint8, device=d.device)
    _lib.check(_lib.load().bh_celestial_checkerboard(ptr(d), n, int(cells), ptr(out),
                                                     stream_handle()),
               "celestial_checkerboard")
    return out.cpu().numpy() if host is not None else out


def render_image_device(spacetime: KerrSpacetime, result, width: int, height: int,
                        cells: int = 12) -> torch.Tensor:
    """The image of a TraceResult as a (height, width, 3) uint8 device tensor.

    ``result.states`` and ``result.status`` hold height * width rays in
    row-major pixel order (imaging.py:73-76); ``spacetime.spin`` may be an
    (n,) array of per-ray spins."""
    n = int(width) * int(height)
    states, _ = to_device_f64(result.states, "states")
    status = result.status
    if not (isinstance(status, torch.Tensor) and status.is_cuda):
        status = torch.as_tensor(numpy.asarray(status), device=states.device)
    status = status.to(torch.int32).contiguous()
    if states.shape[0] != n or status.shape[0] != n:
        raise ValueError("result size does not match image dimensions")
    spins = None
    spin = spacetime.spin
    if numpy.ndim(spin) != 0 or isinstance(spin, torch.Tensor):
        spins, _ = to_device_f64(spin, "spin")
        spin = 0.0
    out = torch.empty((int(height), int(width), 3), dtype=torch.uint8, device=states.device)
    _lib.check(_lib.load().bh_render_image(float(spacetime.mass), float(spin), ptr(spins),
                                           ptr(states), ptr(status), n, int(cells), ptr(out),
                                           stream_handle()), "render_image")
    return out


def render_image(spacetime: KerrSpacetime, result, width: int, height: int) -> numpy.ndarray:
    """Convert a TraceResult into an RGB image array (height, width, 3) uint8
    (imaging.py:53-91)."""
    return render_image_device(spacetime, result, width, height).cpu().numpy()


def save_png(image: numpy.ndarray, path: str) -> None:
    """Write an RGB uint8 image array of shape (h, w, 3) to a PNG file
    (imaging.py:94-96; needs Pillow)."""
    from PIL import Image

    if isinstance(image, torch.Tensor):
        image = image.cpu().numpy()
    Image.fromarray(numpy.ascontiguousarray(image), mode="RGB").save(path)
