"""Camera paths and video frames of the offline package on the b200 backend.

Mirrors blackhorizon/offline/camera_path.py (``CameraKeyframe``,
``CameraPath``, ``orbit_path``: smoothstep-eased keyframe interpolation of an
orbiting camera) and blackhorizon/offline/video.py: ``downsample`` and
``frame_bloom`` run on the device (``bh_downsample``, ``bh_frame_bloom``), and
``render_frames`` renders a path with the real-time viewer's frames
(``realtime.render_frame_device``) in place of the OpenGL engine.  Writing
H.264 (``render_video``) needs the optional ``imageio`` package, as in the
reference.
"""

from __future__ import annotations

import os
from dataclasses import dataclass

import numpy
import torch

from . import _lib
from .backend import ptr, stream_handle
from .offline import FlyCamera


@dataclass
class CameraKeyframe:
    """One camera pose on the path timeline (camera_path.py:19-35): orbit
    radius, polar angle from the spin axis, unwrapped azimuth and field of
    view, all in degrees except the radius (units of M)."""

    time: float
    distance: float
    inclination_degrees: float
    azimuth_degrees: float = 0.0
    fov_degrees: float = 70.0


def _ease(u: float) -> float:
    u = min(max(u, 0.0), 1.0)
    return u * u * (3.0 - 2.0 * u)


class CameraPath:
    """Camera motion through keyframes (camera_path.py:44-95): between two
    keyframes every pose field is blended with the cubic ease of the
    normalised time; times outside the timeline clamp to its ends."""

    def __init__(self, keyframes: list[CameraKeyframe]):
        if not keyframes:
            raise ValueError("a camera path needs at least one keyframe")
        if any(b.time <= a.time for a, b in zip(keyframes, keyframes[1:])):
            raise ValueError("keyframe times must strictly increase")
        self._keyframes = list(keyframes)

    @property
    def duration(self) -> float:
        return self._keyframes[-1].time

    def pose_at(self, time: float) -> CameraKeyframe:
        first, last = self._keyframes[0], self._keyframes[-1]
        if time <= first.time:
            return first
        if time >= last.time:
            return last
        for k0, k1 in zip(self._keyframes, self._keyframes[1:]):
            if k0.time <= time <= k1.time:
                u = _ease((time - k0.time) / (k1.time - k0.time))
                mix = lambda a, b: a + (b - a) * u  # noqa: E731
                return CameraKeyframe(time, mix(k0.distance, k1.distance),
                                      mix(k0.inclination_degrees, k1.inclination_degrees),
                                      mix(k0.azimuth_degrees, k1.azimuth_degrees),
                                      mix(k0.fov_degrees, k1.fov_degrees))
        raise RuntimeError("time inside the timeline matched no segment")

    def camera_at(self, time: float) -> FlyCamera:
        """The FlyCamera at a timeline position, looking at the hole."""
        pose = self.pose_at(time)
        return FlyCamera.from_orbit(pose.distance, pose.inclination_degrees,
                                    pose.azimuth_degrees)


def orbit_path(seconds: float, distance: float, inclination_degrees: float,
               revolutions: float = 1.0, fov_degrees: float = 70.0) -> CameraPath:
    """A constant-radius sweep of ``revolutions`` turns (camera_path.py:98-119)."""
    return CameraPath([
        CameraKeyframe(0.0, distance, inclination_degrees, 0.0, fov_degrees),
        CameraKeyframe(seconds, distance, inclination_degrees, 360.0 * revolutions,
                       fov_degrees),
    ])


def _as_device(image):
    host = not isinstance(image, torch.Tensor)
    dev = torch.device("cuda", torch.cuda.current_device())
    img = torch.as_tensor(numpy.ascontiguousarray(image), device=dev) if host else image
    if img.dim() != 3 or img.shape[2] != 3 or img.dtype != torch.uint8:
        raise ValueError("image must be a (height, width, 3) uint8 array")
    return img.contiguous(), host


def downsample(image, factor: int):
    """Box-average an (h, w, 3) uint8 image by an integer factor
    (video.py:33-43); device tensor in, device tensor out, NumPy in, NumPy
    out."""
    if factor == 1:
        return image
    img, host = _as_device(image)
    h, w = int(img.shape[0]), int(img.shape[1])
    out = torch.empty((h // factor, w // factor, 3), dtype=torch.uint8, device=img.device)
    _lib.check(_lib.load().bh_downsample(ptr(img), w, h, int(factor), ptr(out),
                                         stream_handle()), "downsample")
    return out.cpu().numpy() if host else out


def frame_bloom(image, strength: float):
    """Light bloom on a display-referred frame (video.py:46-59): lifted to
    (x / 255)^2.2, bloomed above 0.55 with sigma 5, clipped and re-encoded."""
    if strength <= 0.0:
        return image
    from .post import gaussian_kernel

    img, host = _as_device(image)
    h, w = int(img.shape[0]), int(img.shape[1])
    lib = _lib.load()
    k = gaussian_kernel(5.0)
    weights = torch.as_tensor(k, device=img.device)
    ws = torch.empty(lib.bh_frame_bloom_workspace_bytes(w, h), dtype=torch.uint8,
                     device=img.device)
    out = torch.empty_like(img)
    _lib.check(lib.bh_frame_bloom(ptr(img), w, h, float(strength), ptr(weights), k.size // 2,
                                  ptr(out), ptr(ws), ws.numel(), stream_handle()), "frame_bloom")
    return out.cpu().numpy() if host else out


def render_frames(path: CameraPath, settings, width: int, height: int, fps: int,
                  supersample: int = 2, bloom_strength: float = 0.25,
                  frames_dir: str | None = None, precision: str = "mixed"):
    """Yield the 8-bit frames of a camera path as render_video makes them
    (video.py:113-134): the viewer's frame at the supersampled size, box
    downsampled, bloomed; each also written as a PNG when frames_dir is
    given.  Frames are device tensors."""
    from .imaging import save_png
    from .realtime import render_frame_device

    if frames_dir:
        os.makedirs(frames_dir, exist_ok=True)
    n_frames = max(2, int(round(path.duration * fps)))
    for index in range(n_frames):
        t = index / fps
        settings.fov_degrees = path.pose_at(t).fov_degrees
        frame = render_frame_device(settings, path.camera_at(t), width * supersample,
                                    height * supersample, precision=precision)
        frame = frame_bloom(downsample(frame, supersample), bloom_strength)
        if frames_dir:
            save_png(frame.cpu().numpy(), os.path.join(frames_dir, f"frame_{index:05d}.png"))
        yield frame


def render_video(path: CameraPath, settings, width: int, height: int, fps: int, output: str,
                 supersample: int = 2, bloom_strength: float = 0.25,
                 frames_dir: str | None = None, progress: bool = True) -> int:
    """Render a camera path to an H.264 video (video.py:62-143); needs the
    optional imageio package.  Returns the number of frames."""
    try:
        import imageio
    except ImportError as error:
        raise RuntimeError("video encoding needs the optional imageio package") from error
    writer = imageio.get_writer(output, fps=fps, codec="libx264", quality=8)
    count = 0
    try:
        for frame in render_frames(path, settings, width, height, fps, supersample,
                                   bloom_strength, frames_dir):
            writer.append_data(frame.cpu().numpy())
            count += 1
    finally:
        writer.close()
    return count


__all__ = ["CameraKeyframe", "CameraPath", "orbit_path", "downsample", "frame_bloom",
           "render_frames", "render_video"]
