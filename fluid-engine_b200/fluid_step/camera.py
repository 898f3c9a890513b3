"""Camera for the headless water pass: a look-at view and a Vulkan-style
perspective (right-handed, depth 0..1, NDC y down), returned as the
fe_camera the library takes (column-major inverse view-projection)."""
from __future__ import annotations

import math

import numpy as np

from . import _abi


def look_at(eye, target, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    eye, target, up = (np.asarray(v, np.float64) for v in (eye, target, up))
    f = target - eye
    f /= np.linalg.norm(f)
    s = np.cross(f, up)
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    m = np.eye(4)
    m[0, :3], m[1, :3], m[2, :3] = s, u, -f
    m[:3, 3] = -m[:3, :3] @ eye
    return m


def perspective(fov_y_deg: float, aspect: float, near: float, far: float) -> np.ndarray:
    f = 1.0 / math.tan(math.radians(fov_y_deg) / 2.0)
    m = np.zeros((4, 4))
    m[0, 0] = f / aspect
    m[1, 1] = -f                      # Vulkan: y down
    m[2, 2] = far / (near - far)
    m[2, 3] = far * near / (near - far)
    m[3, 2] = -1.0
    return m


def make_camera(eye, target, width: int, height: int, fov_y_deg: float = 60.0,
                near: float = 0.05, far: float = 100.0) -> _abi.FeCamera:
    vp = perspective(fov_y_deg, width / height, near, far) @ look_at(eye, target)
    inv = np.linalg.inv(vp).astype(np.float32)
    c = _abi.FeCamera()
    c.inv_view_proj[:] = [float(x) for x in inv.T.reshape(-1)]   # column-major
    c.camera_pos[:] = [float(x) for x in eye]
    c.width, c.height = width, height
    return c


def gradient_sky(width: int = 256, height: int = 128) -> np.ndarray:
    """A synthetic equirectangular sky: blue-to-white with a bright band, so
    that reflection and refraction lookups vary across the image."""
    v = (np.arange(height, dtype=np.float32) + 0.5) / height
    u = (np.arange(width, dtype=np.float32) + 0.5) / width
    sky = np.zeros((height, width, 4), np.float32)
    sky[..., 0] = 0.3 + 0.6 * v[:, None]
    sky[..., 1] = 0.5 + 0.4 * v[:, None]
    sky[..., 2] = 0.9 - 0.2 * np.cos(2 * np.pi * u)[None, :]
    sky[..., 3] = 1.0
    return sky
