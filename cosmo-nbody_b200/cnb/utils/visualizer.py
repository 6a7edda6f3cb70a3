"""Camera matrices and frame colouring (src/utils/visualizer.py of the reference).

The matrix code follows visualizer.py:9-112 (float32 numpy, host side).  One
extension: `get_mvp_matrix` takes an aspect ratio (width / height) for
non-square grids; the reference hard-codes 1.0 (visualizer.py:108).
"""
from __future__ import annotations

import numpy as np


def normalize(v):
    """visualizer.py:9-20."""
    norm = np.linalg.norm(v)
    return v if norm == 0 else v / norm


def look_at(eye, target, up):
    """visualizer.py:22-47: view matrix."""
    z = normalize(eye - target)
    x = normalize(np.cross(up, z))
    y = normalize(np.cross(z, x))
    view = np.identity(4, dtype=np.float32)
    view[0, :3] = x
    view[1, :3] = y
    view[2, :3] = z
    view[0, 3] = -np.dot(x, eye)
    view[1, 3] = -np.dot(y, eye)
    view[2, 3] = -np.dot(z, eye)
    return view


def perspective(fov_deg, aspect, near, far):
    """visualizer.py:50-78: perspective projection."""
    fov_rad = np.radians(fov_deg)
    f = 1.0 / np.tan(fov_rad / 2.0)
    proj = np.zeros((4, 4), dtype=np.float32)
    proj[0, 0] = f / aspect
    proj[1, 1] = f
    proj[2, 2] = (far + near) / (near - far)
    proj[2, 3] = (2 * far * near) / (near - far)
    proj[3, 2] = -1.0
    return proj


def get_mvp_matrix(step, box_center, box_size, config, aspect=1.0, device=None):
    """visualizer.py:81-112: orbiting camera, float32 proj @ view.  Returns a
    numpy [4,4] float32 array, or a torch tensor on `device`."""
    angle = step * config.ROTATION_SPEED
    radius = box_size * config.CAM_DIST_MULT
    eye = np.array([box_center[0] + radius * np.cos(angle),
                    box_center[1] + (box_size * 0.2),
                    box_center[2] + radius * np.sin(angle)], dtype=np.float32)
    target = np.array(box_center, dtype=np.float32)
    up = np.array([0, 1, 0], dtype=np.float32)
    view = look_at(eye, target, up)
    proj = perspective(config.FOV, aspect, 0.1, radius * 3.0)
    mvp = (proj @ view).astype(np.float32)
    if device is not None:
        import torch
        return torch.from_numpy(mvp).to(device)
    return mvp


def colorize_frame(grid_d):
    """visualizer.py:115-171: log1p(120 g), normalise by the maximum, gamma
    2.2, four-band colour map, x1.3, clip to [0, 1].  Works on a torch
    tensor [H, W] and returns [H, W, 3]."""
    import torch
    img = torch.log1p(grid_d * 120.0)
    img = img / (img.max() + 1e-9)
    val = torch.pow(img, 2.2)
    T1, T2, T3 = 0.6, 0.72, 0.82
    r = torch.zeros_like(val)
    g = torch.zeros_like(val)
    b = torch.zeros_like(val)
    m1 = val <= T1
    b = torch.where(m1, val / T1 * 0.8, b)
    m2 = (val > T1) & (val <= T2)
    t2 = (val - T1) / (T2 - T1)
    b = torch.where(m2, (1.0 - t2) * 0.8, b)
    g = torch.where(m2, t2 * 0.9, g)
    m3 = (val > T2) & (val <= T3)
    t3 = (val - T2) / (T3 - T2)
    g = torch.where(m3, 0.9 + t3 * 0.1, g)
    r = torch.where(m3, t3, r)
    m4 = val > T3
    t4 = (val - T3) / (1.0 - T3)
    r = torch.where(m4, torch.ones_like(val), r)
    g = torch.where(m4, 1.0 - t4, g)
    frame = torch.stack([r, g, b], dim=-1) * 1.3
    return torch.clamp(frame, 0, 1)
