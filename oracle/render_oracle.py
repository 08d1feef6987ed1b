"""CPU restatement of the headless renderer (TEST INFRASTRUCTURE).

Follows the frame the reference draws: ViewPort::coords_to_pos_on_viewport
(src/Graphics/lib/ViewPort/src/ViewPort.cpp:90-93), GL points of the body
diameter clipped to circles by the body shader (src/Graphics/src/
Graphics.cpp:20-26, drawn at :122-128), BODY_COLOR (255, 255, 255, 120)
(src/common_lib/Constants/include/Constants/Constants.hpp:39) alpha-blended
over black.  The GL stack cannot run on this machine or the GPU boxes, so the
coverage and blending rules are the ones the CUDA renderer states
(n-body-2d_b200/csrc/k_render.cu), restated here in float32 numpy with the
same operation order; parity with it is exact.
"""
from __future__ import annotations

import math

import numpy as np

F32 = np.float32


def blend_table() -> np.ndarray:
    """8-bit value after k blends of white at alpha 120/255 over black."""
    t = np.zeros(256, dtype=np.uint8)
    c = 0.0
    for k in range(256):
        t[k] = int(c)
        c = math.floor(120.0 + c * 135.0 / 255.0 + 0.5)
    return t


def coverage(pos, x, y, width, height, res_x, res_y, diam) -> np.ndarray:
    """Coverings per pixel, [res_y, res_x] uint32."""
    pos = np.asarray(pos, dtype=np.float64)
    count = np.zeros((res_y, res_x), dtype=np.uint32)
    px = F32(res_x) * ((pos[:, 0] - x) / width).astype(F32)
    py = F32(res_y) * ((pos[:, 1] - y) / height).astype(F32)
    d = F32(diam)
    half = d * F32(0.5)
    for b in range(pos.shape[0]):
        x0, x1 = px[b] - half, px[b] + half
        y0, y1 = py[b] - half, py[b] + half
        if not (x1 > 0 and y1 > 0 and x0 < res_x and y0 < res_y):
            continue
        i0, i1 = max(0, math.floor(x0) - 1), min(res_x - 1, math.ceil(x1) + 1)
        j0, j1 = max(0, math.floor(y0) - 1), min(res_y - 1, math.ceil(y1) + 1)
        for j in range(j0, j1 + 1):
            cy = F32(j) + F32(0.5)
            if not (y0 <= cy < y1):
                continue
            for i in range(i0, i1 + 1):
                cx = F32(i) + F32(0.5)
                if not (x0 <= cx < x1):
                    continue
                if d > 1:
                    u = (cx - x0) / d - F32(0.5)
                    v = (cy - y0) / d - F32(0.5)
                    if u * u + v * v > F32(0.25):
                        continue
                count[j, i] += 1
    return count


def render(pos, x, y, width, height, res_x, res_y, diam) -> np.ndarray:
    """RGBA8 frame, [res_y, res_x, 4]."""
    c = blend_table()[np.minimum(coverage(pos, x, y, width, height, res_x, res_y, diam), 255)]
    out = np.empty((res_y, res_x, 4), dtype=np.uint8)
    out[..., 0] = out[..., 1] = out[..., 2] = c
    out[..., 3] = 255
    return out
