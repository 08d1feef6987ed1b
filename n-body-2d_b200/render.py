"""Headless rendering of the bodies (nb_render) and the reference's viewport.

ViewPort mirrors src/Graphics/lib/ViewPort/src/ViewPort.cpp: a world
rectangle of resolution x pixel_scale centred on the origin at start-up, with
zoom about the cursor and pan by pixels; coords_to_pos_on_viewport is the
mapping the renderer applies on the GPU.  write_png stores an RGBA frame
without any imaging library.
"""
from __future__ import annotations

import ctypes as C
import struct
import zlib
from dataclasses import dataclass

import numpy as np

from ._lib import NbView

ZOOM_FACTOR = 1.1  # Constants::Graphics::ZOOM_FACTOR


@dataclass
class ViewPort:
    res_x: int
    res_y: int
    pixel_scale: float
    x: float = 0.0
    y: float = 0.0
    width: float = 0.0
    height: float = 0.0

    def __post_init__(self):
        # init_rect (ViewPort.cpp:11-15): centred on the origin
        self._size()
        self.x = -self.width / 2.0
        self.y = -self.height / 2.0

    def _size(self) -> None:
        self.width = self.res_x * self.pixel_scale
        self.height = self.res_y * self.pixel_scale

    def zoom(self, zoom_in: bool, cursor_x: float, cursor_y: float) -> None:
        """ViewPort::zoom (ViewPort.cpp:21-47), without the pixel-scale limits."""
        norm = 1.0 / ZOOM_FACTOR
        fx, fy = np.float32(cursor_x) / np.float32(self.res_x), np.float32(cursor_y) / np.float32(self.res_y)
        if zoom_in:
            self.pixel_scale *= norm
            self.x += float(fx) * self.width * (1 - norm)
            self.y += float(fy) * self.height * (1 - norm)
            self._size()
        else:
            self.pixel_scale /= norm
            self._size()
            self.x -= float(fx) * self.width * (1 - norm)
            self.y -= float(fy) * self.height * (1 - norm)

    def pan(self, dx_pixels: float, dy_pixels: float) -> None:
        """ViewPort::pan (ViewPort.cpp:54-57)."""
        self.x += float(np.float32(dx_pixels) / np.float32(self.res_x)) * self.width
        self.y += float(np.float32(dy_pixels) / np.float32(self.res_y)) * self.height

    def coords_to_pos_on_viewport(self, pos: np.ndarray) -> np.ndarray:
        """ViewPort.cpp:90-93: FP64 relative position, rounded to float, times
        the float resolution."""
        pos = np.asarray(pos, dtype=np.float64)
        rel_x = ((pos[..., 0] - self.x) / self.width).astype(np.float32)
        rel_y = ((pos[..., 1] - self.y) / self.height).astype(np.float32)
        return np.stack([np.float32(self.res_x) * rel_x, np.float32(self.res_y) * rel_y], axis=-1)

    def as_view(self, point_diameter: float = 1.0) -> NbView:
        return NbView(self.x, self.y, self.width, self.height, self.res_x, self.res_y,
                      float(point_diameter), 0)


def write_png(path, rgba: np.ndarray) -> None:
    """8-bit RGBA PNG (filter 0 on every row)."""
    rgba = np.ascontiguousarray(rgba, dtype=np.uint8)
    h, w = rgba.shape[:2]
    raw = b"".join(b"\x00" + rgba[r].tobytes() for r in range(h))

    def chunk(kind: bytes, data: bytes) -> bytes:
        body = kind + data
        return struct.pack(">I", len(data)) + body + struct.pack(">I", zlib.crc32(body) & 0xFFFFFFFF)

    png = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0))
    png += chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b"")
    with open(path, "wb") as f:
        f.write(png)
