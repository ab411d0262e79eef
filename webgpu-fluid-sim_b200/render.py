"""Renderer -- the reference's density renderer (src/renderer.ts:1-329),
headless, over the engine's C ABI (bh_renderer_*).

Method names, argument meaning and camera arithmetic follow renderer.ts:
``resizeCanvasToDisplaySize`` (here with an explicit canvas size),
``panCamera`` / ``zoomCamera`` in canvas pixels, ``canvasPxToWorld`` /
``deltaPxToDeltaWorld``, ``getCommands(numBodies)`` returning the frame's
work, which ``submit`` enqueues on the simulation's stream.  Instead of a
swapchain the frame lands in two device buffers (FP32 density and RGBA8
image, display orientation) that ``readDensity`` / ``readImage`` copy out and
``write_ppm`` saves as a binary PPM.  ``rebindSimBuffers`` and
``setNumBodies`` keep their names but have nothing to do: the renderer reads
the simulation's current body buffers at every frame.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


class RenderCommand:
    """The work of one frame (renderer.ts:293-329); submit() enqueues it."""

    def __init__(self, renderer: "Renderer"):
        self._r = renderer

    def submit(self) -> None:
        self._r.frame()


class Renderer:
    def __init__(self, sim, width: int, height: int):
        self._lib = _lib.load()
        self.sim = sim
        h = ctypes.c_void_p()
        _lib.check(self._lib.bh_renderer_create(sim._h, int(width), int(height), ctypes.byref(h)))
        self._h = h
        self.width, self.height = int(width), int(height)

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.bh_renderer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, status: int) -> None:
        if status != _lib.BH_OK:
            msg = self._lib.bh_renderer_last_error(self._h) or b""
            raise _lib.BhError(status, msg.decode(errors="replace") or f"bh status {status}")

    # -- reference API ------------------------------------------------------
    def rebindSimBuffers(self, posBuffer=None, radiusMultiplierBuffer=None) -> None:
        """renderer.ts:206-216; the buffers are read at every frame."""

    def setNumBodies(self, numBodies: int) -> None:
        """renderer.ts:219-222; the body count is read at every frame."""

    def resizeCanvasToDisplaySize(self, width: int, height: int) -> None:
        """renderer.ts:225-252 for an explicit canvas size."""
        self._check(self._lib.bh_renderer_resize(self._h, int(width), int(height)))
        self.width, self.height = int(width), int(height)

    def deltaPxToDeltaWorld(self, deltaPx: float, deltaPy: float) -> tuple[float, float]:
        """renderer.ts:254-260."""
        cx, cy, hx, hy = self.camera
        return (2.0 * deltaPx) / self.width * hx, (2.0 * deltaPy) / self.height * hy

    def canvasPxToWorld(self, px: float, py: float) -> tuple[float, float]:
        """renderer.ts:262-269."""
        cx, cy, hx, hy = self.camera
        return cx + ((2.0 * px) / self.width - 1.0) * hx, cy + ((2.0 * py) / self.height - 1.0) * hy

    def panCamera(self, deltaPx: float, deltaPy: float) -> None:
        """renderer.ts:271-277."""
        self._check(self._lib.bh_renderer_pan(self._h, float(deltaPx), float(deltaPy)))

    def zoomCamera(self, zoomFactor: float, zoomCenterX: float, zoomCenterY: float) -> None:
        """renderer.ts:279-290."""
        self._check(self._lib.bh_renderer_zoom(self._h, float(zoomFactor), float(zoomCenterX),
                                               float(zoomCenterY)))

    def getCommands(self, numBodies: int | None = None) -> RenderCommand:
        """renderer.ts:293-329: clear, density pass, tone-map pass."""
        return RenderCommand(self)

    # -- engine extras ------------------------------------------------------
    @property
    def camera(self) -> tuple[float, float, float, float]:
        """(centre x, centre y, half size x, half size y) in world units."""
        c = (ctypes.c_float * 4)()
        self._check(self._lib.bh_renderer_get_camera(self._h, c))
        return tuple(float(v) for v in c)

    def setCamera(self, cx: float, cy: float, hx: float, hy: float) -> None:
        c = (ctypes.c_float * 4)(cx, cy, hx, hy)
        self._check(self._lib.bh_renderer_set_camera(self._h, c))

    def frame(self) -> None:
        self._check(self._lib.bh_renderer_frame(self._h))

    def targets(self) -> tuple[int, int]:
        """Device pointers of the density (float32) and image (RGBA8) buffers."""
        d, i = ctypes.c_void_p(), ctypes.c_void_p()
        self._check(self._lib.bh_renderer_get_targets(self._h, ctypes.byref(d), ctypes.byref(i),
                                                       None, None))
        return d.value, i.value

    def readDensity(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.float32)
        self._check(self._lib.bh_renderer_read_density(self._h, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def readImage(self) -> np.ndarray:
        out = np.empty((self.height, self.width, 4), np.uint8)
        self._check(self._lib.bh_renderer_read_image(self._h, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def write_ppm(self, path: str) -> None:
        """Save the last frame as a binary PPM (RGB)."""
        img = self.readImage()
        with open(path, "wb") as f:
            f.write(f"P6 {self.width} {self.height} 255\n".encode())
            f.write(np.ascontiguousarray(img[:, :, :3]).tobytes())
