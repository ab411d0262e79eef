"""Density render (the reference's Renderer, src/renderer.ts) against the
oracle's restatement of density.wgsl and tone_map.wgsl.

CPU: known answers of the restated shader math.  GPU (marked): the CUDA
render path through the C ABI against the oracle on the same bodies and
camera.  Tolerances: density per pixel |d_gpu - d_ref| <= 1e-5 d_ref + 1e-9
(FP32 atomics in any order vs an FP64 sum in body order; expf vs the C
library's expf); image bytes: the tone map of the same density agrees to the
byte except where powf rounds across a quantisation step (<= 0.1% of bytes,
never by more than 1).
"""
import math

import numpy as np
import pytest

CAM = np.array([0.0, 0.0, 10.0, 10.0], np.float32)


def pixel_centre_world(i, j, cam, w, h):
    # canvasPxToWorld (renderer.ts:262-269) at the pixel centre
    return (cam[0] + (2.0 * (i + 0.5) / w - 1.0) * cam[2],
            cam[1] + (2.0 * (j + 0.5) / h - 1.0) * cam[3])


# ---- CPU: the restated shader math --------------------------------------------

def test_colormap_stops(orc):
    # tone_map.wgsl:24-46: black, (0.1, 0.2, 0.9) at 0.33, (0.2, 0.9, 0.9) at 0.66, white at 1
    np.testing.assert_allclose(orc.colormap(0.0), [0, 0, 0])
    np.testing.assert_allclose(orc.colormap(0.33), [0.10, 0.20, 0.90], atol=1e-6)
    np.testing.assert_allclose(orc.colormap(0.66), [0.20, 0.90, 0.90], atol=1e-6)
    np.testing.assert_allclose(orc.colormap(1.0), [1, 1, 1], atol=1e-6)
    np.testing.assert_allclose(orc.colormap(0.165), [0.05, 0.10, 0.45], atol=1e-6)
    np.testing.assert_allclose(orc.colormap(-3.0), orc.colormap(0.0))
    np.testing.assert_allclose(orc.colormap(7.0), orc.colormap(1.0))


def test_single_body_disc(orc):
    # A body at the centre of pixel (32, 32) of a 64 x 64 canvas: radius 2 px,
    # 13 pixel centres within the disc, weights base exp(-10 r^2) zoom_scale.
    w = h = 64
    x, y = pixel_centre_world(32, 32, CAM, w, h)
    d = orc.render_density(CAM, w, h, np.array([[x, y]], np.float32), np.array([1.0], np.float32))
    zoom_scale = 1.0 / (1.0 + 0.05 * 10.0)
    assert (d > 0).sum() == 13
    for (di, dj) in [(0, 0), (1, 0), (0, 1), (1, 1), (2, 0), (0, -2), (-1, -1)]:
        r = math.hypot(di, dj) / 2.0
        np.testing.assert_allclose(d[32 + dj, 32 + di], 0.02 * math.exp(-10 * r * r) * zoom_scale,
                                   rtol=1e-6)


def test_large_radius_uses_bright_base_and_wider_disc(orc):
    w = h = 128
    x, y = pixel_centre_world(64, 64, CAM, w, h)
    d = orc.render_density(CAM, w, h, np.array([[x, y]], np.float32), np.array([5.0], np.float32))
    # radius 10 px: pixel centres with |offset| <= 10
    offs = [(a, b) for a in range(-10, 11) for b in range(-10, 11) if a * a + b * b <= 100]
    assert (d > 0).sum() == len(offs)
    np.testing.assert_allclose(d[64, 64], 0.1 / 1.5, rtol=1e-6)  # base 0.1 when rm > 1


def test_zoom_scale_and_offscreen_bodies(orc):
    w = h = 32
    cam = np.array([0.0, 0.0, 40.0, 20.0], np.float32)
    x, y = pixel_centre_world(16, 16, cam, w, h)
    pos = np.array([[x, y], [1e6, 0.0], [np.nan, 0.0], [x, y]], np.float32)
    d = orc.render_density(cam, w, h, pos, np.array([1, 1, 1, np.inf], np.float32))
    assert np.isfinite(d).all()
    np.testing.assert_allclose(d.max(), 0.02 / (1.0 + 0.05 * 40.0), rtol=1e-6)
    assert (d > 0).sum() == 13


def test_tone_map_known_values(orc):
    dens = np.array([[0.0, 1e-3, 0.125, 1e4]], np.float32)
    img = orc.tone_map(dens)
    assert tuple(img[0, 0]) == (0, 0, 0, 255)
    assert tuple(img[0, 3]) == (255, 255, 255, 255)  # saturated
    # density 0.125: x = 1, Reinhard 1/2, gamma -> 0.5^(1/2.2) = 0.7297: last segment
    t = 0.5 ** (1 / 2.2)
    a = (t - 0.66) / 0.34
    want = [round(255 * (0.2 * (1 - a) + a)), round(255 * (0.9 * (1 - a) + a)),
            round(255 * (0.9 * (1 - a) + a))]
    assert np.abs(img[0, 2, :3].astype(int) - want).max() <= 1
    # monotone brightness along the ramp
    ramp = orc.tone_map(np.geomspace(1e-4, 10, 200, dtype=np.float32)[None, :])
    lum = ramp[0, :, :3].astype(int).sum(1)
    assert (np.diff(lum) >= 0).all()


# ---- GPU: the CUDA render path through the C ABI ------------------------------

def _frame(bh, sim, w, h, cam=None):
    r = bh.Renderer(sim, w, h)
    if cam is not None:
        r.setCamera(*cam)
    r.getCommands(sim.getNumBodies()).submit()
    return r, r.readDensity(), r.readImage()


def _compare(orc, r, dens, img, sim):
    mass, pos, vel = sim.download()
    rm = sim.read_buffer("radius_multiplier", np.float32, sim.getNumBodies())
    cam = np.array(r.camera, np.float32)
    ref = orc.render_density(cam, r.width, r.height, pos, rm)
    assert np.all(np.abs(dens - ref) <= 1e-5 * ref + 1e-9), np.abs(dens - ref).max()
    img_ref = orc.tone_map(dens)
    diff = np.abs(img.astype(int) - img_ref.astype(int))
    assert diff.max() <= 1
    assert (diff > 0).mean() <= 1e-3
    return ref


@pytest.mark.gpu
@pytest.mark.parametrize("scenario,n", [("colliding-disks", 20000), ("planetary-disk", 5000),
                                        ("two-clusters", 8000)])
def test_render_matches_oracle(bh, orc, scenario, n):
    sim = bh.Simulation(bh.Config())
    sim.setNumBodies(n)
    sim.setScenario(scenario, 4)
    r, dens, img = _frame(bh, sim, 320, 200)
    assert r.camera[2] == pytest.approx(10.0 * 320 / 200) and r.camera[3] == 10.0
    _compare(orc, r, dens, img, sim)
    assert dens.max() > 0
    r.close()
    sim.close()


@pytest.mark.gpu
def test_render_camera_pan_zoom_resize(bh, orc):
    sim = bh.Simulation(bh.Config())
    sim.setNumBodies(3000)
    sim.setScenario("default", 2)
    r = bh.Renderer(sim, 200, 100)
    # zoomCamera about the canvas centre keeps the centre; half sizes scale
    r.zoomCamera(0.5, 100, 50)
    cx, cy, hx, hy = r.camera
    assert (cx, cy) == pytest.approx((0.0, 0.0), abs=1e-6)
    assert (hx, hy) == pytest.approx((10.0, 5.0))
    # zooming about a corner pulls the centre towards it (renderer.ts:279-290)
    wx, wy = r.canvasPxToWorld(0, 0)
    r.zoomCamera(0.5, 0, 0)
    cx2, cy2, hx2, hy2 = r.camera
    assert cx2 == pytest.approx(cx + (wx - cx) * 0.5) and cy2 == pytest.approx(cy + (wy - cy) * 0.5)
    # panCamera moves the centre against the drag (renderer.ts:271-277)
    dx, dy = r.deltaPxToDeltaWorld(20, -10)
    r.panCamera(20, -10)
    assert r.camera[0] == pytest.approx(cx2 - dx) and r.camera[1] == pytest.approx(cy2 - dy)
    r.getCommands().submit()
    _compare(orc, r, r.readDensity(), r.readImage(), sim)
    # resize keeps the vertical half size and matches the aspect ratio
    r.resizeCanvasToDisplaySize(90, 60)
    assert r.camera[2] == pytest.approx(r.camera[3] * 1.5)
    r.getCommands().submit()
    dens = r.readDensity()
    assert dens.shape == (60, 90)
    _compare(orc, r, dens, r.readImage(), sim)
    # a new body count needs no rebind: the next frame reads the new buffers
    sim.setNumBodies(500)
    r.getCommands().submit()
    _compare(orc, r, r.readDensity(), r.readImage(), sim)
    r.close()
    sim.close()


@pytest.mark.gpu
def test_render_skips_offscreen_and_non_finite_bodies(bh, orc):
    sim = bh.Simulation(bh.Config())
    sim.setNumBodies(4)
    mass = np.ones(4, np.float32)
    x, y = pixel_centre_world(8, 8, CAM, 16, 16)
    pos = np.array([[x, y], [1e30, 0], [np.nan, 1.0], [0.0, -1e9]], np.float32)
    sim.upload(mass, pos, np.zeros((4, 2), np.float32))
    r, dens, img = _frame(bh, sim, 16, 16, cam=CAM)
    assert np.isfinite(dens).all()
    assert (dens > 0).sum() == 13
    assert dens[8, 8] == pytest.approx(0.02 / 1.5, rel=1e-6)
    r.close()
    sim.close()


@pytest.mark.gpu
def test_render_with_no_bodies_and_one_pixel_canvas(bh):
    sim = bh.Simulation(bh.Config())
    sim.setNumBodies(0)
    r, dens, img = _frame(bh, sim, 8, 4)
    assert (dens == 0).all() and (img[:, :, :3] == 0).all() and (img[:, :, 3] == 255).all()
    r.close()
    sim.setNumBodies(10)
    r, dens, img = _frame(bh, sim, 1, 1)
    assert dens.shape == (1, 1) and np.isfinite(dens).all()
    r.close()
    with pytest.raises(bh.BhError):
        bh.Renderer(sim, 0, 10)
    sim.close()
