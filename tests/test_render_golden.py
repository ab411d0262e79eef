"""The oracle's restatement of the render shaders against the reference's
own fragment code.

tests/golden/render_fragments.npz was written by tests/golden/make_golden.py from a
mechanical C++ translation of the fragment stages of the reference's
density.wgsl and tone_map.wgsl (oracle/_ref/libref_render.so): the density a
fragment adds (or its discard) on seeded quad coordinates, radius
multipliers and camera half sizes; the colour of r16float texels; the
colormap.  The oracle must match: the tone map and the colormap bit for bit
(the same f32 operations in the same order), the density within 2e-6
relative (the oracle, like the CUDA kernel, forms (base zoom_scale)
exp(-10 |uv|^2) where the shader forms base exp(-k r r) zoom_scale with
r = length(uv): the exponent arguments differ by about an ulp, which moves
exp's result by up to ~10 ulp where the argument nears -10) and the
same discards except within 1e-6 of the disc's edge (|uv|^2 > 1 against
length(uv) > 1).  The rasteriser and the blending are fixed-function stages
and are not part of the fixture.
"""
import os

import numpy as np
import pytest

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "render_fragments.npz")


@pytest.fixture(scope="module")
def g():
    return np.load(PATH)


def _zoom_scale(hx, hy):
    z = np.float32(max(hx, hy))
    return np.float32(1.0) / (np.float32(1.0) + np.float32(0.05) * z)


def test_density_fragment_matches_reference(orc, g):
    uv, rms, halves = g["uv"], g["radius_multipliers"], g["half_sizes"]
    dens, disc = g["density"], g["discarded"]
    checked = 0
    for a, (hx, hy) in enumerate(halves):
        zs = _zoom_scale(hx, hy)
        for b, rm in enumerate(rms):
            for c, (ux, uy) in enumerate(uv):
                w, d = orc.splat_weight(float(ux), float(uy), float(rm), float(zs))
                r = float(np.hypot(np.float64(ux), np.float64(uy)))
                if abs(r - 1.0) < 1e-6:
                    continue
                assert d == bool(disc[a, b, c]), (ux, uy)
                if not d:
                    ref = float(dens[a, b, c])
                    assert abs(w - ref) <= 2e-6 * ref, (ux, uy, rm, w, ref)
                    checked += 1
    assert checked > 10000


def test_tone_map_matches_reference_bit_for_bit(orc, g):
    for t, rgb in zip(g["texels"], g["rgb"]):
        assert np.array_equal(orc.tone_map_rgb(float(t)), rgb), t


def test_colormap_matches_reference_bit_for_bit(orc, g):
    for t, rgb in zip(g["colormap_t"], g["colormap_rgb"]):
        assert np.array_equal(orc.colormap(float(t)), rgb), t


def test_translated_fragments_still_match_where_built(orc, g):
    # Where the reference checkout and its translation exist, the fixture is
    # what the translation computes now.
    if not orc.ref_render_available():
        pytest.skip("oracle/_ref is built only where the reference checkout exists")
    uv, rms, halves = g["uv"], g["radius_multipliers"], g["half_sizes"]
    for c in range(0, len(uv), 97):
        w, d = orc.ref_density_fragment(float(uv[c, 0]), float(uv[c, 1]), float(rms[1]),
                                        float(halves[0, 0]), float(halves[0, 1]))
        assert (w, d) == (float(g["density"][0, 1, c]), bool(g["discarded"][0, 1, c]))
