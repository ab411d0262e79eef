// ref_render_harness.cpp -- calls the mechanically translated fragment
// stages of the reference's render shaders (oracle/_ref/ref_density.inc,
// ref_tone_map.inc) on the CPU.
//
// TEST INFRASTRUCTURE ONLY: builds oracle/_ref/libref_render.so, used to
// write tests/golden/ref_render.npz, which pins the oracle's restatement of
// the per-pixel render math (the rasteriser and the blending are fixed-
// function stages and are not translated).
#include "wgsl_prelude.h"
#include "ref_density.inc"
#include "ref_tone_map.inc"

// density.wgsl fragment_main for a fragment at quad coordinates uv of a body
// with the given radius multiplier, under a camera of the given half size:
// the density it adds, or discarded = 1.
extern "C" float ref_density_fragment(float uvx, float uvy, float radius_multiplier,
                                      float half_x, float half_y, int* discarded) {
    ref_density::metadata.cam_half_size = wgsl::vec2f(half_x, half_y);
    ref_density::VSOut in;
    in.uv = wgsl::vec2f(uvx, uvy);
    in.radius_multiplier = radius_multiplier;
    wgsl::g_discarded = false;
    const wgsl::vec4f c = ref_density::fragment_main(in);
    *discarded = wgsl::g_discarded ? 1 : 0;
    return c.x;
}

// tone_map.wgsl fragment_main for a texel holding `density`: rgb in [0, 1].
extern "C" void ref_tone_map_fragment(float density, float* rgb) {
    wgsl::g_texel = density;
    ref_tone_map::VSOut in;
    const wgsl::vec4f c = ref_tone_map::fragment_main(in);
    rgb[0] = c.x;
    rgb[1] = c.y;
    rgb[2] = c.z;
}

extern "C" void ref_colormap(float t, float* rgb) {
    const wgsl::vec3f c = ref_tone_map::colormap(t);
    rgb[0] = c.x;
    rgb[1] = c.y;
    rgb[2] = c.z;
}
