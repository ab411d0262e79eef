// render.cu -- headless density render: the two passes of the reference's
// Renderer.getCommands() (src/renderer.ts:293-329) as CUDA kernels.
//
// Pass 1, density (density.wgsl:39-97).  The reference draws one instanced
// quad per body, 2 * radiusMultiplier pixels in radius around the body's
// screen position, and its fragment shader adds
//     base * exp(-10 r^2) * zoom_scale,   r = |uv| <= 1 (else discard),
// (evaluated here as (base * zoom_scale) * exp(-10 |uv|^2), uv scaled by
// 1 / radius, so each pixel costs one hardware exponential),
//     base = 0.1 if radiusMultiplier > 1 else 0.02,
//     zoom_scale = 1 / (1 + 0.05 max(half size x, half size y))
// into an r16float target with additive blending.  Here one warp takes 32
// bodies; for each of them in turn its lanes stride over the pixels of the
// body's bounding square and add the weight of every pixel centre inside
// the disc with a fire-and-forget float atomic into an FP32 buffer (which
// lives in L2 for any screen size: 8 MB at 1920 x 1080).
//
// Pass 2, tone map (tone_map.wgsl:57-84): per pixel, the density rounded to
// FP16 (the reference samples an r16float texture at its texel centres, so
// the sample is the stored value), x = 8 d, Reinhard x / (1 + x), gamma
// 1/2.2, then the four-stop colormap (tone_map.wgsl:24-46), written as RGBA8
// with unorm round-to-nearest (alpha 255: the tone-map blend state of
// renderer.ts:129-131 over a cleared opaque canvas leaves colour unchanged).
//
// Orientation: both buffers are in display order, row 0 at the top.  The
// reference's density texture is upside down relative to the screen (its
// tone-map pass samples uv.y = ndc.y / 2 + 1/2, flipping it back), so its
// canvas pixel (px, py) shows world canvasPxToWorld(px, py) (renderer.ts:
// 262-269): world y grows downwards.  The same holds here.
#include <cuda_fp16.h>

#include <cmath>
#include <cstring>
#include <string>

#include "bh.h"
#include "bh_internal.cuh"

namespace bh {

bool sim_body_view(const bh_sim* s, BodyView* out);
void set_global_error(const std::string& msg);

struct RenderParams {
    float cx, cy, hx, hy;  // camera centre and half size (world units)
    uint32_t w, h;         // canvas size in pixels
};

constexpr int kSplatThreads = 256;
constexpr int kToneThreads = 256;

// density.wgsl:39-97, one warp per 32 bodies.  Each lane sets up its own
// body once (centre and radius in pixels, pixel bounds, weight) and the warp
// then splats the 32 bodies one after the other, the setup of each shuffled
// from its lane.  The lanes cover the body's pixel rectangle in 8 x 4 tiles,
// with integer pixel indices and exactly representable float pixel centres
// stepped by additions: no division or conversion per pixel, one hardware
// exponential per covered pixel.
__global__ void __launch_bounds__(kSplatThreads)
splat_kernel(const float2* __restrict__ pos, const float* __restrict__ radius_mul, uint32_t n,
             const RenderParams P, float* __restrict__ density) {
    const unsigned FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const float W = (float)P.w, H = (float)P.h;
    // zoom compensation (density.wgsl:86-88)
    const float zoom = fmaxf(P.hx, P.hy);
    const float zoom_scale = __fdiv_rn(1.0f, __fadd_rn(1.0f, __fmul_rn(0.05f, zoom)));
    const int tx = lane & 7, ty = lane >> 3;  // the lane's place in an 8 x 4 tile
    for (uint32_t base = warp * 32u; base < n; base += nwarps * 32u) {
        // ---- this lane's body ----
        float cpx = 0.0f, cpy = 0.0f, inv_r = 0.0f, bw = 0.0f;
        int ia = 0, ib = -1, ja = 0, jb = -1;  // pixel rectangle [ia, ib] x [ja, jb]
        if (base + (uint32_t)lane < n) {
            const float2 p = __ldg(&pos[base + lane]);
            const float rm = __ldg(&radius_mul[base + lane]);
            // vertex stage (density.wgsl:60-70): centre in NDC, radius in pixels
            const float cnx = __fdiv_rn(__fsub_rn(p.x, P.cx), P.hx);
            const float cny = __fdiv_rn(__fsub_rn(p.y, P.cy), P.hy);
            const float R = __fmul_rn(2.0f, rm);
            // centre in display pixel coordinates: (ndc + 1) / 2 * size
            cpx = __fmul_rn(__fmul_rn(__fadd_rn(cnx, 1.0f), 0.5f), W);
            cpy = __fmul_rn(__fmul_rn(__fadd_rn(cny, 1.0f), 0.5f), H);
            // a body without a finite centre or radius draws nothing (the
            // rasteriser drops a quad with non-finite vertices)
            if (isfinite(cpx) && isfinite(cpy) && R > 0.0f && isfinite(R)) {
                // pixel centres i + 1/2 within [c - R, c + R], clipped to the canvas
                const float i0 = fmaxf(ceilf(cpx - R - 0.5f), 0.0f);
                const float i1 = fminf(floorf(cpx + R - 0.5f), W - 1.0f);
                const float j0 = fmaxf(ceilf(cpy - R - 0.5f), 0.0f);
                const float j1 = fminf(floorf(cpy + R - 0.5f), H - 1.0f);
                if (i0 <= i1 && j0 <= j1) {
                    ia = (int)i0; ib = (int)i1; ja = (int)j0; jb = (int)j1;
                }
            }
            inv_r = __frcp_rn(R);
            bw = __fmul_rn(rm > 1.0f ? 0.1f : 0.02f, zoom_scale);  // density.wgsl:90-95
        }
        const int cnt = (n - base) < 32u ? (int)(n - base) : 32;
        for (int k = 0; k < cnt; ++k) {
            const int kia = __shfl_sync(FULL, ia, k), kib = __shfl_sync(FULL, ib, k);
            const int kja = __shfl_sync(FULL, ja, k), kjb = __shfl_sync(FULL, jb, k);
            if (kia > kib) continue;  // nothing on screen (uniform)
            const float kcx = __shfl_sync(FULL, cpx, k), kcy = __shfl_sync(FULL, cpy, k);
            const float kir = __shfl_sync(FULL, inv_r, k), kbw = __shfl_sync(FULL, bw, k);
            float yc = (float)(kja + ty) + 0.5f;
            for (int j = kja + ty; j <= kjb; j += 4, yc = __fadd_rn(yc, 4.0f)) {
                // uv and r^2 = |uv|^2; discard outside the disc (density.wgsl:73-78)
                const float uy = __fmul_rn(__fsub_rn(yc, kcy), kir);
                const float uy2 = __fmul_rn(uy, uy);
                float* row = density + (size_t)j * P.w;
                float xc = (float)(kia + tx) + 0.5f;
                for (int i = kia + tx; i <= kib; i += 8, xc = __fadd_rn(xc, 8.0f)) {
                    const float ux = __fmul_rn(__fsub_rn(xc, kcx), kir);
                    const float r2 = __fadd_rn(__fmul_rn(ux, ux), uy2);
                    if (r2 > 1.0f) continue;
                    // w = exp(-k r^2), k = 10 (density.wgsl:81-82): the hardware
                    // exponential, relative error ~1e-6 over r^2 in [0, 1]
                    atomicAdd(&row[i], __fmul_rn(kbw, __expf(__fmul_rn(-10.0f, r2))));
                }
            }
        }
    }
}

// tone_map.wgsl:24-46
__device__ __forceinline__ float mix1(float a, float b, float t) {
    return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, t)), __fmul_rn(b, t));
}

__device__ __forceinline__ float3 colormap(float t) {
    const float x = fminf(fmaxf(t, 0.0f), 1.0f);
    if (x < 0.33f) {
        const float a = __fdiv_rn(x, 0.33f);
        return make_float3(mix1(0.0f, 0.10f, a), mix1(0.0f, 0.20f, a), mix1(0.0f, 0.90f, a));
    } else if (x < 0.66f) {
        const float a = __fdiv_rn(__fsub_rn(x, 0.33f), 0.33f);
        return make_float3(mix1(0.10f, 0.20f, a), mix1(0.20f, 0.90f, a), mix1(0.90f, 0.90f, a));
    }
    const float a = __fdiv_rn(__fsub_rn(x, 0.66f), 0.34f);
    return make_float3(mix1(0.20f, 1.0f, a), mix1(0.90f, 1.0f, a), mix1(0.90f, 1.0f, a));
}

__device__ __forceinline__ unsigned char unorm8(float c) {
    return (unsigned char)__float2uint_rn(__fmul_rn(fminf(fmaxf(c, 0.0f), 1.0f), 255.0f));
}

// tone_map.wgsl:63-84, one thread per pixel.
__global__ void __launch_bounds__(kToneThreads)
tone_map_kernel(const float* __restrict__ density, uint32_t pixels, uchar4* __restrict__ image) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pixels) return;
    const float d = __half2float(__float2half_rn(__ldg(&density[p])));  // r16float texel
    const float x = __fmul_rn(8.0f, d);                                  // exposure 8
    const float mapped = __fdiv_rn(x, __fadd_rn(1.0f, x));               // Reinhard
    const float g = powf(fminf(fmaxf(mapped, 0.0f), 1.0f), (float)(1.0 / 2.2));
    const float3 c = colormap(g);
    image[p] = make_uchar4(unorm8(c.x), unorm8(c.y), unorm8(c.z), 255);
}

}  // namespace bh

// ---- C ABI ------------------------------------------------------------------

struct bh_renderer {
    bh_sim* sim = nullptr;
    int device = 0;
    uint32_t width = 0, height = 0;
    // camera in double precision like the reference's JS numbers; rounded to
    // f32 when a frame is enqueued (renderer.ts:171-185 writes a Float32Array)
    double cam[4] = {0.0, 0.0, 10.0, 10.0};
    float* density = nullptr;
    uint8_t* image = nullptr;
    std::string err;
};

static int rfail(bh_renderer* r, int code, const std::string& msg) {
    if (r) r->err = msg;
    bh::set_global_error(msg);
    return code;
}

static int rcuda(bh_renderer* r, cudaError_t e, const char* what) {
    const int code = (e == cudaErrorMemoryAllocation) ? BH_ERR_OUT_OF_MEMORY : BH_ERR_CUDA;
    return rfail(r, code, std::string(what) + ": " + cudaGetErrorString(e));
}

// Largest canvas: width * height <= 2^28 pixels (index arithmetic in 32 bits).
static constexpr uint64_t kMaxPixels = 1ull << 28;

static int alloc_targets(bh_renderer* r, uint32_t w, uint32_t h) {
    if (w == 0 || h == 0 || (uint64_t)w * h > kMaxPixels)
        return rfail(r, BH_ERR_INVALID_ARGUMENT, "renderer: canvas must be 1..2^28 pixels");
    cudaError_t e = cudaSetDevice(r->device);
    if (e != cudaSuccess) return rcuda(r, e, "cudaSetDevice");
    if (r->density) cudaFree(r->density);
    r->density = nullptr;
    r->image = nullptr;
    const size_t px = (size_t)w * h;
    void* mem = nullptr;
    e = cudaMalloc(&mem, px * sizeof(float) + px * 4);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return rcuda(r, e, "cudaMalloc(render targets)");
    }
    r->density = static_cast<float*>(mem);
    r->image = reinterpret_cast<uint8_t*>(r->density + px);
    r->width = w;
    r->height = h;
    // resizeCanvasToDisplaySize (renderer.ts:242-246): keep the vertical half
    // size, match the horizontal one to the aspect ratio
    r->cam[2] = r->cam[3] * ((double)w / (double)h);
    return BH_OK;
}

extern "C" int bh_renderer_create(bh_sim* sim, uint32_t width, uint32_t height, bh_renderer** out) {
    if (!sim || !out) return rfail(nullptr, BH_ERR_INVALID_ARGUMENT, "bh_renderer_create: null argument");
    bh::BodyView v;
    bh::sim_body_view(sim, &v);
    bh_renderer* r = new bh_renderer();
    r->sim = sim;
    r->device = v.device;
    const int st = alloc_targets(r, width, height);
    if (st != BH_OK) {
        delete r;
        return st;
    }
    *out = r;
    return BH_OK;
}

extern "C" int bh_renderer_destroy(bh_renderer* r) {
    if (!r) return BH_OK;
    if (r->density) {
        cudaSetDevice(r->device);
        cudaFree(r->density);
    }
    delete r;
    return BH_OK;
}

extern "C" int bh_renderer_resize(bh_renderer* r, uint32_t width, uint32_t height) {
    if (!r) return rfail(nullptr, BH_ERR_INVALID_ARGUMENT, "null renderer");
    bh::BodyView v;
    bh::sim_body_view(r->sim, &v);
    cudaSetDevice(r->device);
    cudaStreamSynchronize(v.stream);  // the old targets may still be in use
    return alloc_targets(r, width, height);
}

// renderer.ts:254-260 deltaPxToDeltaWorld, :271-277 panCamera
extern "C" int bh_renderer_pan(bh_renderer* r, float delta_px, float delta_py) {
    if (!r) return rfail(nullptr, BH_ERR_INVALID_ARGUMENT, "null renderer");
    const double dwx = (2.0 * delta_px) / r->width * r->cam[2];
    const double dwy = (2.0 * delta_py) / r->height * r->cam[3];
    r->cam[0] -= dwx;
    r->cam[1] -= dwy;
    return BH_OK;
}

// renderer.ts:262-269 canvasPxToWorld, :279-290 zoomCamera
extern "C" int bh_renderer_zoom(bh_renderer* r, float zoom_factor, float center_px, float center_py) {
    if (!r) return rfail(nullptr, BH_ERR_INVALID_ARGUMENT, "null renderer");
    const double wx = r->cam[0] + ((2.0 * center_px) / r->width - 1.0) * r->cam[2];
    const double wy = r->cam[1] + ((2.0 * center_py) / r->height - 1.0) * r->cam[3];
    r->cam[2] *= zoom_factor;
    r->cam[3] *= zoom_factor;
    r->cam[0] = r->cam[0] + (wx - r->cam[0]) * (1.0 - zoom_factor);
    r->cam[1] = r->cam[1] + (wy - r->cam[1]) * (1.0 - zoom_factor);
    return BH_OK;
}

extern "C" int bh_renderer_set_camera(bh_renderer* r, const float camera[4]) {
    if (!r || !camera) return rfail(r, BH_ERR_INVALID_ARGUMENT, "null argument");
    if (!(camera[2] > 0.0f) || !(camera[3] > 0.0f))
        return rfail(r, BH_ERR_INVALID_ARGUMENT, "camera half sizes must be positive");
    for (int k = 0; k < 4; ++k) r->cam[k] = camera[k];
    return BH_OK;
}

extern "C" int bh_renderer_get_camera(bh_renderer* r, float camera[4]) {
    if (!r || !camera) return rfail(r, BH_ERR_INVALID_ARGUMENT, "null argument");
    for (int k = 0; k < 4; ++k) camera[k] = (float)r->cam[k];
    return BH_OK;
}

extern "C" int bh_renderer_frame(bh_renderer* r) {
    if (!r) return rfail(nullptr, BH_ERR_INVALID_ARGUMENT, "null renderer");
    bh::BodyView v;
    bh::sim_body_view(r->sim, &v);
    cudaError_t e = cudaSetDevice(r->device);
    if (e != cudaSuccess) return rcuda(r, e, "cudaSetDevice");
    const size_t px = (size_t)r->width * r->height;
    e = cudaMemsetAsync(r->density, 0, px * sizeof(float), v.stream);  // loadOp "clear"
    if (e != cudaSuccess) return rcuda(r, e, "cudaMemsetAsync(density)");
    bh::RenderParams P;
    P.cx = (float)r->cam[0];
    P.cy = (float)r->cam[1];
    P.hx = (float)r->cam[2];
    P.hy = (float)r->cam[3];
    P.w = r->width;
    P.h = r->height;
    if (v.n > 0) {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, r->device);
        uint32_t blocks = (uint32_t)sms * 8u;
        const uint32_t need = (v.n + bh::kSplatThreads - 1) / bh::kSplatThreads;
        if (blocks > need) blocks = need;
        bh::splat_kernel<<<blocks, bh::kSplatThreads, 0, v.stream>>>(v.pos, v.radius, v.n, P,
                                                                     r->density);
    }
    bh::tone_map_kernel<<<(uint32_t)((px + bh::kToneThreads - 1) / bh::kToneThreads),
                          bh::kToneThreads, 0, v.stream>>>(r->density, (uint32_t)px,
                                                           reinterpret_cast<uchar4*>(r->image));
    e = cudaGetLastError();
    if (e != cudaSuccess) return rcuda(r, e, "render kernels launch");
    return BH_OK;
}

extern "C" int bh_renderer_get_targets(bh_renderer* r, float** density, uint8_t** image,
                                       uint32_t* width, uint32_t* height) {
    if (!r) return rfail(nullptr, BH_ERR_INVALID_ARGUMENT, "null renderer");
    if (density) *density = r->density;
    if (image) *image = r->image;
    if (width) *width = r->width;
    if (height) *height = r->height;
    return BH_OK;
}

static int read_target(bh_renderer* r, const void* src, void* host, size_t bytes) {
    if (!r || !host) return rfail(r, BH_ERR_INVALID_ARGUMENT, "null argument");
    bh::BodyView v;
    bh::sim_body_view(r->sim, &v);
    cudaSetDevice(r->device);
    cudaError_t e = cudaMemcpyAsync(host, src, bytes, cudaMemcpyDeviceToHost, v.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(v.stream);
    if (e != cudaSuccess) return rcuda(r, e, "render target read");
    return BH_OK;
}

extern "C" int bh_renderer_read_density(bh_renderer* r, float* host) {
    if (!r) return rfail(nullptr, BH_ERR_INVALID_ARGUMENT, "null renderer");
    return read_target(r, r->density, host, (size_t)r->width * r->height * sizeof(float));
}

extern "C" int bh_renderer_read_image(bh_renderer* r, uint8_t* host) {
    if (!r) return rfail(nullptr, BH_ERR_INVALID_ARGUMENT, "null renderer");
    return read_target(r, r->image, host, (size_t)r->width * r->height * 4);
}

extern "C" const char* bh_renderer_last_error(bh_renderer* r) {
    return r ? r->err.c_str() : "";
}
