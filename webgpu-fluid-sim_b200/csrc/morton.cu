// morton.cu -- bounding box, Morton encode with fused digit histograms, and
// the leapfrog opening kick + drift.
//
// Reference: lbvh.wgsl:42-69 (compute_morton_codes_main).  The quantisation
// uses round-to-nearest intrinsics so that no FMA contraction changes a bit:
//   uv = clamp((p - lo) / extent, 0, 1);  q = min(u32(uv * 65535 + 0.5), 65535)
// and the bit interleave puts x on even bits and y on odd bits
// (lbvh.wgsl:59-65).  The reference domain is lo = -1000, extent = 2000
// (lbvh.wgsl:49-53; p + 1000 and p - (-1000) round identically).
//
// Extensions: a tight bounding box for 32-bit keys, and 64-bit keys
// (32 bits per axis) over the power-of-two square [-2^(e-1), 2^(e-1)) that
// holds every body, quantised exactly as floor(p * 2^(32-e)) + 2^31.
//
// The encode kernel also builds the per-pass digit histograms that the
// onesweep sort needs, so the keys are read once for both.  Body ids are not
// written: the first sort pass generates the identity permutation
// (lbvh.wgsl:68) itself.
#include "bh_internal.cuh"

namespace bh {

// Encode grids are capped at this many 256-thread blocks per SM.  Large
// inputs want every block the SM holds (more loads in flight); small ones
// fewer, since each block flushes its digit histograms with global atomics
// at the end (measured, 4 / 8 blocks per SM: 800k bodies 0.019 / 0.024 ms,
// 16.8M 0.166 / 0.157 ms, a 49M-body ensemble 1.34 / 1.05 ms).
static int encode_blocks_per_sm(uint32_t n) { return n >= (1u << 22) ? 8 : 4; }

// ---- order-preserving float <-> uint (max-reductions with atomicMax) -----
__device__ __forceinline__ uint32_t f2ord(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

__device__ __forceinline__ uint32_t spread16(uint32_t v) {
    v &= 0xFFFFu;
    v = (v | (v << 8)) & 0x00FF00FFu;
    v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}
__device__ __forceinline__ uint64_t spread32(uint64_t v) {
    v &= 0xFFFFFFFFull;
    v = (v | (v << 16)) & 0x0000FFFF0000FFFFull;
    v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
    v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full;
    v = (v | (v << 2)) & 0x3333333333333333ull;
    v = (v | (v << 1)) & 0x5555555555555555ull;
    return v;
}

__device__ __forceinline__ uint32_t quant16(float p, float lo, float ext) {
    float u = __fdiv_rn(__fsub_rn(p, lo), ext);
    u = fminf(fmaxf(u, 0.0f), 1.0f);
    float t = __fadd_rn(__fmul_rn(u, 65535.0f), 0.5f);
    uint32_t q = __float2uint_rz(t);
    return q > 65535u ? 65535u : q;
}

__device__ __forceinline__ uint32_t quant32(float p, float scale) {
    long long q = __float2ll_rd(__fmul_rn(p, scale)) + 2147483648LL;
    q = q < 0 ? 0 : q;
    q = q > 4294967295LL ? 4294967295LL : q;
    return (uint32_t)q;
}

// ---- bounding box ---------------------------------------------------------
__device__ __forceinline__ void warp_box(float& a, float& b, float& c, float& d) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a = fmaxf(a, __shfl_xor_sync(0xFFFFFFFFu, a, o));
        b = fmaxf(b, __shfl_xor_sync(0xFFFFFFFFu, b, o));
        c = fmaxf(c, __shfl_xor_sync(0xFFFFFFFFu, c, o));
        d = fmaxf(d, __shfl_xor_sync(0xFFFFFFFFu, d, o));
    }
}

// scratch->bbox = ordered max of {-x, -y, x, y}; zeroed by the step memset.
__global__ void __launch_bounds__(256) bbox_kernel(const float4* __restrict__ pos2, uint32_t n,
                                                   StepScratch* scratch) {
    float nx = -INFINITY, ny = -INFINITY, px = -INFINITY, py = -INFINITY;
    const uint32_t pairs = n / 2;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pairs; i += gridDim.x * blockDim.x) {
        float4 v = __ldg(&pos2[i]);
        nx = fmaxf(nx, fmaxf(-v.x, -v.z));
        px = fmaxf(px, fmaxf(v.x, v.z));
        ny = fmaxf(ny, fmaxf(-v.y, -v.w));
        py = fmaxf(py, fmaxf(v.y, v.w));
    }
    if ((n & 1u) && blockIdx.x == 0 && threadIdx.x == 0) {
        float2 v = reinterpret_cast<const float2*>(pos2)[n - 1];
        nx = fmaxf(nx, -v.x); px = fmaxf(px, v.x);
        ny = fmaxf(ny, -v.y); py = fmaxf(py, v.y);
    }
    warp_box(nx, ny, px, py);
    __shared__ float s[8][4];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) { s[w][0] = nx; s[w][1] = ny; s[w][2] = px; s[w][3] = py; }
    __syncthreads();
    if (threadIdx.x < 4) {
        float m = -INFINITY;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) m = fmaxf(m, s[k][threadIdx.x]);
        atomicMax(&scratch->bbox[threadIdx.x], f2ord(m));
    }
}

void launch_bbox(const DeviceBuffers& b, cudaStream_t s) {
    if (b.n == 0) return;
    uint32_t pairs = (b.n + 1) / 2;
    int blocks = (int)((pairs + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    bbox_kernel<<<blocks, 256, 0, s>>>(reinterpret_cast<const float4*>(b.pos), b.n, b.scratch);
}

// ---- Morton encode + digit histograms --------------------------------------
struct Domain {
    float lo_x, lo_y, ext;  // 32-bit keys
    float scale;            // 64-bit keys: 2^(32-e)
};

__device__ __forceinline__ Domain read_domain(const StepScratch* sc, int domain, int key_bytes) {
    Domain d;
    d.lo_x = -1000.0f;
    d.lo_y = -1000.0f;
    d.ext = 2000.0f;
    d.scale = 1.0f;
    if (key_bytes == 8 || domain == 1) {
        float mnx = -ord2f(sc->bbox[0]), mny = -ord2f(sc->bbox[1]);
        float mxx = ord2f(sc->bbox[2]), mxy = ord2f(sc->bbox[3]);
        if (key_bytes == 8) {
            float m = fmaxf(fmaxf(fabsf(mnx), fabsf(mxx)), fmaxf(fabsf(mny), fabsf(mxy)));
            int e;
            if (m < 0x1p-60f) e = -60;
            else { int ex; frexpf(m, &ex); e = ex + 1; }
            d.scale = ldexpf(1.0f, 32 - e);
        } else {
            float ext = fmaxf(__fsub_rn(mxx, mnx), __fsub_rn(mxy, mny));
            if (!(ext > 0.0f)) ext = 1.0f;
            d.lo_x = mnx;
            d.lo_y = mny;
            d.ext = ext;
        }
    }
    return d;
}

template <typename K>
__device__ __forceinline__ K encode_one(float x, float y, const Domain& d);

template <>
__device__ __forceinline__ uint32_t encode_one<uint32_t>(float x, float y, const Domain& d) {
    return spread16(quant16(x, d.lo_x, d.ext)) | (spread16(quant16(y, d.lo_y, d.ext)) << 1);
}
template <>
__device__ __forceinline__ uint64_t encode_one<uint64_t>(float x, float y, const Domain& d) {
    return spread32(quant32(x, d.scale)) | (spread32(quant32(y, d.scale)) << 1);
}

template <typename K>
__global__ void __launch_bounds__(256) encode_kernel(const float4* __restrict__ pos2, uint32_t n,
                                                     K* __restrict__ codes, int domain,
                                                     StepScratch* scratch,
                                                     const float* __restrict__ mass,
                                                     float4* __restrict__ xm) {
    constexpr int P = (int)sizeof(K);  // digit passes = key bytes
    __shared__ uint32_t sh[P][kRadix];
    for (int i = threadIdx.x; i < P * kRadix; i += blockDim.x) (&sh[0][0])[i] = 0;
    __syncthreads();
    const Domain d = read_domain(scratch, domain, (int)sizeof(K));
    const uint32_t pairs = (n + 1) / 2;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pairs; i += gridDim.x * blockDim.x) {
        uint32_t b0 = 2 * i;
        float4 v;
        if (b0 + 1 < n) v = __ldg(&pos2[i]);
        else {
            float2 t = reinterpret_cast<const float2*>(pos2)[b0];
            v = make_float4(t.x, t.y, 0.f, 0.f);
        }
        K k0 = encode_one<K>(v.x, v.y, d);
        codes[b0] = k0;
        // the body records the hierarchy build gathers by sorted id: one
        // 16-B load there instead of a position and a mass
        if (xm) {
            xm[b0] = make_float4(v.x, v.y, __ldg(&mass[b0]), 0.0f);
            if (b0 + 1 < n) xm[b0 + 1] = make_float4(v.z, v.w, __ldg(&mass[b0 + 1]), 0.0f);
        }
#pragma unroll
        for (int p = 0; p < P; ++p) atomicAdd(&sh[p][(uint32_t)(k0 >> (8 * p)) & 0xFFu], 1u);
        if (b0 + 1 < n) {
            K k1 = encode_one<K>(v.z, v.w, d);
            codes[b0 + 1] = k1;
#pragma unroll
            for (int p = 0; p < P; ++p) atomicAdd(&sh[p][(uint32_t)(k1 >> (8 * p)) & 0xFFu], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < P * kRadix; i += blockDim.x) {
        uint32_t c = (&sh[0][0])[i];
        if (c) atomicAdd(&scratch->hist[i / kRadix][i % kRadix], c);
    }
}

void launch_encode(const DeviceBuffers& b, int domain, cudaStream_t s) {
    if (b.n == 0) return;
    uint32_t pairs = (b.n + 1) / 2;
    int blocks = (int)((pairs + 255) / 256);
    if (blocks > 148 * encode_blocks_per_sm(b.n)) blocks = 148 * encode_blocks_per_sm(b.n);
    if (blocks < 1) blocks = 1;
    const float4* p2 = reinterpret_cast<const float4*>(b.pos);
    if (b.key_bytes == 8)
        encode_kernel<uint64_t><<<blocks, 256, 0, s>>>(p2, b.n, (uint64_t*)b.codes, domain, b.scratch,
                                                       b.mass, b.xm);
    else
        encode_kernel<uint32_t><<<blocks, 256, 0, s>>>(p2, b.n, (uint32_t*)b.codes, domain, b.scratch,
                                                       b.mass, b.xm);
}

// ---- ensembles: one box and one 32-bit Morton domain per system ----------
// A warp whose 32 bodies all belong to one system (the common case: systems
// are contiguous) reduces first and issues one atomic per bound.
__global__ void __launch_bounds__(256) bbox_ensemble_kernel(const float2* __restrict__ pos,
                                                            const uint32_t* __restrict__ body_sys,
                                                            uint32_t n, uint32_t* __restrict__ sys_bbox) {
    const unsigned FULL = 0xFFFFFFFFu;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const bool ok = i < n;
        const float2 p = ok ? __ldg(&pos[i]) : make_float2(0.f, 0.f);
        const uint32_t sys = ok ? __ldg(&body_sys[i]) : kSentinel;
        float v[4] = {ok ? -p.x : -INFINITY, ok ? -p.y : -INFINITY, ok ? p.x : -INFINITY,
                      ok ? p.y : -INFINITY};
        const uint32_t s0 = __shfl_sync(FULL, sys, 0);
        if (__all_sync(FULL, !ok || sys == s0)) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v[k] = fmaxf(v[k], __shfl_xor_sync(FULL, v[k], o));
            if ((threadIdx.x & 31) == 0 && s0 != kSentinel)
#pragma unroll
                for (int k = 0; k < 4; ++k) atomicMax(&sys_bbox[4 * s0 + k], f2ord(v[k]));
        } else if (ok) {
#pragma unroll
            for (int k = 0; k < 4; ++k) atomicMax(&sys_bbox[4 * sys + k], f2ord(v[k]));
        }
    }
}

void launch_bbox_ensemble(const DeviceBuffers& b, cudaStream_t s) {
    if (b.n == 0) return;
    int blocks = (int)((b.n + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    bbox_ensemble_kernel<<<blocks, 256, 0, s>>>(b.pos, b.body_sys, b.n, b.sys_bbox);
}

// key = (system << 32) | morton32 over the system's box (same quantisation as
// the single-system bbox domain); histograms of the sort's digit passes.
__global__ void __launch_bounds__(256) encode_ensemble_kernel(const float2* __restrict__ pos,
                                                              const uint32_t* __restrict__ body_sys,
                                                              const uint32_t* __restrict__ sys_bbox,
                                                              uint32_t n, int passes,
                                                              uint64_t* __restrict__ codes,
                                                              StepScratch* scratch,
                                                              const float* __restrict__ mass,
                                                              float4* __restrict__ xm) {
    __shared__ uint32_t sh[8][kRadix];
    for (int i = threadIdx.x; i < 8 * kRadix; i += blockDim.x) (&sh[0][0])[i] = 0;
    __syncthreads();
    const unsigned FULL = 0xFFFFFFFFu;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const bool ok = i < n;
        uint64_t k = 0;
        if (ok) {
            const float2 p = __ldg(&pos[i]);
            const uint32_t sys = __ldg(&body_sys[i]);
            const float mnx = -ord2f(__ldg(&sys_bbox[4 * sys])), mny = -ord2f(__ldg(&sys_bbox[4 * sys + 1]));
            const float mxx = ord2f(__ldg(&sys_bbox[4 * sys + 2])), mxy = ord2f(__ldg(&sys_bbox[4 * sys + 3]));
            float ext = fmaxf(__fsub_rn(mxx, mnx), __fsub_rn(mxy, mny));
            if (!(ext > 0.0f)) ext = 1.0f;
            const uint32_t m = spread16(quant16(p.x, mnx, ext)) | (spread16(quant16(p.y, mny, ext)) << 1);
            k = ((uint64_t)sys << 32) | m;
            codes[i] = k;
            if (xm) xm[i] = make_float4(p.x, p.y, __ldg(&mass[i]), 0.0f);
        }
        // Morton digits are spread out: one shared atomic per body.  System
        // digits repeat across a warp: one atomic per distinct digit.
        const unsigned act = __ballot_sync(FULL, ok);
        for (int q = 0; q < 4 && q < passes; ++q)
            if (ok) atomicAdd(&sh[q][(uint32_t)(k >> (8 * q)) & 0xFFu], 1u);
        for (int q = 4; q < passes; ++q) {
            if (ok) {
                const uint32_t d = (uint32_t)(k >> (8 * q)) & 0xFFu;
                const unsigned peers = __match_any_sync(act, d);
                if ((threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1)) atomicAdd(&sh[q][d], (uint32_t)__popc(peers));
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x) {
        const uint32_t c = (&sh[0][0])[i];
        if (c) atomicAdd(&scratch->hist[i / kRadix][i % kRadix], c);
    }
}

void launch_encode_ensemble(const DeviceBuffers& b, cudaStream_t s) {
    if (b.n == 0) return;
    int blocks = (int)((b.n + 255) / 256);
    if (blocks > 148 * encode_blocks_per_sm(b.n)) blocks = 148 * encode_blocks_per_sm(b.n);
    encode_ensemble_kernel<<<blocks, 256, 0, s>>>(b.pos, b.body_sys, b.sys_bbox, b.n, b.sort_passes,
                                                  (uint64_t*)b.codes, b.scratch, b.mass, b.xm);
}

// ---- leapfrog opening kick + drift (original order, coalesced) -----------
__global__ void __launch_bounds__(256) kick_drift_kernel(float2* __restrict__ pos,
                                                         float2* __restrict__ vel,
                                                         const float2* __restrict__ acc, uint32_t n,
                                                         float dt, float hdt) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float2 v = vel[i], a = acc[i], p = pos[i];
        v.x = __fadd_rn(v.x, __fmul_rn(a.x, hdt));
        v.y = __fadd_rn(v.y, __fmul_rn(a.y, hdt));
        p.x = __fadd_rn(p.x, __fmul_rn(v.x, dt));
        p.y = __fadd_rn(p.y, __fmul_rn(v.y, dt));
        vel[i] = v;
        pos[i] = p;
    }
}

// ---- per-step reset ---------------------------------------------------------
// Zeroes the step's scratch record and the sort's look-back status in one
// launch (in a captured step, two memset nodes cost more than these writes).
static_assert(sizeof(StepScratch) % 4 == 0, "scratch is cleared in 4-byte words");
__global__ void __launch_bounds__(256) zero_step_kernel(uint32_t* __restrict__ scratch, uint32_t words,
                                                        uint4* __restrict__ status, size_t quads) {
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = t; i < words; i += stride) scratch[i] = 0u;
    for (size_t i = t; i < quads; i += stride) status[i] = make_uint4(0u, 0u, 0u, 0u);
}

void launch_zero_step(const DeviceBuffers& b, cudaStream_t s) {
    // status: key_bytes passes x tiles x 256 words, a multiple of 16 bytes,
    // 256-byte aligned in the arena like the scratch record
    const size_t quads = (size_t)b.key_bytes * b.tiles * kRadix / 4;
    const uint32_t words = (uint32_t)(sizeof(StepScratch) / 4);
    const size_t work = quads > words ? quads : words;
    size_t blocks = (work + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    zero_step_kernel<<<(unsigned)blocks, 256, 0, s>>>(reinterpret_cast<uint32_t*>(b.scratch), words,
                                                      reinterpret_cast<uint4*>(b.status), quads);
}

void launch_kick_drift(const DeviceBuffers& b, float dt, cudaStream_t s) {
    if (b.n == 0) return;
    int blocks = (int)((b.n + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    kick_drift_kernel<<<blocks, 256, 0, s>>>(b.pos, b.vel, b.acc, b.n, dt, 0.5f * dt);
}

}  // namespace bh
