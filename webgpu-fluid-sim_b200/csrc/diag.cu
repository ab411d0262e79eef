// diag.cu -- FP64 diagnostics of a simulation's state (extension).
//
// The reference's only run-time output is an FPS line on the console every
// second (src/main.ts:44-49).  The engine reports conserved quantities
// instead, summed in FP64 over all bodies (original order):
//     M = sum m,  COM = sum m x / M,  P = sum m v,  Lz = sum m (x v_y - y v_x),
//     K = 1/2 sum m |v|^2,
//     W = -G sum_{i<j} m_i m_j / sqrt(|x_i - x_j|^2 + eps_ij^2)
// with the pair softening of the force law in use (Plummer: eps; the
// reference's: eps_ij^2 = epsMult^2 G dt max(m_i, m_j), barnes_hut.wgsl:90-92),
// so that W is the potential whose gradient is the walk's direct-sum force.
//
// moments_kernel: grid-stride FP64 sums, warp shuffles, one FP64 atomic per
// block and quantity.  potential_kernel: the O(N^2) pair sum, tiled through
// shared memory (256 bodies per tile): each thread owns one body, sums a
// tile's terms m_j / r_ij in FP32 (rsqrt, relative error ~1e-7 per term) and
// adds each tile's sum into an FP64 accumulator; blocks add m_i-weighted sums
// with one FP64 atomic.  About 10 operations per pair: 800k bodies take
// ~0.1 s, so W is for diagnostics, not for every step.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "bh.h"
#include "bh_internal.cuh"

namespace bh {

constexpr int kDiagThreads = 256;
constexpr int kDiagMoments = 7;  // m, m x, m y, m vx, m vy, Lz, 2K

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

__global__ void __launch_bounds__(kDiagThreads)
moments_kernel(const float* __restrict__ mass, const float2* __restrict__ pos,
               const float2* __restrict__ vel, uint32_t n, double* __restrict__ out) {
    __shared__ double s[kDiagThreads / 32][kDiagMoments];
    double a[kDiagMoments] = {0, 0, 0, 0, 0, 0, 0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double m = mass[i];
        const float2 x = pos[i], v = vel[i];
        const double px = m * (double)v.x, py = m * (double)v.y;
        a[0] += m;
        a[1] += m * (double)x.x;
        a[2] += m * (double)x.y;
        a[3] += px;
        a[4] += py;
        a[5] += (double)x.x * py - (double)x.y * px;
        a[6] += px * (double)v.x + py * (double)v.y;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kDiagMoments; ++k) {
        const double t = warp_sum_d(a[k]);
        if (lane == 0) s[warp][k] = t;
    }
    __syncthreads();
    if (threadIdx.x < kDiagMoments) {
        double t = 0.0;
        for (int w = 0; w < kDiagThreads / 32; ++w) t += s[w][threadIdx.x];
        atomicAdd(&out[threadIdx.x], t);
    }
}

__global__ void __launch_bounds__(kDiagThreads)
potential_kernel(const float* __restrict__ mass, const float2* __restrict__ pos, uint32_t n,
                 int plummer, float eps2, float eps_coef, double* __restrict__ out) {
    __shared__ float4 tile[kDiagThreads];  // {x, y, m, 0}
    __shared__ double s[kDiagThreads / 32];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float xi = 0.0f, yi = 0.0f, mi = 0.0f;
    if (i < n) {
        const float2 p = pos[i];
        xi = p.x;
        yi = p.y;
        mi = mass[i];
    }
    double acc = 0.0;
    for (uint32_t t0 = 0; t0 < n; t0 += kDiagThreads) {
        __syncthreads();
        const uint32_t j = t0 + threadIdx.x;
        if (j < n) {
            const float2 p = pos[j];
            tile[threadIdx.x] = make_float4(p.x, p.y, mass[j], 0.0f);
        } else {
            tile[threadIdx.x] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        __syncthreads();
        if (i < n) {
            const uint32_t cnt = (n - t0) < (uint32_t)kDiagThreads ? (n - t0) : (uint32_t)kDiagThreads;
            float sum = 0.0f;
            for (uint32_t k = 0; k < cnt; ++k) {
                const float4 o = tile[k];
                const float dx = o.x - xi, dy = o.y - yi;
                const float e2 = plummer ? eps2 : eps_coef * fmaxf(mi, o.z);
                const float r2 = fmaf(dx, dx, fmaf(dy, dy, e2));
                const float term = (t0 + k == i || !(r2 > 0.0f)) ? 0.0f : o.z * rsqrt_ftz(r2);
                sum += term;
            }
            acc += (double)sum;
        }
    }
    acc *= (double)mi;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double t = warp_sum_d(acc);
    if (lane == 0) s[warp] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < kDiagThreads / 32; ++w) b += s[w];
        atomicAdd(out, b);
    }
}

// FP64 direct-sum acceleration of sampled bodies: block (k, c) adds body
// sample[k]'s pull from the bodies of chunk c.  Consecutive blocks take
// consecutive samples of the same chunk, so the blocks resident together
// read the same ~1M bodies and the chunk is read from DRAM about once.
constexpr uint32_t kDirectChunks = 16;

__global__ void __launch_bounds__(kDiagThreads)
direct_fp64_kernel(const float* __restrict__ mass, const float2* __restrict__ pos, uint32_t n,
                   const uint32_t* __restrict__ sample, int plummer, double eps2, double eps_coef,
                   double* __restrict__ out) {
    __shared__ double s[2][kDiagThreads / 32];
    const uint32_t i = sample[blockIdx.x];
    const uint32_t chunk = (n + gridDim.y - 1) / gridDim.y;
    const uint32_t lo = blockIdx.y * chunk;
    const uint32_t hi = (lo + chunk) < n ? (lo + chunk) : n;
    const float2 pi = pos[i];
    const double xi = pi.x, yi = pi.y, mi = mass[i];
    double ax = 0.0, ay = 0.0;
    for (uint32_t j = lo + threadIdx.x; j < hi; j += kDiagThreads) {
        if (j == i) continue;
        const float2 pj = pos[j];
        const double mj = mass[j];
        const double dx = (double)pj.x - xi, dy = (double)pj.y - yi;
        const double e2 = plummer ? eps2 : eps_coef * fmax(mi, mj);
        const double r2 = dx * dx + dy * dy + e2;
        if (!(r2 > 0.0)) continue;
        const double inv = rsqrt(r2);
        const double f = mj * inv * inv * inv;
        ax += f * dx;
        ay += f * dy;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    ax = warp_sum_d(ax);
    ay = warp_sum_d(ay);
    if (lane == 0) {
        s[0][warp] = ax;
        s[1][warp] = ay;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double t = 0.0;
        for (int w = 0; w < kDiagThreads / 32; ++w) t += s[threadIdx.x][w];
        atomicAdd(&out[2 * (size_t)blockIdx.x + threadIdx.x], t);
    }
}

bool sim_body_view(const bh_sim* s, BodyView* out);
void set_global_error(const std::string& msg);

}  // namespace bh

static int dfail(int code, const std::string& msg) {
    bh::set_global_error(msg);
    return code;
}

extern "C" int bh_diagnostics_compute(bh_sim* sim, int with_potential, bh_diagnostics* out) {
    if (!sim || !out) return dfail(BH_ERR_INVALID_ARGUMENT, "bh_diagnostics_compute: null argument");
    bh_config cfg;
    const int st = bh_get_config(sim, &cfg);
    if (st != BH_OK) return st;
    bh::BodyView v;
    bh::sim_body_view(sim, &v);
    cudaError_t e = cudaSetDevice(v.device);
    if (e != cudaSuccess) return dfail(BH_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    double h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (v.n > 0) {
        double* d = nullptr;
        e = cudaMallocAsync((void**)&d, sizeof(h), v.stream);
        if (e != cudaSuccess) return dfail(BH_ERR_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
        cudaMemsetAsync(d, 0, sizeof(h), v.stream);
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, v.device);
        uint32_t blocks = (uint32_t)sms * 4u;
        const uint32_t need = (v.n + bh::kDiagThreads - 1) / bh::kDiagThreads;
        if (blocks > need) blocks = need;
        bh::moments_kernel<<<blocks, bh::kDiagThreads, 0, v.stream>>>(v.mass, v.pos, v.vel, v.n, d);
        if (with_potential) {
            const int plummer = cfg.softening == BH_SOFTENING_PLUMMER;
            const float eps2 = cfg.plummer_eps * cfg.plummer_eps;
            // (epsMult sqrt(G dt m))^2, barnes_hut.wgsl:90-92
            const float coef = cfg.epsilon_multiplier * cfg.epsilon_multiplier * cfg.grav_constant *
                               cfg.delta_time;
            bh::potential_kernel<<<need, bh::kDiagThreads, 0, v.stream>>>(v.mass, v.pos, v.n, plummer,
                                                                           eps2, coef, d + 7);
        }
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, v.stream);
        cudaFreeAsync(d, v.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(v.stream);
        if (e != cudaSuccess) return dfail(BH_ERR_CUDA, std::string("diagnostics: ") + cudaGetErrorString(e));
    }
    out->total_mass = h[0];
    out->com[0] = h[0] > 0.0 ? h[1] / h[0] : 0.0;
    out->com[1] = h[0] > 0.0 ? h[2] / h[0] : 0.0;
    out->momentum[0] = h[3];
    out->momentum[1] = h[4];
    out->angular_momentum = h[5];
    out->kinetic_energy = 0.5 * h[6];
    // each pair was summed from both sides
    out->potential_energy = with_potential ? -0.5 * (double)cfg.grav_constant * h[7] : NAN;
    out->pairs = (with_potential && v.n > 1) ? (uint64_t)v.n * (v.n - 1) / 2 : 0;
    return BH_OK;
}

extern "C" int bh_direct_forces_fp64(bh_sim* sim, const uint32_t* sample, uint32_t count,
                                     double* acc_out) {
    if (!sim || (count && (!sample || !acc_out)))
        return dfail(BH_ERR_INVALID_ARGUMENT, "bh_direct_forces_fp64: null argument");
    if (count > (1u << 20))
        return dfail(BH_ERR_INVALID_ARGUMENT, "bh_direct_forces_fp64: at most 2^20 samples per call");
    bh_config cfg;
    const int st = bh_get_config(sim, &cfg);
    if (st != BH_OK) return st;
    bh::BodyView v;
    bh::sim_body_view(sim, &v);
    for (uint32_t k = 0; k < count; ++k)
        if (sample[k] >= v.n) return dfail(BH_ERR_INVALID_ARGUMENT, "bh_direct_forces_fp64: sample index out of range");
    if (count == 0) return BH_OK;
    cudaError_t e = cudaSetDevice(v.device);
    if (e != cudaSuccess) return dfail(BH_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    const size_t out_bytes = 2 * sizeof(double) * (size_t)count;
    const size_t idx_off = (out_bytes + 255) & ~(size_t)255;
    unsigned char* d = nullptr;
    e = cudaMallocAsync((void**)&d, idx_off + 4 * (size_t)count, v.stream);
    if (e != cudaSuccess) return dfail(BH_ERR_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    double* dacc = reinterpret_cast<double*>(d);
    uint32_t* didx = reinterpret_cast<uint32_t*>(d + idx_off);
    e = cudaMemsetAsync(dacc, 0, out_bytes, v.stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(didx, sample, 4 * (size_t)count, cudaMemcpyHostToDevice, v.stream);
    if (e == cudaSuccess) {
        const int plummer = cfg.softening == BH_SOFTENING_PLUMMER;
        const double eps2 = (double)cfg.plummer_eps * (double)cfg.plummer_eps;
        // (epsMult sqrt(G dt m))^2, barnes_hut.wgsl:90-92
        const double coef = (double)cfg.epsilon_multiplier * cfg.epsilon_multiplier *
                            cfg.grav_constant * cfg.delta_time;
        uint32_t chunks = bh::kDirectChunks;
        if (v.n < chunks * bh::kDiagThreads) chunks = 1;
        bh::direct_fp64_kernel<<<dim3(count, chunks), bh::kDiagThreads, 0, v.stream>>>(
            v.mass, v.pos, v.n, didx, plummer, eps2, coef, dacc);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(acc_out, dacc, out_bytes, cudaMemcpyDeviceToHost, v.stream);
    cudaFreeAsync(d, v.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(v.stream);
    if (e != cudaSuccess) return dfail(BH_ERR_CUDA, std::string("direct forces: ") + cudaGetErrorString(e));
    const double G = cfg.grav_constant;
    for (size_t k = 0; k < 2 * (size_t)count; ++k) acc_out[k] *= G;
    return BH_OK;
}
