// generate.cu -- seeded scenario generators on the GPU (extension).
//
// The reference builds its initial conditions on the CPU from Math.random()
// (src/simulation.ts:233-374) and uploads them; the engine's host generators
// (scenarios.cpp) do the same from one sequential PCG32 stream.  At 16.8M
// bodies that is seconds of host work and a 400 MB upload.  Here every body
// i draws from its own PCG32 stream (O'Neill 2014, XSH-RR output, sequence
// selector splitmix64(i)), so all bodies are generated in parallel, in FP64
// like the host generators (JavaScript numbers), and stored as FP32.  The
// distributions and formulas are those of scenarios.cpp; the sample is a
// different one than the host generator's for the same seed (different
// streams).  Draws per body that depend on data (the colliding disks' radius
// rejection, the Gaussian mixture's duplicates) stay within the body's own
// stream, so the result does not depend on the launch shape.
//
// Gaussian mixture: the 64 components come from PCG32(seed) on the host (the
// same draws as scenarios.cpp); a body that duplicates an earlier body j
// (1%) takes body j's coordinates, found by replaying j's stream (and j's
// own duplicate, if any, down to a body that is not one).  Masses are
// log-normal, normalised to total 1 by an FP64 sum of per-block partial sums
// taken in block order: positions and velocities do not depend on the launch
// shape; the normalised masses can differ in their last bit between GPUs
// with different SM counts (the total's summation order).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include "bh.h"
#include "bh_internal.cuh"

namespace bh {

void set_global_error(const std::string& msg);

enum GenScenario : int {
    kGenDefault = 0,
    kGenTwoClusters,
    kGenPlanetaryDisk,
    kGenUniformDiskKepler,
    kGenCollidingDisks,
    kGenGaussianMixture,
    kGenPlummerProjection,
};

constexpr int kGenThreads = 256;
constexpr int kMixtureK = 64;

struct GenParams {
    uint32_t n;
    uint64_t seed;
    double G;
    int scenario;
    double cx[kMixtureK], cy[kMixtureK], sig[kMixtureK];  // Gaussian mixture
};

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

struct DevPcg32 {
    uint64_t state, inc;
    __host__ __device__ DevPcg32(uint64_t seed, uint64_t seq) : state(0), inc((seq << 1u) | 1u) {
        next();
        state += seed;
        next();
    }
    __host__ __device__ uint32_t next() {
        const uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        const uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        const uint32_t rot = (uint32_t)(old >> 59u);
        return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
    }
    // uniform double in [0, 1) from 53 random bits
    __host__ __device__ double uniform() {
        const uint64_t a = next() >> 5, b = next() >> 6;
        return (double)(a * 67108864ULL + b) * (1.0 / 9007199254740992.0);
    }
    __host__ __device__ double normal() {  // Box-Muller, cosine branch
        double u1 = uniform();
        const double u2 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
    }
};

// Body i's stream.
__device__ __forceinline__ DevPcg32 body_stream(uint64_t seed, uint32_t i) {
    return DevPcg32(seed, splitmix64((uint64_t)i));
}

__device__ __forceinline__ void put(float* mass, float2* pos, float2* vel, uint32_t i, double m,
                                    double x, double y, double vx, double vy) {
    mass[i] = (float)m;
    pos[i] = make_float2((float)x, (float)y);
    vel[i] = make_float2((float)vx, (float)vy);
}

// Coordinates of mixture body j (a duplicate takes an earlier body's).
__device__ float2 mixture_point(const GenParams& P, uint32_t j) {
    while (true) {
        DevPcg32 rng = body_stream(P.seed, j);
        (void)rng.normal();  // the body's mass draw
        if (j > 0 && rng.uniform() < 0.01) {
            j = (uint32_t)(rng.uniform() * (double)j);
            continue;
        }
        int k = (int)(rng.uniform() * kMixtureK);
        if (k >= kMixtureK) k = kMixtureK - 1;
        const double x = P.cx[k] + P.sig[k] * rng.normal();
        const double y = P.cy[k] + P.sig[k] * rng.normal();
        return make_float2((float)x, (float)y);
    }
}

__global__ void __launch_bounds__(kGenThreads)
generate_kernel(const GenParams P, float* __restrict__ mass, float2* __restrict__ pos,
                float2* __restrict__ vel, float* __restrict__ radius, double* __restrict__ partial) {
    __shared__ double s_sum[kGenThreads / 32];
    const uint32_t n = P.n;
    const double G = P.G;
    double msum = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (radius) radius[i] = 1.0f;
        DevPcg32 rng = body_stream(P.seed, i);
        switch (P.scenario) {
            case kGenDefault: {  // simulation.ts:243-266
                const double angle = rng.uniform() * 2.0 * M_PI;
                const double r = 5.0 * sqrt(rng.uniform());
                const double x = r * cos(angle), y = r * sin(angle);
                const double dist = sqrt(x * x + y * y);
                const double speed = 0.1 * sqrt(G * (double)n / dist);
                put(mass, pos, vel, i, 1.0, x, y, -speed * (y / dist), speed * (x / dist));
                break;
            }
            case kGenTwoClusters: {  // simulation.ts:267-306
                const double angle = rng.uniform() * 2.0 * M_PI;
                const double r = 3.0 * sqrt(rng.uniform());
                const double xb = r * cos(angle), yb = r * sin(angle);
                const bool first = (double)i < (double)n / 2.0;
                const double dist = sqrt(xb * xb + yb * yb);
                const double speed = 0.12 * sqrt(G * ((double)n / 2.0) / dist);
                put(mass, pos, vel, i, 1.0, first ? xb - 15.0 : xb + 15.0, yb,
                    first ? -speed * (yb / dist) : speed * (yb / dist),
                    first ? speed * (xb / dist) : -speed * (xb / dist));
                break;
            }
            case kGenPlanetaryDisk: {  // simulation.ts:308-361
                const double central = 1000.0, planet = 10.0;
                if (i == 0) {
                    put(mass, pos, vel, i, central, 0.0, 0.0, 0.0, 0.0);
                    if (radius) radius[i] = 12.0f;
                } else if (i == 1) {
                    put(mass, pos, vel, i, planet, 2.5, 0.0, 0.0, 0.8 * sqrt(G * central / 2.5));
                    if (radius) radius[i] = 5.0f;
                } else if (i == 2) {
                    put(mass, pos, vel, i, planet, 12.0, 0.0, 0.0, sqrt(G * central / 12.5));
                    if (radius) radius[i] = 5.0f;
                } else {
                    const double angle = rng.uniform() * 2.0 * M_PI;
                    const double r = sqrt(rng.uniform() * (15.0 * 15.0 - 0.1 * 0.1) + 0.1 * 0.1);
                    const double x = r * cos(angle), y = r * sin(angle);
                    const double dist = sqrt(x * x + y * y);
                    const double speed = 1.01 * sqrt(G * central / (2.0 + dist));
                    put(mass, pos, vel, i, central / (100.0 * (double)n), x, y, -speed * (y / dist),
                        speed * (x / dist));
                }
                break;
            }
            case kGenUniformDiskKepler: {
                const double angle = rng.uniform() * 2.0 * M_PI;
                const double r = sqrt(rng.uniform());
                const double x = r * cos(angle), y = r * sin(angle);
                const double v = sqrt(G * r * r / (r > 1e-12 ? r : 1e-12));
                const double c = r > 0 ? x / r : 1.0, s = r > 0 ? y / r : 0.0;
                put(mass, pos, vel, i, 1.0 / (double)n, x, y, -v * s, v * c);
                break;
            }
            case kGenCollidingDisks: {
                const double h = 0.2, rmax = 10.0 * h;
                const double md = 1.0 / 2.2, mc = 0.1 * md;
                const uint32_t half = n / 2;
                const int gal = i < half ? 0 : 1;
                const uint32_t lo = gal == 0 ? 0 : half, hi = gal == 0 ? half : n;
                const uint32_t cnt = hi - lo;
                const double cx = gal == 0 ? 1.5 : -1.5;
                const double bvx = gal == 0 ? -0.3 : 0.3, bvy = gal == 0 ? 0.1 : -0.1;
                if (i == lo) {
                    put(mass, pos, vel, i, cnt > 1 ? mc : md + mc, cx, 0.0, bvx, bvy);
                    break;
                }
                double R = rmax;
                for (int t = 0; t < 64; ++t) {  // Gamma(2, h) radius, rejected above rmax
                    double u1 = rng.uniform(), u2 = rng.uniform();
                    if (u1 < 1e-300) u1 = 1e-300;
                    if (u2 < 1e-300) u2 = 1e-300;
                    R = -h * log(u1 * u2);
                    if (R <= rmax) break;
                }
                if (R > rmax) R = rmax;
                const double angle = rng.uniform() * 2.0 * M_PI;
                const double x = R * cos(angle), y = R * sin(angle);
                const double menc = mc + md * (1.0 - (1.0 + R / h) * exp(-R / h));
                const double Rs = R > 1e-6 ? R : 1e-6;
                const double v = sqrt(G * menc / Rs);
                put(mass, pos, vel, i, md / (double)(cnt - 1), cx + x, y, bvx - v * (y / Rs),
                    bvy + v * (x / Rs));
                break;
            }
            case kGenGaussianMixture: {
                const double m = exp(rng.normal());
                msum += (double)(float)m;
                mass[i] = (float)m;  // normalised by normalise_kernel
                pos[i] = mixture_point(P, i);
                vel[i] = make_float2(0.0f, 0.0f);
                break;
            }
            default: {  // kGenPlummerProjection
                const double a = 0.1;
                const double u = rng.uniform() * 0.999;
                const double R = a * sqrt(u / (1.0 - u));
                const double angle = rng.uniform() * 2.0 * M_PI;
                const double x = R * cos(angle), y = R * sin(angle);
                const double menc = R * R / (R * R + a * a);
                const double Rs = R > 1e-9 ? R : 1e-9;
                const double v = sqrt(G * menc / Rs);
                put(mass, pos, vel, i, 1.0 / (double)n, x, y, -v * (y / Rs), v * (x / Rs));
                break;
            }
        }
    }
    if (partial) {
        // block sum of the masses, in a fixed order
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) msum += __shfl_xor_sync(0xFFFFFFFFu, msum, o);
        if ((threadIdx.x & 31) == 0) s_sum[threadIdx.x >> 5] = msum;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < kGenThreads / 32; ++w) t += s_sum[w];
            partial[blockIdx.x] = t;
        }
    }
}

// mass[i] /= sum of the partial sums (added in block order by every thread).
__global__ void __launch_bounds__(kGenThreads)
normalise_kernel(float* __restrict__ mass, uint32_t n, const double* __restrict__ partial,
                 uint32_t nparts) {
    double total = 0.0;
    for (uint32_t k = 0; k < nparts; ++k) total += partial[k];
    if (!(total > 0.0)) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        mass[i] = (float)((double)mass[i] / total);
}

// Host-side: the mixture components, the first draws of PCG32(seed) as in
// scenarios.cpp's gen_gaussian_mixture.
static void mixture_components(uint64_t seed, GenParams& P) {
    DevPcg32 rng(seed, 0x5851f42d4c957f2dULL);
    for (int k = 0; k < kMixtureK; ++k) {
        P.cx[k] = -4.0 + 8.0 * rng.uniform();
        P.cy[k] = -4.0 + 8.0 * rng.uniform();
        P.sig[k] = std::exp(std::log(1e-3) + (std::log(0.5) - std::log(1e-3)) * rng.uniform());
    }
}

int scenario_id(const char* name) {
    if (!name) return -1;
    static const char* names[] = {"default", "two-clusters", "planetary-disk",
                                  "uniform-disk-kepler", "colliding-disks", "gaussian-mixture",
                                  "plummer-projection"};
    for (int k = 0; k < 7; ++k)
        if (std::strcmp(name, names[k]) == 0) return k;
    return -1;
}

// Enqueue the generator for `n` bodies on `stream`; returns a CUDA status.
cudaError_t launch_generate(int scenario, uint32_t n, uint64_t seed, float grav_constant,
                            float* mass, float2* pos, float2* vel, float* radius, int device,
                            cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    GenParams P;
    std::memset(&P, 0, sizeof(P));
    P.n = n;
    P.seed = seed;
    P.G = grav_constant;
    P.scenario = scenario;
    if (scenario == kGenGaussianMixture) mixture_components(seed, P);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    uint32_t blocks = (uint32_t)sms * 8u;
    const uint32_t need = (n + kGenThreads - 1) / kGenThreads;
    if (blocks > need) blocks = need;
    double* partial = nullptr;
    if (scenario == kGenGaussianMixture) {
        cudaError_t e = cudaMallocAsync((void**)&partial, sizeof(double) * blocks, stream);
        if (e != cudaSuccess) return e;
    }
    generate_kernel<<<blocks, kGenThreads, 0, stream>>>(P, mass, pos, vel, radius, partial);
    if (partial) {
        normalise_kernel<<<blocks, kGenThreads, 0, stream>>>(mass, n, partial, blocks);
        cudaFreeAsync(partial, stream);
    }
    return cudaGetLastError();
}

}  // namespace bh

extern "C" int bh_generate_scenario_device(const char* name, uint32_t n, uint64_t seed,
                                           float grav_constant, float* mass, float* pos, float* vel,
                                           float* radius_multiplier, void* stream) {
    const int id = bh::scenario_id(name);
    if (id < 0) {
        bh::set_global_error(std::string("Unknown scenario: ") + (name ? name : "(null)"));
        return BH_ERR_UNKNOWN_SCENARIO;
    }
    if (n > 0 && (!mass || !pos || !vel)) {
        bh::set_global_error("bh_generate_scenario_device: null body array");
        return BH_ERR_INVALID_ARGUMENT;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    const cudaError_t e = bh::launch_generate(id, n, seed, grav_constant, mass,
                                              reinterpret_cast<float2*>(pos),
                                              reinterpret_cast<float2*>(vel), radius_multiplier, dev,
                                              static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        bh::set_global_error(std::string("bh_generate_scenario_device: ") + cudaGetErrorString(e));
        return BH_ERR_CUDA;
    }
    return BH_OK;
}
