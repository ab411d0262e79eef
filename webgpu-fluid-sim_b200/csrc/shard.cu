// shard.cu -- the exchange step of a single system sharded across GPUs
// (extension; the reference runs on one WebGPU device).
//
// Every rank keeps the whole state and builds the same tree from it (the
// pipeline is deterministic: same inputs, same codes, permutation, nodes and
// groups).  Rank r walks and integrates only the groups whose first sorted
// slot lies in its slot range [lo, hi), i.e. exactly the bodies in sorted
// slots [a, b) with a = first group start >= lo and b = first group start
// >= hi (or n); the ranks' [a, b) tile [0, n).  After the step each rank
// packs what it updated -- (pos, vel) for symplectic Euler, (vel, acc) for
// leapfrog, whose next opening kick-drift every rank then repeats on all
// bodies -- in sorted-slot order into a fixed-size chunk; one all-gather of
// the chunks (NCCL, by the caller) and an unpack by the same sorted
// permutation leave every rank with the state a single GPU would have.
//
// Chunk layout (16-byte aligned): uint32 {a, count, 0, 0}, then count
// records of float4 {field0.x, field0.y, field1.x, field1.y}; its size is
// 16 + 16 * capacity bytes.  A range longer than the capacity is not packed
// (count 0) and raises kErrShardCapacity; unpacking checks every header
// against the capacity and n.
#include <cuda_runtime.h>

#include "bh_internal.cuh"

namespace bh {

constexpr int kShardThreads = 256;

__global__ void __launch_bounds__(kShardThreads)
shard_bounds_kernel(const uint2* __restrict__ groups, const unsigned int* __restrict__ group_ctr,
                    uint32_t n, uint32_t lo, uint32_t hi, StepScratch* __restrict__ sc) {
    const uint32_t ng = group_ctr[1];
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
        const uint32_t f = groups[g].x;
        if (f >= lo && f < hi) atomicMax(&sc->shard_ma, n - f);
        if (f >= hi) atomicMax(&sc->shard_mb, n - f);
    }
}

__global__ void __launch_bounds__(kShardThreads)
shard_pack_kernel(const uint32_t* __restrict__ ids, const float2* __restrict__ pos,
                  const float2* __restrict__ vel, const float2* __restrict__ acc, uint32_t n,
                  int kdk, const StepScratch* __restrict__ sc, uint4* __restrict__ chunk,
                  uint32_t capacity, uint32_t* __restrict__ err) {
    const uint32_t ma = sc->shard_ma, mb = sc->shard_mb;
    const uint32_t a = n - ma, b = n - mb;  // no group: n
    uint32_t count = b > a ? b - a : 0u;
    if (count > capacity) count = 0u;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        chunk[0] = make_uint4(a, count, 0u, 0u);
        if (b > a && b - a > capacity) atomicOr(err, kErrShardCapacity);
    }
    float4* rec = reinterpret_cast<float4*>(chunk + 1);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint32_t body = ids[a + k];
        const float2 f0 = kdk ? vel[body] : pos[body];
        const float2 f1 = kdk ? acc[body] : vel[body];
        rec[k] = make_float4(f0.x, f0.y, f1.x, f1.y);
    }
}

__global__ void __launch_bounds__(kShardThreads)
shard_unpack_kernel(const uint32_t* __restrict__ ids, float2* __restrict__ pos,
                    float2* __restrict__ vel, float2* __restrict__ acc, uint32_t n, int kdk,
                    const uint4* __restrict__ chunks, uint32_t capacity, uint32_t* __restrict__ err) {
    const uint4* chunk = chunks + (size_t)blockIdx.y * (1u + capacity);
    const uint4 h = chunk[0];
    const uint32_t a = h.x, count = h.y;
    if (count > capacity || a > n || count > n - a) {
        if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(err, kErrShardCapacity);
        return;
    }
    const float4* rec = reinterpret_cast<const float4*>(chunk + 1);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint32_t body = ids[a + k];
        const float4 r = rec[k];
        if (kdk) {
            vel[body] = make_float2(r.x, r.y);
            acc[body] = make_float2(r.z, r.w);
        } else {
            pos[body] = make_float2(r.x, r.y);
            vel[body] = make_float2(r.z, r.w);
        }
    }
}

static uint32_t grid_for(uint32_t items, int device_sms) {
    uint32_t blocks = (items + kShardThreads - 1) / kShardThreads;
    const uint32_t cap = (uint32_t)device_sms * 8u;
    if (blocks > cap) blocks = cap;
    return blocks ? blocks : 1u;
}

static int sm_count() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

void launch_shard_pack(const DeviceBuffers& b, uint32_t lo, uint32_t hi, int kdk, void* chunk,
                       uint32_t capacity, cudaStream_t s) {
    if (!b.groups || b.n == 0) return;
    const int sms = sm_count();
    shard_bounds_kernel<<<grid_for(b.n / 32u + 1u, sms), kShardThreads, 0, s>>>(
        b.groups, b.scratch->group_ctr, b.n, lo, hi, b.scratch);
    shard_pack_kernel<<<grid_for(capacity, sms), kShardThreads, 0, s>>>(
        b.ids, b.pos, b.vel, b.acc, b.n, kdk, b.scratch, static_cast<uint4*>(chunk), capacity,
        b.err);
}

void launch_shard_unpack(const DeviceBuffers& b, int kdk, const void* chunks, uint32_t nchunks,
                         uint32_t capacity, cudaStream_t s) {
    if (b.n == 0 || nchunks == 0) return;
    const dim3 grid(grid_for(capacity, sm_count() / 2 + 1), nchunks);
    shard_unpack_kernel<<<grid, kShardThreads, 0, s>>>(b.ids, b.pos, b.vel, b.acc, b.n, kdk,
                                                       static_cast<const uint4*>(chunks), capacity,
                                                       b.err);
}

}  // namespace bh
