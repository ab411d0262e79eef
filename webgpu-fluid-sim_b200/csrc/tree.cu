// tree.cu -- launches the hierarchy build + fill for the engine's step: the
// block-local phase (build_fill_kernel<K, true>) and the climb of the
// frontier nodes it leaves (build_climb_kernel).  The kernels and their
// derivation are in tree_kernel.cuh.
#include "tree_kernel.cuh"

namespace bh {

bool split_build(uint32_t n, uint32_t debug_flags) {
    return n >= kSplitBuildMin || (n >= 2 && (debug_flags & kDebugSplitBuild));
}

template <typename K, bool SPLIT>
static cudaError_t set_build_attributes() {
    return cudaFuncSetAttribute(build_fill_kernel<K, SPLIT>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(BuildShared<K, build_block<SPLIT>()>));
}

// Allow the build kernels their shared memory (dynamic; once per device,
// before any launch or capture).
cudaError_t build_init_attributes() {
    cudaError_t e;
    if ((e = set_build_attributes<uint32_t, false>()) != cudaSuccess) return e;
    if ((e = set_build_attributes<uint32_t, true>()) != cudaSuccess) return e;
    if ((e = set_build_attributes<uint64_t, false>()) != cudaSuccess) return e;
    return set_build_attributes<uint64_t, true>();
}

void init_bound(const DeviceBuffers& b, cudaStream_t s) {
    if (b.n > 1) cudaMemsetAsync(b.bound, 0xFF, sizeof(uint32_t) * (b.n - 1), s);
}

template <typename K>
static void launch_typed(const DeviceBuffers& b, int fp64_levels, cudaStream_t s) {
    BuildArgs<K> a;
    a.keys = (const K*)b.codes;
    a.ids = b.ids;
    a.mass = b.mass;
    a.pos = b.pos;
    a.node4 = b.node4;
    a.children = b.children;
    a.parent = b.parent;
    a.aabb = b.aabb;
    a.range = b.range;
    a.big = b.big;
    a.bound = b.bound;
    a.n = b.n;
    a.fp64 = fp64_levels;
    a.gnode = b.gnode;
    a.groups = b.groups;
    a.group_count = b.groups ? &b.scratch->group_ctr[1] : nullptr;
    a.gmax = b.group_max;
    a.xm = b.xm;
    a.err = b.err;
    if (!split_build(b.n, b.debug_flags)) {
        constexpr uint32_t B = build_block<false>();
        build_fill_kernel<K, false><<<(b.n + B - 1) / B, B, sizeof(BuildShared<K, B>), s>>>(a);
        return;
    }
    a.frontier = b.frontier;
    a.frontier_count = &b.scratch->frontier_ctr;
    constexpr uint32_t B = build_block<true>();
    const uint32_t grid = (b.n + B - 1) / B;
    build_fill_kernel<K, true><<<grid, B, sizeof(BuildShared<K, B>), s>>>(a);
    // Frontier nodes number far fewer than bodies (a handful per CTA), but
    // only the device knows how many: a resident grid strides over them.
    static int blocks_per_sm[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    int& bps = blocks_per_sm[dev & 63];
    if (bps == 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, build_climb_kernel<K>, kClimbBlock, 0);
        if (bps < 1) bps = 1;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint32_t blocks = (uint32_t)(sms * bps);
    if (blocks > grid) blocks = grid;
    build_climb_kernel<K><<<blocks, kClimbBlock, 0, s>>>(a);
}

// Reference-layout internal-node arrays from the packed records: node4
// {com, mass, length}, aabb, children {left, right} and the slot range.
static __global__ void __launch_bounds__(256)
ref_layout_kernel(const GNode* __restrict__ gnode, uint32_t ni, float4* __restrict__ node4,
                  float4* __restrict__ aabb, uint2* __restrict__ children, uint2* __restrict__ range) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < ni; v += gridDim.x * blockDim.x) {
        const float4 box = __ldg(&gnode[v].box);
        const float4 mom = __ldg(&gnode[v].mom);
        const uint4 lk = __ldg(&gnode[v].link);
        node4[v] = mom;
        aabb[v] = box;
        children[v] = make_uint2(lk.x, lk.y);
        range[v] = make_uint2(lk.z, lk.z + lk.w - 1u);
    }
}

void launch_ref_layout(const DeviceBuffers& b, cudaStream_t s) {
    if (!b.gnode || b.n < 2) return;
    const uint32_t ni = b.n - 1;
    int blocks = (int)((ni + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    ref_layout_kernel<<<blocks, 256, 0, s>>>(b.gnode, ni, b.node4, b.aabb, b.children, b.range);
}

void launch_build_fill(const DeviceBuffers& b, int fp64_levels, cudaStream_t s) {
    if (b.n == 0) return;
    if (b.key_bytes == 8) launch_typed<uint64_t>(b, fp64_levels, s);
    else launch_typed<uint32_t>(b, fp64_levels, s);
}

}  // namespace bh
