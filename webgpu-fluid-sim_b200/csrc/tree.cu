// tree.cu -- launches the fused hierarchy build + fill for the engine's step.
// The kernel and its derivation are in tree_kernel.cuh.
#include "tree_kernel.cuh"

namespace bh {

void init_bound(const DeviceBuffers& b, cudaStream_t s) {
    if (b.n > 1) cudaMemsetAsync(b.bound, 0xFF, sizeof(uint32_t) * (b.n - 1), s);
}

void launch_build_fill(const DeviceBuffers& b, int fp64_levels, cudaStream_t s) {
    if (b.n == 0) return;
    const int blocks = (int)((b.n + 255) / 256);
    if (b.key_bytes == 8)
        build_fill_kernel<uint64_t><<<blocks, 256, 0, s>>>(
            (const uint64_t*)b.codes, b.ids, b.mass, b.pos, b.node4, b.children, b.parent, b.aabb,
            b.range, b.big, b.bound, b.n, fp64_levels, b.gnode, b.groups,
            b.groups ? &b.scratch->group_ctr[1] : nullptr, b.group_max);
    else
        build_fill_kernel<uint32_t><<<blocks, 256, 0, s>>>(
            (const uint32_t*)b.codes, b.ids, b.mass, b.pos, b.node4, b.children, b.parent, b.aabb,
            b.range, b.big, b.bound, b.n, fp64_levels, b.gnode, b.groups,
            b.groups ? &b.scratch->group_ctr[1] : nullptr, b.group_max);
}

}  // namespace bh
