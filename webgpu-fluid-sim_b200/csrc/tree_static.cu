// tree_static.cu -- hierarchy build + fill that allocates no device memory.
//
// Some callers cannot let this library call cudaMalloc: a host that plans all
// device memory itself (for example an embedding runtime that owns the GPU
// heap and hands out every buffer), a frame loop that cannot afford the
// implicit device-wide synchronisation of cudaMalloc/cudaFree, or code that
// must not allocate once it is running.  For them,
// bh_build_hierarchy_static() runs the same fused build + fill kernel as the
// engine's step (tree_kernel.cuh) on buffers the caller passes in, and keeps
// the kernel's scratch -- the split exchange slots, the FP64 mass/moment sums
// and the per-node slot ranges -- in the file-scope array below.
//
// Limits and sharing rules:
//  - at most kStaticMaxBodies bodies per call (the array is ~11.5 MB and
//    every GPU that loads the library holds it until the process exits);
//  - all calls share the one array, which keeps the last call's contents;
//    each call resets the exchange slots it uses before its launch, and the
//    other parts are written before they are read.  Calls whose kernels
//    overlap on the GPU (different streams, or different host threads on
//    the same device) race on the array: serialise them;
//  - every call looks up the array's device address on the current device
//    with cudaGetSymbolAddress (no cached pointer outlives a context reset);
//    under CUDA's lazy module loading the first call on a device may load
//    the library's module, which reserves the array and may synchronise, so
//    a caller that must not allocate while running makes one warm-up call
//    at start-up, and before any stream capture.
#include <cuda_runtime.h>

#include <string>

#include "bh.h"
#include "tree_kernel.cuh"

namespace bh {

void set_global_error(const std::string& msg);

constexpr uint32_t kStaticMaxBodies = 262144;
constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t v) { return (v + kAlign - 1) & ~(kAlign - 1); }
// Layout inside the array (internal nodes: kStaticMaxBodies - 1).
constexpr size_t kBoundOff = 0;
constexpr size_t kRangeOff = align_up(kBoundOff + sizeof(uint32_t) * (kStaticMaxBodies - 1));
constexpr size_t kBigOff = align_up(kRangeOff + sizeof(uint2) * (kStaticMaxBodies - 1));
constexpr size_t kScratchBytes = align_up(kBigOff + 2 * sizeof(double2) * (kStaticMaxBodies - 1));

static __device__ __align__(256) unsigned char g_tree_scratch[kScratchBytes];

// Device address of g_tree_scratch in the current context.  Looked up on
// every call: cheap once the module is loaded, and never stale after a
// cudaDeviceReset or a new primary context.
static cudaError_t scratch_address(unsigned char** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_tree_scratch);
    if (e != cudaSuccess) return e;
    *out = static_cast<unsigned char*>(p);
    return cudaSuccess;
}

template <typename K>
static void launch_static(const void* codes, const uint32_t* ids, const float* mass,
                          const float* pos, uint32_t n, float* node4, uint32_t* children,
                          uint32_t* parent, float* aabb, uint2* range, double2* big,
                          uint32_t* bound, int fp64, cudaStream_t s) {
    BuildArgs<K> a;
    a.keys = static_cast<const K*>(codes);
    a.ids = ids;
    a.mass = mass;
    a.pos = reinterpret_cast<const float2*>(pos);
    a.node4 = reinterpret_cast<float4*>(node4);
    a.children = reinterpret_cast<uint2*>(children);
    a.parent = parent;
    a.aabb = reinterpret_cast<float4*>(aabb);
    a.range = range;
    a.big = big;
    a.bound = bound;
    a.n = n;
    a.fp64 = fp64;
    a.gnode = nullptr;
    a.groups = nullptr;
    a.group_count = nullptr;
    a.gmax = 0u;
    constexpr uint32_t B = build_block<false>();
    build_fill_kernel<K, false><<<(n + B - 1) / B, B, sizeof(BuildShared<K, B>), s>>>(a);
}

}  // namespace bh

static int static_fail(int code, const std::string& msg) {
    bh::set_global_error(msg);
    return code;
}

extern "C" int bh_build_hierarchy_static(const void* sorted_codes, int32_t morton_bits,
                                         const uint32_t* sorted_ids, const float* mass,
                                         const float* pos, uint32_t n, float* node4,
                                         uint32_t* node_children, uint32_t* node_parent,
                                         float* node_aabb, int32_t fp64_levels, void* stream) {
    using namespace bh;
    if (morton_bits != 32 && morton_bits != 64)
        return static_fail(BH_ERR_INVALID_ARGUMENT, "bh_build_hierarchy_static: morton_bits must be 32 or 64");
    if (n > kStaticMaxBodies)
        return static_fail(BH_ERR_INVALID_ARGUMENT,
                           "bh_build_hierarchy_static: " + std::to_string(n) +
                               " bodies exceed the static scratch limit of " +
                               std::to_string(kStaticMaxBodies));
    if (n == 0) return BH_OK;
    if (!sorted_codes || !sorted_ids || !mass || !pos || !node4 || !node_parent ||
        (n > 1 && (!node_children || !node_aabb)))
        return static_fail(BH_ERR_INVALID_ARGUMENT, "bh_build_hierarchy_static: null buffer");
    unsigned char* base = nullptr;
    cudaError_t e = scratch_address(&base);
    if (e != cudaSuccess)
        return static_fail(BH_ERR_CUDA, std::string("cudaGetSymbolAddress(static tree scratch): ") +
                                            cudaGetErrorString(e));
    uint32_t* bound = reinterpret_cast<uint32_t*>(base + kBoundOff);
    uint2* range = reinterpret_cast<uint2*>(base + kRangeOff);
    double2* big = reinterpret_cast<double2*>(base + kBigOff);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The exchange slots must start at kSentinel (the previous call may have
    // been cut short by an error).
    if (n > 1) {
        e = cudaMemsetAsync(bound, 0xFF, sizeof(uint32_t) * (n - 1), s);
        if (e != cudaSuccess)
            return static_fail(BH_ERR_CUDA, std::string("cudaMemsetAsync(static exchange slots): ") +
                                                cudaGetErrorString(e));
    }
    if (morton_bits == 64)
        launch_static<uint64_t>(sorted_codes, sorted_ids, mass, pos, n, node4, node_children,
                                node_parent, node_aabb, range, big, bound, fp64_levels, s);
    else
        launch_static<uint32_t>(sorted_codes, sorted_ids, mass, pos, n, node4, node_children,
                                node_parent, node_aabb, range, big, bound, fp64_levels, s);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return static_fail(BH_ERR_CUDA, std::string("build_fill_kernel launch: ") + cudaGetErrorString(e));
    return BH_OK;
}
