// bh_internal.cuh -- device data layout and kernel launchers of the engine.
//
// Stage map (reference: src/simulation.ts:394-420, one step):
//   morton.cu  bounding box (extension) + Morton encode + digit histograms
//   sort.cu    onesweep LSD radix sort of (key, id) pairs
//   tree.cu    fused bottom-up hierarchy build + mass/COM/AABB fill
//   walk.cu    warp-cooperative theta-criterion walk + kick (+ drift)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace bh {

constexpr uint32_t kSentinel = 0xFFFFFFFFu;
constexpr int kStackSize = 256;  // barnes_hut.wgsl:67
// Nodes with at least this many bodies aggregate mass/COM in FP64.
#ifndef BH_FP64_MIN_BODIES
#define BH_FP64_MIN_BODIES 1024
#endif
constexpr uint32_t kFp64MinBodies = BH_FP64_MIN_BODIES;

// Sort tiling (a tile is kSortThreads x kSortItems keys).
#ifndef BH_SORT_THREADS
#define BH_SORT_THREADS 512
#endif
#ifndef BH_SORT_ITEMS
#define BH_SORT_ITEMS 12
#endif
constexpr int kSortThreads = BH_SORT_THREADS;
constexpr int kSortItems = BH_SORT_ITEMS;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadixBits = 8;
constexpr int kRadix = 256;

// Device error word bits (read by the host after a sync).
constexpr uint32_t kErrLookbackSpin = 1u << 0;  // decoupled look-back gave up waiting
constexpr uint32_t kErrStackOverflow = 1u << 1; // walk stack would have overflowed (children dropped)
constexpr uint32_t kErrTreeSpin = 1u << 2;
// Failures after which the rest of a step has no valid input: the build and
// the walk then skip their work for that step instead of consuming it.
constexpr uint32_t kErrSkipMask = kErrLookbackSpin;
// Default spins of the sort's bounded look-back wait (several seconds).
constexpr uint32_t kSpinCapDefault = 1u << 22;
// Test hook: the second tile of the first sort pass waits on a predecessor
// status that never reads as published, so its bounded wait runs out.
constexpr uint32_t kDebugLookbackUnpublished = 1u << 0;
// the split hierarchy build (local phase + frontier climb) at every body count from 2
constexpr uint32_t kDebugSplitBuild = 1u << 1;

// Packed internal-node record of the group walk (64 B, one per internal node):
// the criterion reads `box`, an accepted node contributes `mom` + `quad`, an
// opened node continues through `link`.
struct __align__(16) GNode {
    float4 box;   // {min.x, min.y, max.x, max.y}
    float4 mom;   // {com.x, com.y, mass, length}
    float4 quad;  // raw second moments about the COM {Sxx, Sxy, Syy, 0}
    uint4 link;   // {left, right, first slot, body count}
};

// Group acceptance test.  A node stands in for its bodies, as one multipole,
// for a whole group when its size L and the distance d from the group's box
// to the node's centre of mass satisfy L < theta d -- then every body of the
// group meets the per-body test length / d_body < theta -- and the node's box
// lies apart from the group's box.  Every operation rounds to nearest (no
// contraction), so a CPU restatement reproduces each decision.
__device__ __forceinline__ bool group_accepts(const float4& box, float cx, float cy, float glox,
                                              float gloy, float ghix, float ghiy, float th2) {
    const float dx = fmaxf(0.0f, fmaxf(__fsub_rn(cx, ghix), __fsub_rn(glox, cx)));
    const float dy = fmaxf(0.0f, fmaxf(__fsub_rn(cy, ghiy), __fsub_rn(gloy, cy)));
    const float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
    const float L = fmaxf(__fsub_rn(box.z, box.x), __fsub_rn(box.w, box.y));
    const float sx = fmaxf(__fsub_rn(box.x, ghix), __fsub_rn(glox, box.z));
    const float sy = fmaxf(__fsub_rn(box.y, ghiy), __fsub_rn(gloy, box.w));
    return __fmul_rn(L, L) < __fmul_rn(th2, d2) && (sx > 0.0f || sy > 0.0f);
}

// True when an earlier stage of this step left no valid input (its bounded
// wait gave up, kErrSkipMask); the build and the walk then skip their work.
__device__ __forceinline__ bool step_failed(const uint32_t* err) {
    return err && (__ldcg(err) & kErrSkipMask) != 0u;
}

// Reciprocal square root with subnormal inputs flushed to zero, which drops
// the subnormal-input handling around each hardware rsqrt.  It changes a
// result only for |r|^2 + eps^2 below 1.2e-38 (coincident bodies without
// softening), where the force is not finite either way.
__device__ __forceinline__ float rsqrt_ftz(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
// Group-walk stack and list capacities (per warp).
constexpr int kGroupStack = 1024;
constexpr int kGroupDfsAt = kGroupStack - 128;  // switch to one node per step above this depth
constexpr int kGroupList = 64;
constexpr int kGroupMaxLeaf = 8;                // leaf_size cap of the group walk
constexpr uint32_t kErrGroupStack = 1u << 3;    // group-walk stack overflow (never expected)
constexpr uint32_t kErrShardCapacity = 1u << 4; // a shard's updated range exceeded its chunk

// Walk modes.
enum WalkMode : int {
    kWalkForces = 0,       // acc[b] = a
    kWalkEulerKickDrift,   // v += a*dt; x += v*dt (reference, barnes_hut.wgsl:110,119-120)
    kWalkKdkClose,         // v += a*dt/2; acc[b] = a (leapfrog closing kick)
};

struct WalkParams {
    uint32_t n;
    float g;
    float theta;
    float dt;
    float eps_coef;   // reference softening: eps^2 = eps_coef * max(m1, m2)
    float eps2;       // Plummer softening: eps^2 (constant)
    int plummer;      // 1 = Plummer
    int leaf_size;    // bucket size (1 = reference walk)
    int mode;         // WalkMode
    int count;        // 1 = instrumented launch: accumulate visit/interaction counters
    unsigned long long* counters;  // exact walk: {node visits, interactions};
                                   // group walk: {node visits, node interactions, body interactions}
    // group walk
    int multipole;    // 1 or 2
    int bpl;          // bodies per lane
    unsigned int* group_ctr;  // dynamic group counter (zeroed per step)
    // ensemble: a group only sees its own system's slot range
    uint32_t num_systems;
    const uint32_t* sys_off;
    // sharding: only groups whose first sorted slot lies in [slot_lo, slot_hi)
    uint32_t slot_lo;
    uint32_t slot_hi;
    // stack entries a warp may use (0 = the kernel's full capacity); a test
    // lowers it to make the overflow check trip
    int stack_cap = 0;
    // group walk, Plummer softening: far_alpha^2 (0 = no far field); an
    // accepted node with r_g^2 < far_alpha^2 R^2 goes through the group's
    // local expansion (far_field.cuh)
    float far_alpha2 = 0.0f;
};

// Per-step scratch that must start at zero.  One memset clears it.
struct StepScratch {
    uint32_t hist[8][kRadix];  // digit histograms per pass
    uint32_t tile_ctr[8];      // dynamic tile counters per pass
    uint32_t bbox[4];          // ordered-int max of {-minx, -miny, maxx, maxy} (see morton.cu)
    unsigned long long walk_counts[4];  // instrumented walk counters
    unsigned int group_ctr[4];          // group walk: [0] work counter, [1] number of groups
    unsigned int frontier_ctr;          // hierarchy build: frontier nodes of the local phase
    unsigned int shard_ma, shard_mb;    // sharding: n - (first / next group start), max-reduced
};

struct DeviceBuffers {
    uint32_t n = 0;
    uint32_t capacity = 0;  // bodies allocated
    int key_bytes = 4;      // 4 or 8
    // bodies, original order (simulation.ts:82-87)
    float* mass = nullptr;
    float2* pos = nullptr;
    float2* vel = nullptr;
    float2* acc = nullptr;
    float* radius = nullptr;
    float4* xm = nullptr;   // {x, y, m, 0} per body (original order), written by the encode
    // sort
    void* codes = nullptr;      // sorted keys after a step
    void* codes_alt = nullptr;
    uint32_t* ids = nullptr;    // sorted permutation after a step
    uint32_t* ids_alt = nullptr;
    // tree
    float4* node4 = nullptr;     // 2n-1 {com.x, com.y, mass, length}
    uint2* children = nullptr;   // n-1 {left, right}
    uint32_t* parent = nullptr;  // 2n-1
    float4* aabb = nullptr;      // n-1 {min.x, min.y, max.x, max.y}
    uint2* range = nullptr;      // n-1 {first slot, last slot}
    double2* big = nullptr;      // 2(n-1) FP64 {mass, mass*x}, {mass*y, 0} for big nodes
    uint32_t* bound = nullptr;   // n-1 exchange slots, kSentinel between steps
    GNode* gnode = nullptr;      // n-1 packed records (group walk only; else null)
    uint2* groups = nullptr;     // n {first slot, count}: maximal subtrees of <= G bodies (group walk)
    uint32_t group_max = 0;      // G = 32 x bodies per lane (0: no groups)
    uint2* frontier = nullptr;   // n {first slot, last slot}: nodes left by the build's local phase
    // scratch
    StepScratch* scratch = nullptr;
    uint32_t* status = nullptr;  // look-back status: passes * tiles * 256
    uint32_t tiles = 0;
    uint32_t* err = nullptr;     // device error word
    uint32_t spin_cap = kSpinCapDefault;  // sort look-back wait bound (spins)
    uint32_t debug_flags = 0;    // kDebug* test hooks
    int sort_passes = 0;         // 0: one per key byte; ensembles sort fewer (even count)
    // ensemble of independent systems (num_systems = 0: one system)
    uint32_t num_systems = 0;
    const uint32_t* sys_off = nullptr;  // E+1 body offsets (original order = sorted order by system)
    const uint32_t* body_sys = nullptr; // n: system of each body (original order)
    uint32_t* sys_bbox = nullptr;       // 4E ordered-int max of {-minx, -miny, maxx, maxy}
};

// Body buffers of a simulation handle (renderer, diagnostics).
struct BodyView {
    const float* mass = nullptr;
    const float2* pos = nullptr;
    const float2* vel = nullptr;
    const float* radius = nullptr;
    uint32_t n = 0;
    cudaStream_t stream = nullptr;
    int device = 0;
};

// ---- launchers (all asynchronous on `s`) --------------------------------
// morton.cu
void launch_bbox(const DeviceBuffers& b, cudaStream_t s);
// domain: 0 fixed2000, 1 bbox; key_bytes 4 or 8.
void launch_encode(const DeviceBuffers& b, int domain, cudaStream_t s);
// leapfrog opening kick + drift: v += a*hdt; x += v*dt (original order)
void launch_kick_drift(const DeviceBuffers& b, float dt, cudaStream_t s);
// ensemble: per-system boxes, and keys (system << 32) | morton32(system box)
void launch_bbox_ensemble(const DeviceBuffers& b, cudaStream_t s);
void launch_encode_ensemble(const DeviceBuffers& b, cudaStream_t s);
// sort.cu
void launch_zero_step(const DeviceBuffers& b, cudaStream_t s);  // scratch + sort status
void launch_sort(const DeviceBuffers& b, cudaStream_t s);
cudaError_t sort_init_attributes();
// walk_group.cu: the group walk's dynamic shared memory limit (per device),
// and its largest block (threads) for a bodies_per_lane
cudaError_t walk_init_attributes();
int walk_group_max_block(int bpl);
// tree.cu: the hierarchy build's dynamic shared memory limit (per device)
cudaError_t build_init_attributes();
int sort_passes(const DeviceBuffers& b);
// tree.cu
void launch_build_fill(const DeviceBuffers& b, int fp64_levels, cudaStream_t s);
// Bodies from which the build runs as two kernels (local phase + frontier climb).
// Measured crossover (tree stage, B200): 0.8M fused 0.137 / split 0.151 ms, 1.5M
// equal (0.211), 3M fused 0.371 / split 0.342, 4.2M 0.556 / 0.470.
#ifndef BH_SPLIT_BUILD_MIN
#define BH_SPLIT_BUILD_MIN (1u << 21)
#endif
constexpr uint32_t kSplitBuildMin = BH_SPLIT_BUILD_MIN;
bool split_build(uint32_t n, uint32_t debug_flags);
void launch_ref_layout(const DeviceBuffers& b, cudaStream_t s);  // group walk: node4/aabb/children/range on request
void init_bound(const DeviceBuffers& b, cudaStream_t s);
// walk.cu
void launch_walk(const DeviceBuffers& b, const WalkParams& p, int block, cudaStream_t s);
// walk_group.cu
void launch_walk_group(const DeviceBuffers& b, const WalkParams& p, int block, cudaStream_t s);
// shard.cu: the bodies a sharded step updated, packed / unpacked in sorted-slot order
void launch_shard_pack(const DeviceBuffers& b, uint32_t lo, uint32_t hi, int kdk, void* chunk,
                       uint32_t capacity, cudaStream_t s);
void launch_shard_unpack(const DeviceBuffers& b, int kdk, const void* chunks, uint32_t nchunks,
                         uint32_t capacity, cudaStream_t s);

}  // namespace bh
