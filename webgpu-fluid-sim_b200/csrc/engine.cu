// engine.cu -- the C ABI of include/bh.h: handle lifetime, device buffers,
// stream-ordered steps replayed from CUDA graphs, profiling and errors.
//
// Reference host class: Simulation (src/simulation.ts:39-433).  Buffers
// (:68-104), scenario set-up (:227-374), metadata (:212-225) and the per-frame
// command encoding (:386-425) map onto bh_create / bh_set_* / bh_step here.
#include <cuda_runtime.h>

#include <cstdio>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "bh.h"
#include "bh_internal.cuh"

namespace bh {
int generate_scenario(const char* name, uint32_t n, uint64_t seed, float grav_constant,
                      float* mass, float* pos, float* vel, float* radius_mul);
}

using bh::DeviceBuffers;

static constexpr int kMarkers = 6;  // stage boundaries of one step
static constexpr uint32_t kMaxBodies = (1u << 30) - 1;

struct bh_sim {
    bh_config cfg{};
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t n = 50000;  // simulation.ts:60
    std::string scenario = "default";
    uint64_t seed = 0;
    bool device_gen = false;  // the scenario comes from the GPU generators
    // sharding: the step's walk integrates only groups starting in these slots
    uint32_t shard_lo = 0, shard_hi = 0xFFFFFFFFu;
    // test hooks of the device-side checks (bh_debug_set_limits): 0 = defaults
    uint32_t debug_flags = 0, debug_spin_cap = 0, debug_stack_cap = 0;
    DeviceBuffers b;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    bool acc_valid = false;
    // graphs: [0] plain, [1] with event-record nodes at the stage boundaries;
    // for the first step after an upload still being copied (see bh_upload):
    // [2] the tree stages, [3] the walk, [4] the tree stages up to the sort
    // without packed leaf records, [5] the build reading masses and positions
    static constexpr int kGraphs = 6;
    cudaGraph_t graph[kGraphs] = {};
    cudaGraphExec_t exec[kGraphs] = {};
    // Uploads are staged: bh_upload copies each array into its staging
    // buffer on copy_stream as soon as the last staged copy of that array has
    // been moved out (Staged::freed), so the copy may overlap steps still
    // running; the handle's stream waits on Staged::landed and moves the
    // array into place before its next reader (settle_*).
    cudaStream_t copy_stream = nullptr;
    struct Staged {
        void* buf = nullptr;  // staging buffer (in the arena)
        size_t width = 0;     // bytes per body
        cudaEvent_t landed = nullptr, freed = nullptr;
        mutable bool pending = false;
    };
    enum { kPos = 0, kMass = 1, kVel = 2 };
    Staged up[3];
    // bh_download_async: the requested arrays are copied on the handle's
    // stream into a device snapshot (ev_snap_ready), and from there to the
    // host on d2h_stream (ev_snap_free), so the next steps need not wait for
    // the host copy.
    float* snap_mass = nullptr;
    float2 *snap_pos = nullptr, *snap_vel = nullptr;
    cudaStream_t d2h_stream = nullptr;
    cudaEvent_t ev_snap_ready = nullptr, ev_snap_free = nullptr;
    mutable bool snap_busy = false;
    cudaGraphNode_t ev_node[kMarkers] = {};
    cudaEvent_t markers[kMarkers] = {};
    // profiling
    bool profiling = false;
    uint32_t prof_max = 0, prof_used = 0;
    std::vector<cudaEvent_t> prof_ev;
    // adjoint (bh_force_vjp / bh_rollout_grad), allocated on first use
    struct Adjoint {
        void* arena = nullptr;
        uint32_t n = 0, nck = 0, seg = 0;
        float* node_adj = nullptr;
        float2 *xbar_slot = nullptr, *abar = nullptr, *xbar = nullptr, *vbar = nullptr,
               *apend = nullptr, *target = nullptr, *ck_pos = nullptr, *ck_vel = nullptr,
               *seg_pos = nullptr, *fin_pos = nullptr, *fin_vel = nullptr;
        float *mbar_slot = nullptr, *mbar = nullptr;
        double* loss = nullptr;
        // Trees of one replayed segment, one record per step (null when the
        // segment does not fit the memory budget: the reverse sweep then
        // rebuilds each tree).
        void* slab = nullptr;
        size_t slab_stride = 0;
        uint32_t slab_steps = 0;
    } adj;
    // ensemble of independent systems (empty: one system)
    std::vector<uint32_t> sys_sizes;
    std::string err;
    uint32_t* err_host = nullptr;  // page-locked copy of the device error word
};

static thread_local std::string g_err;

// Order the handle's stream after uploads still in flight on the copy
// stream.  Every entry point calls settle_uploads (through BH_HANDLE) before
// it touches the body buffers, except bh_upload and bh_step, which order the
// copies themselves.
// Returns the first CUDA error; the array stays pending unless all three
// calls were enqueued.
static cudaError_t settle(const bh_sim* s, int k, void* dst) {
    const bh_sim::Staged& u = s->up[k];
    if (!u.pending) return cudaSuccess;
    cudaError_t e = cudaStreamWaitEvent(s->stream, u.landed, 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dst, u.buf, u.width * (size_t)s->b.n, cudaMemcpyDeviceToDevice, s->stream);
    if (e == cudaSuccess) e = cudaEventRecord(u.freed, s->stream);
    if (e == cudaSuccess) u.pending = false;
    return e;
}
static cudaError_t settle_pos(const bh_sim* s) { return settle(s, bh_sim::kPos, s->b.pos); }
static cudaError_t settle_mass(const bh_sim* s) { return settle(s, bh_sim::kMass, s->b.mass); }
static cudaError_t settle_vel(const bh_sim* s) { return settle(s, bh_sim::kVel, s->b.vel); }
static cudaError_t settle_uploads(const bh_sim* s) {
    cudaError_t e = settle_pos(s);
    if (e == cudaSuccess) e = settle_mass(s);
    if (e == cudaSuccess) e = settle_vel(s);
    return e;
}

namespace bh {
// Message for bh_global_last_error() from entry points without a handle.
void set_global_error(const std::string& msg) { g_err = msg; }
}  // namespace bh

namespace bh {
// The handle's body buffers without side effects (bh_get_buffers also
// refreshes the reference node layout); false for a null handle.
bool sim_body_view(const bh_sim* s, BodyView* out) {
    if (!s || !out) return false;
    cudaSetDevice(s->device);  // settling may copy staged positions on the handle's stream
    // Callers use the buffers on the handle's stream.  A settling error (a
    // broken context) also fails their own launches, which report it; the
    // view is filled either way so no caller sees null buffers.
    settle_uploads(s);
    out->mass = s->b.mass;
    out->pos = s->b.pos;
    out->vel = s->b.vel;
    out->radius = s->b.radius;
    out->n = s->b.n;
    out->stream = s->stream;
    out->device = s->device;
    return true;
}
}  // namespace bh

static int fail(bh_sim* s, int code, const std::string& msg) {
    if (s) s->err = msg;
    g_err = msg;
    return code;
}

static int cuda_fail(bh_sim* s, cudaError_t e, const char* what) {
    int code = (e == cudaErrorMemoryAllocation) ? BH_ERR_OUT_OF_MEMORY : BH_ERR_CUDA;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) code = BH_ERR_NO_DEVICE;
    return fail(s, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define BH_CUDA(s, expr)                                 \
    do {                                                 \
        cudaError_t _e = (expr);                         \
        if (_e != cudaSuccess) return cuda_fail(s, _e, #expr); \
    } while (0)

// ---- configuration --------------------------------------------------------

extern "C" int bh_default_config(bh_config* out) {
    if (!out) return fail(nullptr, BH_ERR_INVALID_ARGUMENT, "bh_default_config: null output");
    std::memset(out, 0, sizeof(*out));
    // config.ts:10-14
    out->grav_constant = 1.0f;
    out->bh_theta = 0.6f;
    out->substeps = 1;
    out->delta_time = (float)(0.1 * 1.0 / (60.0 * 1.0));
    out->epsilon_multiplier = 1.0f;
    out->softening = BH_SOFTENING_REFERENCE;
    out->plummer_eps = 1e-3f;
    out->morton_bits = 32;
    out->morton_domain = BH_DOMAIN_FIXED2000;
    out->integrator = BH_INTEGRATOR_SYMPLECTIC_EULER;
    out->leaf_size = 1;
    out->walk_block = 0;
    out->device = 0;
    out->use_graphs = 1;
    out->fp64_levels = 1;
    out->walk_mode = BH_WALK_EXACT;
    out->multipole_order = 2;
    out->bodies_per_lane = 2;
    return BH_OK;
}

static int validate_config(bh_sim* s, const bh_config& c) {
    if (c.morton_bits != 32 && c.morton_bits != 64)
        return fail(s, BH_ERR_INVALID_ARGUMENT, "morton_bits must be 32 or 64");
    if (c.morton_domain != BH_DOMAIN_FIXED2000 && c.morton_domain != BH_DOMAIN_BBOX)
        return fail(s, BH_ERR_INVALID_ARGUMENT, "unknown morton_domain");
    if (c.softening != BH_SOFTENING_REFERENCE && c.softening != BH_SOFTENING_PLUMMER)
        return fail(s, BH_ERR_INVALID_ARGUMENT, "unknown softening");
    if (c.integrator != BH_INTEGRATOR_SYMPLECTIC_EULER && c.integrator != BH_INTEGRATOR_LEAPFROG_KDK)
        return fail(s, BH_ERR_INVALID_ARGUMENT, "unknown integrator");
    if (c.substeps < 1) return fail(s, BH_ERR_INVALID_ARGUMENT, "substeps must be >= 1");
    if (c.leaf_size < 1 || c.leaf_size > 64)
        return fail(s, BH_ERR_INVALID_ARGUMENT, "leaf_size must be in [1, 64]");
    if (c.walk_mode == BH_WALK_GROUP && c.leaf_size > bh::kGroupMaxLeaf)
        return fail(s, BH_ERR_INVALID_ARGUMENT, "leaf_size must be <= 8 with the group walk");
    if (c.walk_mode != BH_WALK_EXACT && c.walk_mode != BH_WALK_GROUP)
        return fail(s, BH_ERR_INVALID_ARGUMENT, "unknown walk_mode");
    if (c.walk_mode == BH_WALK_GROUP && c.multipole_order != 1 && c.multipole_order != 2)
        return fail(s, BH_ERR_INVALID_ARGUMENT, "multipole_order must be 1 or 2");
    if (c.walk_mode == BH_WALK_GROUP && c.bodies_per_lane != 0 && c.bodies_per_lane != 1 &&
        c.bodies_per_lane != 2 && c.bodies_per_lane != 4)
        return fail(s, BH_ERR_INVALID_ARGUMENT, "bodies_per_lane must be 1, 2 or 4");
    if (c.walk_block != 0 && c.walk_block != 64 && c.walk_block != 128 && c.walk_block != 256)
        return fail(s, BH_ERR_INVALID_ARGUMENT, "walk_block must be 0, 64, 128 or 256");
    if (!(c.far_alpha >= 0.0f && c.far_alpha <= 0.5f))
        return fail(s, BH_ERR_INVALID_ARGUMENT, "far_alpha must be in [0, 0.5]");
    if (!(c.delta_time == c.delta_time) || !(c.bh_theta >= 0.0f))
        return fail(s, BH_ERR_INVALID_ARGUMENT, "delta_time must be a number and bh_theta >= 0");
    return BH_OK;
}

// ---- buffers --------------------------------------------------------------

static void destroy_graphs(bh_sim* s) {
    for (int v = 0; v < bh_sim::kGraphs; ++v) {
        if (s->exec[v]) cudaGraphExecDestroy(s->exec[v]);
        if (s->graph[v]) cudaGraphDestroy(s->graph[v]);
        s->exec[v] = nullptr;
        s->graph[v] = nullptr;
    }
}

static void free_adjoint(bh_sim* s) {
    if (s->adj.arena) cudaFree(s->adj.arena);
    if (s->adj.slab) cudaFree(s->adj.slab);
    s->adj = bh_sim::Adjoint();
}

// Per-step record of the slab: what the force VJP reads of a tree.
struct TreeRecord {
    size_t gnode, node4, groups, ids, parent, ctr, bytes;
};

static TreeRecord tree_record(uint32_t n) {
    const size_t nn = n ? 2 * (size_t)n - 1 : 1, ni = n > 1 ? (size_t)n - 1 : 1, nb = n ? n : 1;
    auto up = [](size_t v) { return (v + 255) & ~(size_t)255; };
    TreeRecord r;
    r.gnode = 0;
    r.node4 = up(r.gnode + sizeof(bh::GNode) * ni);  // full node4 extent; only the leaves are copied
    r.groups = up(r.node4 + sizeof(float4) * nn);
    r.ids = up(r.groups + sizeof(uint2) * nb);
    r.parent = up(r.ids + sizeof(uint32_t) * nb);
    r.ctr = up(r.parent + sizeof(uint32_t) * nn);
    r.bytes = up(r.ctr + 4 * sizeof(unsigned int));
    return r;
}

// Device buffers whose tree (and walk work counters) come from slab record k.
static DeviceBuffers slab_view(bh_sim* s, uint32_t k) {
    const TreeRecord r = tree_record(s->b.n);
    char* base = (char*)s->adj.slab + (size_t)k * s->adj.slab_stride;
    DeviceBuffers bb = s->b;
    bb.gnode = (bh::GNode*)(base + r.gnode);
    bb.node4 = (float4*)(base + r.node4);
    bb.groups = (uint2*)(base + r.groups);
    bb.ids = (uint32_t*)(base + r.ids);
    bb.parent = (uint32_t*)(base + r.parent);
    return bb;
}

// Save the tree just built by a step into slab record k.
static int save_tree(bh_sim* s, uint32_t k) {
    const uint32_t n = s->b.n;
    const TreeRecord r = tree_record(n);
    char* base = (char*)s->adj.slab + (size_t)k * s->adj.slab_stride;
    const DeviceBuffers& b = s->b;
    cudaStream_t st = s->stream;
    const size_t nm1 = n - 1;
    if (n > 1) BH_CUDA(s, cudaMemcpyAsync(base + r.gnode, b.gnode, sizeof(bh::GNode) * nm1, cudaMemcpyDeviceToDevice, st));
    BH_CUDA(s, cudaMemcpyAsync(base + r.node4 + sizeof(float4) * nm1, b.node4 + nm1, sizeof(float4) * (size_t)n,
                               cudaMemcpyDeviceToDevice, st));
    BH_CUDA(s, cudaMemcpyAsync(base + r.groups, b.groups, sizeof(uint2) * (size_t)n, cudaMemcpyDeviceToDevice, st));
    BH_CUDA(s, cudaMemcpyAsync(base + r.ids, b.ids, sizeof(uint32_t) * (size_t)n, cudaMemcpyDeviceToDevice, st));
    BH_CUDA(s, cudaMemcpyAsync(base + r.parent, b.parent, sizeof(uint32_t) * (2 * (size_t)n - 1),
                               cudaMemcpyDeviceToDevice, st));
    BH_CUDA(s, cudaMemcpyAsync(base + r.ctr, b.scratch->group_ctr, 4 * sizeof(unsigned int),
                               cudaMemcpyDeviceToDevice, st));
    return BH_OK;
}

static void free_buffers(bh_sim* s) {
    // no copy into or out of freed memory
    if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
    if (s->d2h_stream) cudaStreamSynchronize(s->d2h_stream);
    s->snap_busy = false;
    for (auto& u : s->up) {
        u.pending = false;
        u.buf = nullptr;
    }
    s->snap_pos = s->snap_vel = nullptr;
    s->snap_mass = nullptr;
    destroy_graphs(s);
    free_adjoint(s);
    if (s->arena) cudaFree(s->arena);
    s->arena = nullptr;
    s->arena_bytes = 0;
    s->b = DeviceBuffers();
}

struct Carver {
    size_t off = 0;
    template <typename T>
    size_t take(size_t count) {
        size_t o = off;
        off += (count * sizeof(T) + 255) & ~(size_t)255;
        return o;
    }
};

static int alloc_buffers(bh_sim* s, uint32_t n) {
    free_buffers(s);
    const uint32_t E = (uint32_t)s->sys_sizes.size();
    // Ensembles key (system << 32) | 32-bit Morton code: 64-bit keys.
    const int kb = E ? 8 : s->cfg.morton_bits / 8;
    const size_t nn = n ? 2 * (size_t)n - 1 : 1, ni = n > 1 ? (size_t)n - 1 : 1, nb = n ? n : 1;
    const uint32_t tiles = (uint32_t)((n + bh::kSortTile - 1) / bh::kSortTile);
    Carver c;
    size_t o_mass = c.take<float>(nb), o_pos = c.take<float2>(nb), o_vel = c.take<float2>(nb);
    size_t o_acc = c.take<float2>(nb), o_rad = c.take<float>(nb), o_xm = c.take<float4>(nb);
    size_t o_codes = c.take<uint8_t>(nb * kb), o_codes2 = c.take<uint8_t>(nb * kb);
    size_t o_ids = c.take<uint32_t>(nb), o_ids2 = c.take<uint32_t>(nb);
    size_t o_node4 = c.take<float4>(nn), o_child = c.take<uint2>(ni), o_parent = c.take<uint32_t>(nn);
    size_t o_aabb = c.take<float4>(ni), o_range = c.take<uint2>(ni), o_big = c.take<double2>(2 * ni);
    size_t o_bound = c.take<uint32_t>(ni);
    size_t o_front = c.take<uint2>(nb);
    const bool group = s->cfg.walk_mode == BH_WALK_GROUP;
    size_t o_gnode = group ? c.take<bh::GNode>(ni) : 0;
    size_t o_groups = group ? c.take<uint2>(nb) : 0;
    size_t o_scr = c.take<bh::StepScratch>(1);
    size_t o_status = c.take<uint32_t>((size_t)kb * (tiles ? tiles : 1) * bh::kRadix);
    size_t o_err = c.take<uint32_t>(1);
    size_t o_soff = E ? c.take<uint32_t>(E + 1) : 0, o_bsys = E ? c.take<uint32_t>(nb) : 0;
    size_t o_sbox = E ? c.take<uint32_t>(4 * (size_t)E) : 0;
    // staged uploads and the asynchronous download's snapshot
    size_t o_stpos = c.take<float2>(nb), o_stmass = c.take<float>(nb), o_stvel = c.take<float2>(nb);
    size_t o_smass = c.take<float>(nb);
    size_t o_spos = c.take<float2>(nb), o_svel = c.take<float2>(nb);
    void* arena = nullptr;
    cudaError_t e = cudaMalloc(&arena, c.off);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(s, e, "cudaMalloc(body and tree buffers)");
    }
    s->arena = arena;
    s->arena_bytes = c.off;
    char* a = (char*)arena;
    DeviceBuffers& b = s->b;
    b.n = n;
    b.capacity = n;
    b.key_bytes = kb;
    b.mass = (float*)(a + o_mass);
    b.pos = (float2*)(a + o_pos);
    b.vel = (float2*)(a + o_vel);
    b.acc = (float2*)(a + o_acc);
    b.radius = (float*)(a + o_rad);
    b.xm = (float4*)(a + o_xm);
    b.codes = a + o_codes;
    b.codes_alt = a + o_codes2;
    b.ids = (uint32_t*)(a + o_ids);
    b.ids_alt = (uint32_t*)(a + o_ids2);
    b.node4 = (float4*)(a + o_node4);
    b.children = (uint2*)(a + o_child);
    b.parent = (uint32_t*)(a + o_parent);
    b.aabb = (float4*)(a + o_aabb);
    b.range = (uint2*)(a + o_range);
    b.big = (double2*)(a + o_big);
    b.bound = (uint32_t*)(a + o_bound);
    b.frontier = (uint2*)(a + o_front);
    b.gnode = group ? (bh::GNode*)(a + o_gnode) : nullptr;
    b.groups = group ? (uint2*)(a + o_groups) : nullptr;
    b.group_max = group ? 32u * (uint32_t)(s->cfg.bodies_per_lane > 0 ? s->cfg.bodies_per_lane : 2) : 0u;
    b.scratch = (bh::StepScratch*)(a + o_scr);
    b.status = (uint32_t*)(a + o_status);
    b.tiles = tiles;
    b.err = (uint32_t*)(a + o_err);
    b.spin_cap = s->debug_spin_cap ? s->debug_spin_cap : bh::kSpinCapDefault;
    b.debug_flags = s->debug_flags;
    s->up[bh_sim::kPos].buf = a + o_stpos;
    s->up[bh_sim::kPos].width = sizeof(float2);
    s->up[bh_sim::kMass].buf = a + o_stmass;
    s->up[bh_sim::kMass].width = sizeof(float);
    s->up[bh_sim::kVel].buf = a + o_stvel;
    s->up[bh_sim::kVel].width = sizeof(float2);
    s->snap_mass = (float*)(a + o_smass);
    s->snap_pos = (float2*)(a + o_spos);
    s->snap_vel = (float2*)(a + o_svel);
    BH_CUDA(s, cudaMemsetAsync(arena, 0, c.off, s->stream));
    BH_CUDA(s, cudaMemsetAsync(b.bound, 0xFF, sizeof(uint32_t) * ni, s->stream));
    if (E) {
        // offsets and per-body system ids (systems are contiguous)
        std::vector<uint32_t> off(E + 1, 0), bsys(nb, 0);
        for (uint32_t k = 0; k < E; ++k) {
            off[k + 1] = off[k] + s->sys_sizes[k];
            for (uint32_t i = off[k]; i < off[k + 1]; ++i) bsys[i] = k;
        }
        b.num_systems = E;
        b.sys_off = (uint32_t*)(a + o_soff);
        b.body_sys = (uint32_t*)(a + o_bsys);
        b.sys_bbox = (uint32_t*)(a + o_sbox);
        // key bits = 32 + bits of the largest system id; an even pass count
        // lands the sorted keys back in `codes`
        int sb = 0;
        while (sb < 32 && ((E - 1) >> sb)) ++sb;
        int passes = (32 + sb + 7) / 8;
        b.sort_passes = passes + (passes & 1);
        // On the handle's stream, after the arena memset above: the stream is
        // non-blocking, so a copy on the legacy stream would not be ordered
        // against that memset (which could then clear the offsets).
        BH_CUDA(s, cudaMemcpyAsync((void*)b.sys_off, off.data(), 4 * (size_t)(E + 1),
                                   cudaMemcpyHostToDevice, s->stream));
        BH_CUDA(s, cudaMemcpyAsync((void*)b.body_sys, bsys.data(), 4 * (size_t)nb,
                                   cudaMemcpyHostToDevice, s->stream));
        BH_CUDA(s, cudaStreamSynchronize(s->stream));
    }
    BH_CUDA(s, cudaStreamSynchronize(s->stream));
    s->acc_valid = false;
    return BH_OK;
}

// ---- step enqueue -----------------------------------------------------------

static bh::WalkParams walk_params(const bh_sim* s, int mode) {
    const bh_config& c = s->cfg;
    bh::WalkParams p;
    p.n = s->b.n;
    p.g = c.grav_constant;
    p.theta = c.bh_theta;
    p.dt = c.delta_time;
    // (epsMult * sqrt(G m dt))^2 = epsMult^2 G dt m   (barnes_hut.wgsl:90-92)
    p.eps_coef = c.epsilon_multiplier * c.epsilon_multiplier * c.grav_constant * c.delta_time;
    p.eps2 = c.plummer_eps * c.plummer_eps;
    p.plummer = c.softening == BH_SOFTENING_PLUMMER;
    p.leaf_size = c.leaf_size;
    p.mode = mode;
    p.count = 0;
    p.counters = nullptr;
    p.multipole = c.multipole_order;
    p.bpl = c.bodies_per_lane > 0 ? c.bodies_per_lane : 2;
    p.group_ctr = s->b.scratch ? s->b.scratch->group_ctr : nullptr;
    p.num_systems = s->b.num_systems;
    p.sys_off = s->b.sys_off;
    // Sharding restricts the integrating walk of a step; force evaluations
    // (the first leapfrog force, bh_compute_accelerations) cover every body.
    const bool integrating = mode == bh::kWalkEulerKickDrift || mode == bh::kWalkKdkClose;
    p.slot_lo = integrating ? s->shard_lo : 0u;
    p.slot_hi = integrating ? s->shard_hi : 0xFFFFFFFFu;
    p.stack_cap = (int)s->debug_stack_cap;
    p.far_alpha2 = c.walk_mode == BH_WALK_GROUP ? c.far_alpha * c.far_alpha : 0.0f;
    return p;
}

static void launch_walk_any(bh_sim* s, const bh::WalkParams& p) {
    if (s->cfg.walk_mode == BH_WALK_GROUP) bh::launch_walk_group(s->b, p, s->cfg.walk_block, s->stream);
    else bh::launch_walk(s->b, p, s->cfg.walk_block, s->stream);
}

static bool needs_bbox(const bh_sim* s) {
    return s->cfg.morton_bits == 64 || s->cfg.morton_domain == BH_DOMAIN_BBOX;
}

// Tree stages: scratch reset, bbox, Morton encode, sort (the front), then
// build + fill.  With b.xm null the encode writes no packed leaf records (and
// reads no masses) and the build reads masses and positions directly.
template <class Mark>
static void enqueue_tree_front(bh_sim* s, const DeviceBuffers& b, Mark mark) {
    cudaStream_t st = s->stream;
    bh::launch_zero_step(b, st);  // scratch record + sort look-back status
    mark(1);
    if (b.num_systems > 0) {
        cudaMemsetAsync(b.sys_bbox, 0, sizeof(uint32_t) * 4 * (size_t)b.num_systems, st);
        bh::launch_bbox_ensemble(b, st);
        bh::launch_encode_ensemble(b, st);
    } else {
        if (needs_bbox(s)) bh::launch_bbox(b, st);
        bh::launch_encode(b, s->cfg.morton_domain, st);
    }
    mark(2);
    bh::launch_sort(b, st);
    mark(3);
}

template <class Mark>
static void enqueue_tree_on(bh_sim* s, const DeviceBuffers& b, Mark mark) {
    enqueue_tree_front(s, b, mark);
    bh::launch_build_fill(b, s->cfg.fp64_levels, s->stream);
    mark(4);
}

template <class Mark>
static void enqueue_tree(bh_sim* s, Mark mark) {
    enqueue_tree_on(s, s->b, mark);
}

// One integration step (simulation.ts:394-420).
template <class Mark>
static void enqueue_step(bh_sim* s, Mark mark) {
    const bool kdk = s->cfg.integrator == BH_INTEGRATOR_LEAPFROG_KDK;
    mark(0);
    if (kdk) bh::launch_kick_drift(s->b, s->cfg.delta_time, s->stream);
    enqueue_tree(s, mark);
    launch_walk_any(s, walk_params(s, kdk ? bh::kWalkKdkClose : bh::kWalkEulerKickDrift));
    mark(5);
}

template <class Mark>
static void enqueue_forces(bh_sim* s, Mark mark) {
    mark(0);
    enqueue_tree(s, mark);
    launch_walk_any(s, walk_params(s, bh::kWalkForces));
    mark(5);
}

static int capture_graph(bh_sim* s, int variant) {
    cudaStream_t st = s->stream;
    BH_CUDA(s, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    if (variant == 2) {
        enqueue_tree(s, [](int) {});  // symplectic Euler: the step's stages before the walk
    } else if (variant == 4 || variant == 5) {
        DeviceBuffers b = s->b;
        b.xm = nullptr;  // the masses may still be on their way
        if (variant == 4) enqueue_tree_front(s, b, [](int) {});
        else bh::launch_build_fill(b, s->cfg.fp64_levels, st);
    } else if (variant == 3) {
        launch_walk_any(s, walk_params(s, bh::kWalkEulerKickDrift));
    } else {
        enqueue_step(s, [&](int k) {
            if (variant == 1) cudaEventRecordWithFlags(s->markers[k], st, cudaEventRecordExternal);
        });
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (e != cudaSuccess) return cuda_fail(s, e, "cudaStreamEndCapture(step)");
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(s, e, "kernel launch during capture");
    }
    if (variant == 1) {
        size_t count = 0;
        BH_CUDA(s, cudaGraphGetNodes(g, nullptr, &count));
        std::vector<cudaGraphNode_t> nodes(count);
        BH_CUDA(s, cudaGraphGetNodes(g, nodes.data(), &count));
        for (int k = 0; k < kMarkers; ++k) s->ev_node[k] = nullptr;
        for (auto nd : nodes) {
            cudaGraphNodeType t;
            BH_CUDA(s, cudaGraphNodeGetType(nd, &t));
            if (t != cudaGraphNodeTypeEventRecord) continue;
            cudaEvent_t ev;
            BH_CUDA(s, cudaGraphEventRecordNodeGetEvent(nd, &ev));
            for (int k = 0; k < kMarkers; ++k)
                if (ev == s->markers[k]) s->ev_node[k] = nd;
        }
        for (int k = 0; k < kMarkers; ++k)
            if (!s->ev_node[k]) {
                cudaGraphDestroy(g);
                return fail(s, BH_ERR_CUDA, "profiling graph lost a stage marker");
            }
    }
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(s, e, "cudaGraphInstantiate(step)");
    }
    s->graph[variant] = g;
    s->exec[variant] = ex;
    return BH_OK;
}

static cudaEvent_t* prof_slot(bh_sim* s) {
    if (!s->profiling || s->prof_used >= s->prof_max) return nullptr;
    return &s->prof_ev[(size_t)s->prof_used * kMarkers];
}

// Synchronises the handle's stream once, after the work the caller enqueued
// and a copy of the device error word into page-locked host memory.
static int check_device_errors(bh_sim* s) {
    // an asynchronous download still copying to the host finishes first
    if (s->snap_busy) BH_CUDA(s, cudaStreamWaitEvent(s->stream, s->ev_snap_free, 0));
    BH_CUDA(s, cudaMemcpyAsync(s->err_host, s->b.err, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                               s->stream));
    BH_CUDA(s, cudaStreamSynchronize(s->stream));
    s->snap_busy = false;
    const uint32_t e = *s->err_host;
    if (e == 0) return BH_OK;
    BH_CUDA(s, cudaMemsetAsync(s->b.err, 0, sizeof(uint32_t), s->stream));
    std::string msg = "device check failed:";
    if (e & bh::kErrLookbackSpin) msg += " sort look-back gave up waiting;";
    if (e & bh::kErrStackOverflow) msg += " walk stack full (children dropped);";
    if (e & bh::kErrTreeSpin) msg += " tree build gave up waiting;";
    if (e & bh::kErrGroupStack) msg += " group-walk stack full;";
    if (e & bh::kErrShardCapacity) msg += " shard chunk too small for its updated bodies;";
    // Restore the build's exchange slots so the next step starts clean.
    if (s->b.n > 1) BH_CUDA(s, cudaMemsetAsync(s->b.bound, 0xFF, sizeof(uint32_t) * (s->b.n - 1), s->stream));
    return fail(s, BH_ERR_DEVICE_CHECK, msg);
}

#define BH_HANDLE_NO_SETTLE(s)                                                              \
    do {                                                                                    \
        if (!(s)) return fail(nullptr, BH_ERR_INVALID_ARGUMENT, "null bh_sim handle");      \
        cudaError_t _d = cudaSetDevice((s)->device);                                        \
        if (_d != cudaSuccess) return cuda_fail((s), _d, "cudaSetDevice");                  \
    } while (0)
#define BH_HANDLE(s)                                                                        \
    do {                                                                                    \
        BH_HANDLE_NO_SETTLE(s);                                                             \
        cudaError_t _u = settle_uploads(s);                                                 \
        if (_u != cudaSuccess) return cuda_fail((s), _u, "settling staged uploads");        \
    } while (0)

// ---- lifetime ------------------------------------------------------------------

static int create_sim(const bh_config* config, const uint32_t* sizes, uint32_t num_systems,
                      bh_sim** out);

extern "C" int bh_create(const bh_config* config, bh_sim** out) {
    return create_sim(config, nullptr, 0, out);
}

// Smallest system of an ensemble: larger than the biggest walk group (4 x 32),
// so no group can hold bodies of two systems (a subtree holding parts of two
// systems holds both of them whole).
static constexpr uint32_t kMinSystemBodies = 256;

extern "C" int bh_ensemble_create(const bh_config* config, const uint32_t* bodies_per_system,
                                  uint32_t num_systems, bh_sim** out) {
    if (!bodies_per_system || num_systems == 0)
        return fail(nullptr, BH_ERR_INVALID_ARGUMENT, "bh_ensemble_create: no systems");
    if (num_systems > (1u << 24))
        return fail(nullptr, BH_ERR_INVALID_ARGUMENT, "bh_ensemble_create: at most 2^24 systems");
    uint64_t total = 0;
    for (uint32_t k = 0; k < num_systems; ++k) {
        if (bodies_per_system[k] < kMinSystemBodies)
            return fail(nullptr, BH_ERR_INVALID_ARGUMENT,
                        "bh_ensemble_create: every system needs at least 256 bodies");
        total += bodies_per_system[k];
    }
    if (total > kMaxBodies)
        return fail(nullptr, BH_ERR_INVALID_ARGUMENT, "bh_ensemble_create: more than 2^30 - 1 bodies");
    bh_config c;
    if (config) c = *config;
    else bh_default_config(&c);
    if (c.walk_mode != BH_WALK_GROUP || c.morton_bits != 32)
        return fail(nullptr, BH_ERR_NOT_SUPPORTED,
                    "ensembles need the group walk and 32-bit Morton codes per system");
    return create_sim(&c, bodies_per_system, num_systems, out);
}

static int create_sim(const bh_config* config, const uint32_t* sizes, uint32_t num_systems,
                      bh_sim** out) {
    if (!out) return fail(nullptr, BH_ERR_INVALID_ARGUMENT, "bh_create: null output");
    *out = nullptr;
    bh_sim* s = new bh_sim();
    if (config) s->cfg = *config;
    else bh_default_config(&s->cfg);
    if (num_systems) {
        s->sys_sizes.assign(sizes, sizes + num_systems);
        uint64_t total = 0;
        for (uint32_t k = 0; k < num_systems; ++k) total += sizes[k];
        s->n = (uint32_t)total;
        s->scenario = "";
    }
    int rc = validate_config(s, s->cfg);
    if (rc != BH_OK) {
        delete s;
        return rc;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        delete s;
        return fail(nullptr, BH_ERR_NO_DEVICE,
                    std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "0 devices"));
    }
    if (s->cfg.device < 0 || s->cfg.device >= ndev) {
        delete s;
        return fail(nullptr, BH_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    }
    s->device = s->cfg.device;
    if ((e = cudaSetDevice(s->device)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&s->up[0].landed, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&s->up[0].freed, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&s->up[1].landed, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&s->up[1].freed, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&s->up[2].landed, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&s->up[2].freed, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&s->d2h_stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&s->ev_snap_ready, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&s->ev_snap_free, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaHostAlloc((void**)&s->err_host, sizeof(uint32_t), cudaHostAllocDefault)) != cudaSuccess ||
        (e = bh::sort_init_attributes()) != cudaSuccess ||
        (e = bh::walk_init_attributes()) != cudaSuccess ||
        (e = bh::build_init_attributes()) != cudaSuccess) {
        int r = cuda_fail(nullptr, e, "bh_create");
        delete s;
        return r;
    }
    for (int k = 0; k < kMarkers; ++k) cudaEventCreate(&s->markers[k]);
    rc = alloc_buffers(s, s->n);
    if (rc != BH_OK) {
        std::string m = s->err;
        bh_destroy(s);
        return fail(nullptr, rc, m);
    }
    *out = s;
    return BH_OK;
}

static void free_profile(bh_sim* s) {
    // The profiled graph's event nodes may still name events of this pool:
    // point them back at the persistent markers before the pool goes away.
    if (s->exec[1] && !s->prof_ev.empty()) {
        cudaStreamSynchronize(s->stream);
        for (int k = 0; k < kMarkers; ++k)
            if (s->ev_node[k]) cudaGraphExecEventRecordNodeSetEvent(s->exec[1], s->ev_node[k], s->markers[k]);
    }
    for (auto ev : s->prof_ev) cudaEventDestroy(ev);
    s->prof_ev.clear();
    s->profiling = false;
    s->prof_max = s->prof_used = 0;
}

extern "C" int bh_destroy(bh_sim* s) {
    if (!s) return BH_OK;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    free_buffers(s);
    free_profile(s);
    for (int k = 0; k < kMarkers; ++k)
        if (s->markers[k]) cudaEventDestroy(s->markers[k]);
    if (s->err_host) cudaFreeHost(s->err_host);
    for (auto& u : s->up) {
        if (u.landed) cudaEventDestroy(u.landed);
        if (u.freed) cudaEventDestroy(u.freed);
    }
    if (s->ev_snap_ready) cudaEventDestroy(s->ev_snap_ready);
    if (s->ev_snap_free) cudaEventDestroy(s->ev_snap_free);
    if (s->d2h_stream) cudaStreamDestroy(s->d2h_stream);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return BH_OK;
}

extern "C" int bh_generate_scenario(const char* name, uint32_t n, uint64_t seed,
                                    float grav_constant, float* mass, float* pos, float* vel,
                                    float* radius_multiplier) {
    if (!name) return fail(nullptr, BH_ERR_INVALID_ARGUMENT, "null scenario name");
    if (n > 0 && (!mass || !pos || !vel))
        return fail(nullptr, BH_ERR_INVALID_ARGUMENT, "null output array");
    if (bh::generate_scenario(name, n, seed, grav_constant, mass, pos, vel, radius_multiplier) != 0)
        return fail(nullptr, BH_ERR_UNKNOWN_SCENARIO, std::string("Unknown scenario: ") + name);
    return BH_OK;
}

namespace bh {
int scenario_id(const char* name);
cudaError_t launch_generate(int scenario, uint32_t n, uint64_t seed, float grav_constant,
                            float* mass, float2* pos, float2* vel, float* radius, int device,
                            cudaStream_t stream);
}  // namespace bh

// The scenario generated on the GPU (one PCG32 stream per body).
static int load_scenario_device(bh_sim* s, const std::string& name, uint64_t seed, uint32_t n) {
    const int id = bh::scenario_id(name.c_str());
    if (id < 0) return fail(s, BH_ERR_UNKNOWN_SCENARIO, "Unknown scenario: " + name);
    int rc = alloc_buffers(s, n);
    if (rc != BH_OK) return rc;
    s->scenario = name;
    s->seed = seed;
    s->n = n;
    s->device_gen = true;
    BH_CUDA(s, bh::launch_generate(id, n, seed, s->cfg.grav_constant, s->b.mass, s->b.pos,
                                   s->b.vel, s->b.radius, s->device, s->stream));
    BH_CUDA(s, cudaStreamSynchronize(s->stream));
    return BH_OK;
}

static int load_scenario(bh_sim* s, const std::string& name, uint64_t seed, uint32_t n) {
    if (s->device_gen) return load_scenario_device(s, name, seed, n);
    std::vector<float> mass(n), pos(2 * (size_t)n), vel(2 * (size_t)n), rad(n);
    if (bh::generate_scenario(name.c_str(), n, seed, s->cfg.grav_constant, mass.data(), pos.data(),
                              vel.data(), rad.data()) != 0)
        return fail(s, BH_ERR_UNKNOWN_SCENARIO, "Unknown scenario: " + name);
    // New buffers on every scenario change (simulation.ts:367-369).
    int rc = alloc_buffers(s, n);
    if (rc != BH_OK) return rc;
    s->scenario = name;
    s->seed = seed;
    s->n = n;
    if (n) {
        BH_CUDA(s, cudaMemcpyAsync(s->b.mass, mass.data(), 4 * (size_t)n, cudaMemcpyHostToDevice, s->stream));
        BH_CUDA(s, cudaMemcpyAsync(s->b.pos, pos.data(), 8 * (size_t)n, cudaMemcpyHostToDevice, s->stream));
        BH_CUDA(s, cudaMemcpyAsync(s->b.vel, vel.data(), 8 * (size_t)n, cudaMemcpyHostToDevice, s->stream));
        BH_CUDA(s, cudaMemcpyAsync(s->b.radius, rad.data(), 4 * (size_t)n, cudaMemcpyHostToDevice, s->stream));
    }
    BH_CUDA(s, cudaStreamSynchronize(s->stream));
    return BH_OK;
}

extern "C" int bh_set_num_bodies(bh_sim* s, uint32_t n) {
    BH_HANDLE(s);
    if (!s->sys_sizes.empty())
        return fail(s, BH_ERR_NOT_SUPPORTED, "an ensemble's body counts are fixed at creation");
    if (n > kMaxBodies) return fail(s, BH_ERR_INVALID_ARGUMENT, "body count above 2^30 - 1");
    return load_scenario(s, s->scenario, s->seed, n);  // simulation.ts:227-231
}

extern "C" int bh_set_scenario(bh_sim* s, const char* name, uint64_t seed) {
    BH_HANDLE(s);
    if (!name) return fail(s, BH_ERR_INVALID_ARGUMENT, "null scenario name");
    if (!s->sys_sizes.empty())
        return fail(s, BH_ERR_NOT_SUPPORTED, "use bh_ensemble_set_scenarios on an ensemble");
    s->device_gen = false;
    return load_scenario(s, name, seed, s->n);
}

extern "C" int bh_set_scenario_device(bh_sim* s, const char* name, uint64_t seed) {
    BH_HANDLE(s);
    if (!name) return fail(s, BH_ERR_INVALID_ARGUMENT, "null scenario name");
    if (!s->sys_sizes.empty())
        return fail(s, BH_ERR_NOT_SUPPORTED, "use bh_ensemble_set_scenarios on an ensemble");
    return load_scenario_device(s, name, seed, s->n);
}

// ---- ensembles (extension) ------------------------------------------------------

namespace bh {
double pcg_uniform(uint64_t seed, uint64_t stream, uint32_t draw);
}

extern "C" int bh_ensemble_sizes(uint32_t num_systems, uint64_t seed, uint32_t min_bodies,
                                 uint32_t max_bodies, uint32_t* out) {
    if (!out || num_systems == 0 || min_bodies == 0 || max_bodies < min_bodies)
        return fail(nullptr, BH_ERR_INVALID_ARGUMENT, "bh_ensemble_sizes: bad arguments");
    const double lo = std::log((double)min_bodies), hi = std::log((double)max_bodies);
    for (uint32_t k = 0; k < num_systems; ++k) {
        const double u = bh::pcg_uniform(seed, k, 0);
        uint32_t v = (uint32_t)std::floor(std::exp(lo + (hi - lo) * u));
        out[k] = v < min_bodies ? min_bodies : (v > max_bodies ? max_bodies : v);
    }
    return BH_OK;
}

extern "C" int bh_ensemble_set_scenarios(bh_sim* s, const char* const* names, uint64_t seed) {
    BH_HANDLE(s);
    const uint32_t E = (uint32_t)s->sys_sizes.size();
    if (E == 0) return fail(s, BH_ERR_NOT_SUPPORTED, "not an ensemble");
    const size_t n = s->b.n;
    std::vector<float> mass(n), pos(2 * n), vel(2 * n), rad(n);
    size_t off = 0;
    for (uint32_t k = 0; k < E; ++k) {
        // Per system: its own seed; without names, a Plummer-sphere projection
        // (scale radius 0.1) or a uniform disk, chosen 50/50.
        const uint64_t sk = seed * 0x9E3779B97F4A7C15ULL + k;
        const char* nm = names ? names[k]
                               : (bh::pcg_uniform(seed, k, 1) < 0.5 ? "plummer-projection"
                                                                   : "uniform-disk-kepler");
        if (!nm || bh::generate_scenario(nm, s->sys_sizes[k], sk, s->cfg.grav_constant,
                                         mass.data() + off, pos.data() + 2 * off,
                                         vel.data() + 2 * off, rad.data() + off) != 0)
            return fail(s, BH_ERR_UNKNOWN_SCENARIO,
                        std::string("Unknown scenario: ") + (nm ? nm : "(null)"));
        off += s->sys_sizes[k];
    }
    BH_CUDA(s, cudaMemcpyAsync(s->b.mass, mass.data(), 4 * n, cudaMemcpyHostToDevice, s->stream));
    BH_CUDA(s, cudaMemcpyAsync(s->b.pos, pos.data(), 8 * n, cudaMemcpyHostToDevice, s->stream));
    BH_CUDA(s, cudaMemcpyAsync(s->b.vel, vel.data(), 8 * n, cudaMemcpyHostToDevice, s->stream));
    BH_CUDA(s, cudaMemcpyAsync(s->b.radius, rad.data(), 4 * n, cudaMemcpyHostToDevice, s->stream));
    BH_CUDA(s, cudaStreamSynchronize(s->stream));
    s->acc_valid = false;
    return BH_OK;
}

extern "C" int bh_get_num_systems(bh_sim* s, uint32_t* out) {
    if (!s || !out) return fail(s, BH_ERR_INVALID_ARGUMENT, "null argument");
    *out = (uint32_t)s->sys_sizes.size();
    return BH_OK;
}

extern "C" int bh_get_system_offsets(bh_sim* s, uint32_t* out) {
    if (!s || !out) return fail(s, BH_ERR_INVALID_ARGUMENT, "null argument");
    uint32_t acc = 0;
    out[0] = 0;
    for (size_t k = 0; k < s->sys_sizes.size(); ++k) out[k + 1] = (acc += s->sys_sizes[k]);
    return BH_OK;
}

extern "C" int bh_update_metadata(bh_sim* s) {
    BH_HANDLE(s);
    return validate_config(s, s->cfg);
}

extern "C" int bh_upload(bh_sim* s, const float* mass, const float* pos, const float* vel, uint32_t n) {
    BH_HANDLE_NO_SETTLE(s);
    if (n != s->b.n) return fail(s, BH_ERR_INVALID_ARGUMENT, "bh_upload: n differs from the body count");
    if (n == 0) return BH_OK;
    // Each array into its staging buffer on the copy stream, once the last
    // staged copy of that array has been moved out: the copies need not wait
    // for steps still running.  Positions first (the step's first reader),
    // then masses (the build), then velocities (the walk).
    const void* src[3] = {pos, mass, vel};
    for (int k : {(int)bh_sim::kPos, (int)bh_sim::kMass, (int)bh_sim::kVel}) {
        bh_sim::Staged& u = s->up[k];
        if (!src[k]) continue;
        BH_CUDA(s, cudaStreamWaitEvent(s->copy_stream, u.freed, 0));
        BH_CUDA(s, cudaMemcpyAsync(u.buf, src[k], u.width * (size_t)n, cudaMemcpyHostToDevice, s->copy_stream));
        BH_CUDA(s, cudaEventRecord(u.landed, s->copy_stream));
        u.pending = true;
    }
    if (mass || pos) s->acc_valid = false;
    return BH_OK;
}

extern "C" int bh_download(bh_sim* s, float* mass, float* pos, float* vel, uint32_t n) {
    BH_HANDLE(s);
    if (n != s->b.n) return fail(s, BH_ERR_INVALID_ARGUMENT, "bh_download: n differs from the body count");
    if (n) {
        // host arrays are written in call order: after an earlier asynchronous download
        if (s->snap_busy) BH_CUDA(s, cudaStreamWaitEvent(s->stream, s->ev_snap_free, 0));
        if (mass) BH_CUDA(s, cudaMemcpyAsync(mass, s->b.mass, 4 * (size_t)n, cudaMemcpyDeviceToHost, s->stream));
        if (pos) BH_CUDA(s, cudaMemcpyAsync(pos, s->b.pos, 8 * (size_t)n, cudaMemcpyDeviceToHost, s->stream));
        if (vel) BH_CUDA(s, cudaMemcpyAsync(vel, s->b.vel, 8 * (size_t)n, cudaMemcpyDeviceToHost, s->stream));
    }
    return check_device_errors(s);  // one synchronisation for the copies and the error word
}

extern "C" int bh_download_async(bh_sim* s, float* mass, float* pos, float* vel, uint32_t n) {
    BH_HANDLE(s);
    if (n != s->b.n)
        return fail(s, BH_ERR_INVALID_ARGUMENT, "bh_download_async: n differs from the body count");
    if (n == 0 || !(mass || pos || vel)) return BH_OK;
    // The snapshot is reused once the previous asynchronous download has
    // copied it to the host.
    if (s->snap_busy) BH_CUDA(s, cudaStreamWaitEvent(s->stream, s->ev_snap_free, 0));
    if (mass) BH_CUDA(s, cudaMemcpyAsync(s->snap_mass, s->b.mass, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s->stream));
    if (pos) BH_CUDA(s, cudaMemcpyAsync(s->snap_pos, s->b.pos, 8 * (size_t)n, cudaMemcpyDeviceToDevice, s->stream));
    if (vel) BH_CUDA(s, cudaMemcpyAsync(s->snap_vel, s->b.vel, 8 * (size_t)n, cudaMemcpyDeviceToDevice, s->stream));
    BH_CUDA(s, cudaEventRecord(s->ev_snap_ready, s->stream));
    BH_CUDA(s, cudaStreamWaitEvent(s->d2h_stream, s->ev_snap_ready, 0));
    if (mass) BH_CUDA(s, cudaMemcpyAsync(mass, s->snap_mass, 4 * (size_t)n, cudaMemcpyDeviceToHost, s->d2h_stream));
    if (pos) BH_CUDA(s, cudaMemcpyAsync(pos, s->snap_pos, 8 * (size_t)n, cudaMemcpyDeviceToHost, s->d2h_stream));
    if (vel) BH_CUDA(s, cudaMemcpyAsync(vel, s->snap_vel, 8 * (size_t)n, cudaMemcpyDeviceToHost, s->d2h_stream));
    BH_CUDA(s, cudaEventRecord(s->ev_snap_free, s->d2h_stream));
    s->snap_busy = true;
    return BH_OK;
}

// ---- stepping --------------------------------------------------------------------

static int step_once(bh_sim* s) {
    const bool kdk = s->cfg.integrator == BH_INTEGRATOR_LEAPFROG_KDK;
    cudaEvent_t* ev = prof_slot(s);
    BH_CUDA(s, settle_pos(s));  // the reset and bounding box come first: positions are read at once
    const bool overlap = (s->up[bh_sim::kMass].pending || s->up[bh_sim::kVel].pending) && !kdk && !ev &&
                         s->cfg.use_graphs;
    if (!overlap) BH_CUDA(s, settle_uploads(s));  // leapfrog reads both at once (force evaluation, opening kick)
    if (kdk && !s->acc_valid) {
        enqueue_forces(s, [](int) {});  // first force evaluation of a leapfrog run
        s->acc_valid = true;
    }
    if (overlap) {
        // The last upload's masses and velocities may still be crossing PCIe
        // into their staging buffers (masses first).  The build is the masses' first
        // reader and the walk the velocities', so the stages before them run
        // meanwhile: the same kernels in the same order as the whole-step
        // graph, except that with masses pending the encode writes no packed
        // leaf records and the build gathers masses and positions instead
        // (the same values).
        const bool m = s->up[bh_sim::kMass].pending;
        const int need[3] = {m ? 4 : 2, m ? 5 : 3, 3};
        for (int v : need)
            if (!s->exec[v]) {
                int rc = capture_graph(s, v);
                if (rc != BH_OK) return rc;
            }
        if (m) {
            BH_CUDA(s, cudaGraphLaunch(s->exec[4], s->stream));
            BH_CUDA(s, settle_mass(s));
            BH_CUDA(s, cudaGraphLaunch(s->exec[5], s->stream));
        } else {
            BH_CUDA(s, cudaGraphLaunch(s->exec[2], s->stream));
        }
        BH_CUDA(s, settle_vel(s));
        BH_CUDA(s, cudaGraphLaunch(s->exec[3], s->stream));
        s->acc_valid = false;
        return BH_OK;
    }
    if (s->cfg.use_graphs) {
        const int v = ev ? 1 : 0;
        if (!s->exec[v]) {
            int rc = capture_graph(s, v);
            if (rc != BH_OK) return rc;
        }
        if (ev)
            for (int k = 0; k < kMarkers; ++k)
                BH_CUDA(s, cudaGraphExecEventRecordNodeSetEvent(s->exec[1], s->ev_node[k], ev[k]));
        BH_CUDA(s, cudaGraphLaunch(s->exec[v], s->stream));
    } else {
        enqueue_step(s, [&](int k) {
            if (ev) cudaEventRecord(ev[k], s->stream);
        });
        BH_CUDA(s, cudaGetLastError());
    }
    if (ev) s->prof_used++;
    s->acc_valid = kdk;
    return BH_OK;
}

extern "C" int bh_step(bh_sim* s, uint32_t frames) {
    BH_HANDLE_NO_SETTLE(s);  // step_once orders a pending velocity upload
    if (s->b.n == 0) return BH_OK;
    const uint64_t steps = (uint64_t)frames * (uint64_t)s->cfg.substeps;  // simulation.ts:393
    for (uint64_t i = 0; i < steps; ++i) {
        int rc = step_once(s);
        if (rc != BH_OK) return rc;
    }
    return BH_OK;
}

// ---- sharding (extension) ---------------------------------------------------------

extern "C" int bh_set_walk_slots(bh_sim* s, uint32_t slot_lo, uint32_t slot_hi) {
    BH_HANDLE(s);
    if (s->cfg.walk_mode != BH_WALK_GROUP)
        return fail(s, BH_ERR_NOT_SUPPORTED, "sharded steps need the group walk");
    if (s->b.num_systems > 0)
        return fail(s, BH_ERR_NOT_SUPPORTED, "shard an ensemble by systems, not by slots");
    if (slot_lo > slot_hi) return fail(s, BH_ERR_INVALID_ARGUMENT, "bh_set_walk_slots: lo > hi");
    s->shard_lo = slot_lo;
    s->shard_hi = slot_hi;
    destroy_graphs(s);  // captured steps carry the old walk parameters
    return BH_OK;
}

extern "C" int bh_shard_pack(bh_sim* s, void* chunk, uint32_t capacity) {
    BH_HANDLE(s);
    if (!chunk) return fail(s, BH_ERR_INVALID_ARGUMENT, "null chunk");
    const int kdk = s->cfg.integrator == BH_INTEGRATOR_LEAPFROG_KDK;
    bh::launch_shard_pack(s->b, s->shard_lo, s->shard_hi, kdk, chunk, capacity, s->stream);
    BH_CUDA(s, cudaGetLastError());
    return BH_OK;
}

extern "C" int bh_shard_unpack(bh_sim* s, const void* chunks, uint32_t nchunks, uint32_t capacity) {
    BH_HANDLE(s);
    if (!chunks && nchunks) return fail(s, BH_ERR_INVALID_ARGUMENT, "null chunks");
    const int kdk = s->cfg.integrator == BH_INTEGRATOR_LEAPFROG_KDK;
    bh::launch_shard_unpack(s->b, kdk, chunks, nchunks, capacity, s->stream);
    BH_CUDA(s, cudaGetLastError());
    return BH_OK;
}

extern "C" int bh_sync(bh_sim* s) {
    BH_HANDLE(s);
    return check_device_errors(s);  // synchronises the stream
}

extern "C" int bh_compute_accelerations(bh_sim* s, float* acc_host) {
    BH_HANDLE(s);
    if (s->b.n == 0) return BH_OK;
    enqueue_forces(s, [](int) {});
    BH_CUDA(s, cudaGetLastError());
    if (acc_host)
        BH_CUDA(s, cudaMemcpyAsync(acc_host, s->b.acc, 8 * (size_t)s->b.n, cudaMemcpyDeviceToHost, s->stream));
    BH_CUDA(s, cudaStreamSynchronize(s->stream));
    s->acc_valid = true;
    return check_device_errors(s);
}

// ---- adjoint (extension) -----------------------------------------------------------

namespace bh {
void launch_force_vjp(const DeviceBuffers& b, const WalkParams& p, const float2* abar,
                      float* node_adj, float2* xbar_slot, float* mbar_slot, float2* xbar,
                      float* mbar, cudaStream_t s);
void launch_adj_init(const float2* pos, const float2* target, uint32_t n, float2* xbar,
                     float2* vbar, float* mbar, float2* apend, double* loss, cudaStream_t s);
void launch_adj_pre(const float2* apend, const float2* vbar, float h, uint32_t n, float2* abar,
                    cudaStream_t s);
void launch_adj_post(const float2* xbar, float2* vbar, float2* apend, float dt, float h, uint32_t n,
                     cudaStream_t s);
}  // namespace bh

static int adjoint_supported(bh_sim* s) {
    if (s->cfg.walk_mode != BH_WALK_GROUP || s->cfg.softening != BH_SOFTENING_PLUMMER)
        return fail(s, BH_ERR_NOT_SUPPORTED,
                    "the adjoint needs the group walk and Plummer softening");
    if (s->b.num_systems > 0)
        return fail(s, BH_ERR_NOT_SUPPORTED, "the adjoint runs on single systems, not ensembles");
    if (s->cfg.far_alpha > 0.0f)
        return fail(s, BH_ERR_NOT_SUPPORTED,
                    "the adjoint differentiates the walk without the far field (far_alpha = 0)");
    return BH_OK;
}

static int ensure_adjoint(bh_sim* s, uint32_t nck, uint32_t seg) {
    const uint32_t n = s->b.n;
    bh_sim::Adjoint& a = s->adj;
    if (a.arena && a.n == n && a.nck >= nck && a.seg >= seg) return BH_OK;
    free_adjoint(s);
    const size_t nb = n ? n : 1, ni = n > 1 ? n - 1 : 1;
    Carver c;
    size_t o_na = c.take<float>(6 * ni), o_xs = c.take<float2>(nb), o_ms = c.take<float>(nb);
    size_t o_ab = c.take<float2>(nb), o_xb = c.take<float2>(nb), o_vb = c.take<float2>(nb);
    size_t o_mb = c.take<float>(nb), o_ap = c.take<float2>(nb), o_tg = c.take<float2>(nb);
    size_t o_cp = c.take<float2>(nb * nck), o_cv = c.take<float2>(nb * nck);
    size_t o_sp = c.take<float2>(nb * (seg + 1)), o_fp = c.take<float2>(nb), o_fv = c.take<float2>(nb);
    size_t o_ls = c.take<double>(1);
    void* arena = nullptr;
    cudaError_t e = cudaMalloc(&arena, c.off);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(s, e, "cudaMalloc(adjoint buffers)");
    }
    char* p = (char*)arena;
    a.arena = arena;
    a.n = n;
    a.nck = nck;
    a.seg = seg;
    a.node_adj = (float*)(p + o_na);
    a.xbar_slot = (float2*)(p + o_xs);
    a.mbar_slot = (float*)(p + o_ms);
    a.abar = (float2*)(p + o_ab);
    a.xbar = (float2*)(p + o_xb);
    a.vbar = (float2*)(p + o_vb);
    a.mbar = (float*)(p + o_mb);
    a.apend = (float2*)(p + o_ap);
    a.target = (float2*)(p + o_tg);
    a.ck_pos = (float2*)(p + o_cp);
    a.ck_vel = (float2*)(p + o_cv);
    a.seg_pos = (float2*)(p + o_sp);
    a.fin_pos = (float2*)(p + o_fp);
    a.fin_vel = (float2*)(p + o_fv);
    a.loss = (double*)(p + o_ls);
    // Replayed trees for the reverse sweep: one record per step of a segment,
    // within 4 GB and a quarter of the free device memory.
    const TreeRecord r = tree_record(n);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        free_b = 0;
    }
    const size_t want = r.bytes * (size_t)seg;
    const size_t budget = free_b / 4 < ((size_t)4 << 30) ? free_b / 4 : ((size_t)4 << 30);
    if (n > 1 && s->cfg.walk_mode == BH_WALK_GROUP && want <= budget) {
        void* slab = nullptr;
        if (cudaMalloc(&slab, want) == cudaSuccess) {
            a.slab = slab;
            a.slab_stride = r.bytes;
            a.slab_steps = seg;
        } else {
            cudaGetLastError();  // fall back to rebuilding each tree
        }
    }
    return BH_OK;
}

// (xbar, mbar) += J^T abar for the force at positions `at` (tree rebuilt there).
static void enqueue_force_vjp(bh_sim* s, const float2* at, const float2* abar) {
    DeviceBuffers bb = s->b;
    bb.pos = const_cast<float2*>(at);
    enqueue_tree_on(s, bb, [](int) {});
    bh::launch_force_vjp(bb, walk_params(s, bh::kWalkForces), abar, s->adj.node_adj,
                         s->adj.xbar_slot, s->adj.mbar_slot, s->adj.xbar, s->adj.mbar, s->stream);
}

// Same, on the tree saved in slab record k (built at those positions).
static void enqueue_force_vjp_saved(bh_sim* s, uint32_t k, const float2* abar) {
    DeviceBuffers bb = slab_view(s, k);
    const TreeRecord r = tree_record(s->b.n);
    unsigned int* ctr = (unsigned int*)((char*)s->adj.slab + (size_t)k * s->adj.slab_stride + r.ctr);
    cudaMemsetAsync(ctr, 0, sizeof(unsigned int), s->stream);  // work counter; [1] = group count
    bh::WalkParams p = walk_params(s, bh::kWalkForces);
    p.group_ctr = ctr;
    bh::launch_force_vjp(bb, p, abar, s->adj.node_adj, s->adj.xbar_slot, s->adj.mbar_slot,
                         s->adj.xbar, s->adj.mbar, s->stream);
}

extern "C" int bh_force_vjp(bh_sim* s, const float* abar, float* xbar, float* mbar) {
    BH_HANDLE(s);
    int rc = adjoint_supported(s);
    if (rc != BH_OK) return rc;
    const uint32_t n = s->b.n;
    if (n == 0) return BH_OK;
    if (!abar) return fail(s, BH_ERR_INVALID_ARGUMENT, "null abar");
    if ((rc = ensure_adjoint(s, 1, 1)) != BH_OK) return rc;
    bh_sim::Adjoint& a = s->adj;
    BH_CUDA(s, cudaMemcpyAsync(a.abar, abar, 8 * (size_t)n, cudaMemcpyHostToDevice, s->stream));
    BH_CUDA(s, cudaMemsetAsync(a.xbar, 0, 8 * (size_t)n, s->stream));
    BH_CUDA(s, cudaMemsetAsync(a.mbar, 0, 4 * (size_t)n, s->stream));
    enqueue_force_vjp(s, s->b.pos, a.abar);
    BH_CUDA(s, cudaGetLastError());
    if (xbar) BH_CUDA(s, cudaMemcpyAsync(xbar, a.xbar, 8 * (size_t)n, cudaMemcpyDeviceToHost, s->stream));
    if (mbar) BH_CUDA(s, cudaMemcpyAsync(mbar, a.mbar, 4 * (size_t)n, cudaMemcpyDeviceToHost, s->stream));
    BH_CUDA(s, cudaStreamSynchronize(s->stream));
    return check_device_errors(s);
}

extern "C" int bh_rollout_grad(bh_sim* s, uint32_t steps, uint32_t checkpoint_every,
                               const float* target_pos, float* loss, float* grad_pos,
                               float* grad_vel, float* grad_mass) {
    BH_HANDLE(s);
    int rc = adjoint_supported(s);
    if (rc != BH_OK) return rc;
    if (s->cfg.integrator != BH_INTEGRATOR_LEAPFROG_KDK)
        return fail(s, BH_ERR_NOT_SUPPORTED, "the rollout gradient needs the leapfrog integrator");
    if (steps == 0 || checkpoint_every == 0 || !target_pos)
        return fail(s, BH_ERR_INVALID_ARGUMENT, "steps, checkpoint_every and target_pos are required");
    const uint32_t n = s->b.n;
    if (n == 0) return BH_OK;
    const uint32_t K = checkpoint_every < steps ? checkpoint_every : steps;
    const uint32_t nck = (steps + K - 1) / K;  // checkpoints at 0, K, 2K, ... < steps
    if ((rc = ensure_adjoint(s, nck, K)) != BH_OK) return rc;
    bh_sim::Adjoint& a = s->adj;
    cudaStream_t st = s->stream;
    const size_t vb = 8 * (size_t)n;
    const float dt = s->cfg.delta_time, h = 0.5f * dt;
    BH_CUDA(s, cudaMemcpyAsync(a.target, target_pos, vb, cudaMemcpyHostToDevice, st));
    // Forward: T steps, saving (x, v) at every checkpoint.  The last segment
    // is recorded as its replay would record it (positions per step, trees in
    // the slab): a replayed step reproduces the forward step bit for bit (same
    // inputs, same deterministic pipeline), so that segment needs no replay.
    const uint32_t c_last = (nck - 1) * K;
    const bool last_saved = a.slab && a.slab_steps >= steps - c_last;
    for (uint32_t k = 0; k < steps; ++k) {
        if (k % K == 0) {
            BH_CUDA(s, cudaMemcpyAsync(a.ck_pos + (size_t)(k / K) * n, s->b.pos, vb, cudaMemcpyDeviceToDevice, st));
            BH_CUDA(s, cudaMemcpyAsync(a.ck_vel + (size_t)(k / K) * n, s->b.vel, vb, cudaMemcpyDeviceToDevice, st));
        }
        if (k == c_last) BH_CUDA(s, cudaMemcpyAsync(a.seg_pos, s->b.pos, vb, cudaMemcpyDeviceToDevice, st));
        if ((rc = step_once(s)) != BH_OK) return rc;
        if (k >= c_last) {
            BH_CUDA(s, cudaMemcpyAsync(a.seg_pos + (size_t)(k + 1 - c_last) * n, s->b.pos, vb,
                                       cudaMemcpyDeviceToDevice, st));
            if (last_saved && (rc = save_tree(s, k - c_last)) != BH_OK) return rc;
        }
    }
    BH_CUDA(s, cudaMemcpyAsync(a.fin_pos, s->b.pos, vb, cudaMemcpyDeviceToDevice, st));
    BH_CUDA(s, cudaMemcpyAsync(a.fin_vel, s->b.vel, vb, cudaMemcpyDeviceToDevice, st));
    // dL/dx_T for L = (1/n) sum_i |x_T,i - target_i|^2
    bh::launch_adj_init(s->b.pos, a.target, n, a.xbar, a.vbar, a.mbar, a.apend, a.loss, st);
    // Reverse sweep, one checkpoint segment at a time (replay rebuilds the trees).
    for (int64_t seg = (int64_t)nck - 1; seg >= 0; --seg) {
        const uint32_t c = (uint32_t)seg * K, e = (c + K < steps) ? c + K : steps;
        const bool saved = a.slab && a.slab_steps >= e - c;
        if (c != c_last) {  // the last segment was recorded by the forward pass
            BH_CUDA(s, cudaMemcpyAsync(s->b.pos, a.ck_pos + (size_t)seg * n, vb, cudaMemcpyDeviceToDevice, st));
            BH_CUDA(s, cudaMemcpyAsync(s->b.vel, a.ck_vel + (size_t)seg * n, vb, cudaMemcpyDeviceToDevice, st));
            s->acc_valid = false;
            BH_CUDA(s, cudaMemcpyAsync(a.seg_pos, s->b.pos, vb, cudaMemcpyDeviceToDevice, st));
            for (uint32_t k = c; k < e; ++k) {
                if ((rc = step_once(s)) != BH_OK) return rc;
                BH_CUDA(s, cudaMemcpyAsync(a.seg_pos + (size_t)(k + 1 - c) * n, s->b.pos, vb,
                                           cudaMemcpyDeviceToDevice, st));
                // the step's tree is the one at x_{k+1}, where its reverse step needs the VJP
                if (saved && (rc = save_tree(s, k - c)) != BH_OK) return rc;
            }
        }
        for (int64_t k = (int64_t)e - 1; k >= (int64_t)c; --k) {
            // closing kick of step k (force at x_{k+1}) plus the pending opening
            // kick of step k+1 at the same point
            bh::launch_adj_pre(a.apend, a.vbar, h, n, a.abar, st);
            if (saved) enqueue_force_vjp_saved(s, (uint32_t)(k - c), a.abar);
            else enqueue_force_vjp(s, a.seg_pos + (size_t)(k + 1 - c) * n, a.abar);
            // drift, then the opening kick of step k (force at x_k, pending)
            bh::launch_adj_post(a.xbar, a.vbar, a.apend, dt, h, n, st);
        }
    }
    // the opening kick of step 0 acts at x_0
    bh::launch_adj_pre(a.apend, a.vbar, 0.0f, n, a.abar, st);
    enqueue_force_vjp(s, a.ck_pos, a.abar);
    BH_CUDA(s, cudaGetLastError());
    double L = 0.0;
    BH_CUDA(s, cudaMemcpyAsync(&L, a.loss, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (grad_pos) BH_CUDA(s, cudaMemcpyAsync(grad_pos, a.xbar, vb, cudaMemcpyDeviceToHost, st));
    if (grad_vel) BH_CUDA(s, cudaMemcpyAsync(grad_vel, a.vbar, vb, cudaMemcpyDeviceToHost, st));
    if (grad_mass) BH_CUDA(s, cudaMemcpyAsync(grad_mass, a.mbar, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
    // leave the handle at step T
    BH_CUDA(s, cudaMemcpyAsync(s->b.pos, a.fin_pos, vb, cudaMemcpyDeviceToDevice, st));
    BH_CUDA(s, cudaMemcpyAsync(s->b.vel, a.fin_vel, vb, cudaMemcpyDeviceToDevice, st));
    s->acc_valid = false;
    BH_CUDA(s, cudaStreamSynchronize(st));
    if (loss) *loss = (float)L;
    return check_device_errors(s);
}

extern "C" int bh_walk_stats(bh_sim* s, uint64_t* node_visits, uint64_t* multipole_interactions,
                             uint64_t* body_interactions, uint64_t* far_nodes) {
    BH_HANDLE(s);
    unsigned long long h[4] = {0, 0, 0, 0};
    if (s->b.n > 0) {
        enqueue_tree(s, [](int) {});
        bh::WalkParams p = walk_params(s, bh::kWalkForces);
        p.count = 1;
        p.counters = s->b.scratch->walk_counts;
        launch_walk_any(s, p);
        BH_CUDA(s, cudaGetLastError());
        BH_CUDA(s, cudaMemcpyAsync(h, s->b.scratch->walk_counts, sizeof(h), cudaMemcpyDeviceToHost,
                                   s->stream));
        BH_CUDA(s, cudaStreamSynchronize(s->stream));
        s->acc_valid = true;
    }
    if (node_visits) *node_visits = h[0];
    if (multipole_interactions) *multipole_interactions = h[1];
    if (body_interactions) *body_interactions = h[2];
    if (far_nodes) *far_nodes = h[3];
    return check_device_errors(s);
}

// ---- test hooks of the device-side checks ------------------------------------------

extern "C" int bh_debug_set_limits(bh_sim* s, uint32_t flags, uint32_t lookback_spin_cap,
                                   uint32_t walk_stack_cap) {
    BH_HANDLE(s);
    if (flags & ~(bh::kDebugLookbackUnpublished | bh::kDebugSplitBuild))
        return fail(s, BH_ERR_INVALID_ARGUMENT, "bh_debug_set_limits: unknown flag");
    if (walk_stack_cap == 1)
        return fail(s, BH_ERR_INVALID_ARGUMENT, "bh_debug_set_limits: a walk stack needs 2 entries");
    s->debug_flags = flags;
    s->debug_spin_cap = lookback_spin_cap;
    s->debug_stack_cap = walk_stack_cap;
    s->b.spin_cap = lookback_spin_cap ? lookback_spin_cap : bh::kSpinCapDefault;
    s->b.debug_flags = flags;
    destroy_graphs(s);  // captured steps carry the old kernel parameters
    return BH_OK;
}

// ---- buffers -----------------------------------------------------------------------

extern "C" int bh_get_buffers(bh_sim* s, bh_buffers* out) {
    BH_HANDLE(s);
    if (!out) return fail(s, BH_ERR_INVALID_ARGUMENT, "null output");
    const DeviceBuffers& b = s->b;
    // Group walk: the reference-layout internal-node arrays are derived from
    // the packed records on request (stream-ordered after the last step).
    if (b.gnode) bh::launch_ref_layout(b, s->stream);
    out->mass = b.mass;
    out->pos = (float*)b.pos;
    out->vel = (float*)b.vel;
    out->radius_multiplier = b.radius;
    out->acc = (float*)b.acc;
    out->morton_codes = b.codes;
    out->body_indices = b.ids;
    out->node4 = (float*)b.node4;
    out->node_children = (uint32_t*)b.children;
    out->node_parent = b.parent;
    out->node_aabb = (float*)b.aabb;
    out->num_bodies = b.n;
    out->morton_bits = s->cfg.morton_bits;
    out->stream = (void*)s->stream;
    return BH_OK;
}

extern "C" int bh_get_num_bodies(bh_sim* s, uint32_t* out) {
    if (!s || !out) return fail(s, BH_ERR_INVALID_ARGUMENT, "null argument");
    *out = s->b.n;
    return BH_OK;
}

extern "C" int bh_read_buffer(bh_sim* s, const char* name, void* host, size_t bytes) {
    BH_HANDLE(s);
    if (!name || (!host && bytes)) return fail(s, BH_ERR_INVALID_ARGUMENT, "null argument");
    const DeviceBuffers& b = s->b;
    const size_t n = b.n, nn = n ? 2 * n - 1 : 0, ni = n > 1 ? n - 1 : 0;
    const std::string nm(name);
    const void* src = nullptr;
    size_t cap = 0;
    if (nm == "mass") { src = b.mass; cap = 4 * n; }
    else if (nm == "pos") { src = b.pos; cap = 8 * n; }
    else if (nm == "vel") { src = b.vel; cap = 8 * n; }
    else if (nm == "acc") { src = b.acc; cap = 8 * n; }
    else if (nm == "radius_multiplier") { src = b.radius; cap = 4 * n; }
    else if (nm == "morton_codes") { src = b.codes; cap = (size_t)b.key_bytes * n; }
    else if (nm == "body_indices") { src = b.ids; cap = 4 * n; }
    else if (nm == "node4") { src = b.node4; cap = 16 * nn; }
    else if (nm == "node_children") { src = b.children; cap = 8 * ni; }
    else if (nm == "node_parent") { src = b.parent; cap = 4 * nn; }
    else if (nm == "node_aabb") { src = b.aabb; cap = 16 * ni; }
    else return fail(s, BH_ERR_INVALID_ARGUMENT, "unknown buffer name: " + nm);
    if (bytes > cap) return fail(s, BH_ERR_INVALID_ARGUMENT, "bh_read_buffer: size above the buffer");
    if (b.gnode && (nm == "node4" || nm == "node_children" || nm == "node_aabb"))
        bh::launch_ref_layout(b, s->stream);
    if (bytes) BH_CUDA(s, cudaMemcpyAsync(host, src, bytes, cudaMemcpyDeviceToHost, s->stream));
    BH_CUDA(s, cudaStreamSynchronize(s->stream));
    return BH_OK;
}

// ---- profiling -----------------------------------------------------------------------

extern "C" int bh_profile_begin(bh_sim* s, uint32_t max_steps) {
    BH_HANDLE(s);
    if (max_steps == 0 || max_steps > 100000)
        return fail(s, BH_ERR_INVALID_ARGUMENT, "max_steps must be in [1, 100000]");
    free_profile(s);
    s->prof_ev.resize((size_t)max_steps * kMarkers);
    for (auto& ev : s->prof_ev) BH_CUDA(s, cudaEventCreate(&ev));
    s->prof_max = max_steps;
    s->prof_used = 0;
    s->profiling = true;
    return BH_OK;
}

extern "C" int bh_profile_end(bh_sim* s, double* stage_ms, uint32_t* steps_recorded) {
    BH_HANDLE(s);
    if (!s->profiling) return fail(s, BH_ERR_INVALID_ARGUMENT, "profiling was not started");
    BH_CUDA(s, cudaStreamSynchronize(s->stream));
    double acc[BH_NUM_STAGES] = {0, 0, 0, 0, 0};
    // marker k -> stage: [0,1] other, [1,2] morton, [2,3] sort, [3,4] tree, [4,5] walk
    const int stage_of[5] = {BH_STAGE_OTHER, BH_STAGE_MORTON, BH_STAGE_SORT, BH_STAGE_TREE, BH_STAGE_WALK};
    for (uint32_t i = 0; i < s->prof_used; ++i) {
        cudaEvent_t* ev = &s->prof_ev[(size_t)i * kMarkers];
        for (int k = 0; k < 5; ++k) {
            float ms = 0.f;
            BH_CUDA(s, cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
            acc[stage_of[k]] += ms;
        }
    }
    if (stage_ms)
        for (int k = 0; k < BH_NUM_STAGES; ++k) stage_ms[k] = acc[k];
    if (steps_recorded) *steps_recorded = s->prof_used;
    free_profile(s);
    return check_device_errors(s);
}

// ---- autotuner (extension) -----------------------------------------------------------
// Times the group walk on force evaluations at the current positions (which
// do not advance the state) for every (bodies per lane, leaf size) candidate,
// then the block shape (64, 128 or 256 threads) of the fastest, and keeps
// the fastest of all.  The walk's result depends on the first two (group boxes and
// bucket sizes change the interaction lists), so every candidate is a valid
// configuration with its own accuracy; all stay far inside the group walk's
// error budget at a given theta.
extern "C" int bh_autotune(bh_sim* s, uint32_t trials, bh_tune_result* out) {
    BH_HANDLE(s);
    if (s->cfg.walk_mode != BH_WALK_GROUP)
        return fail(s, BH_ERR_NOT_SUPPORTED, "the autotuner tunes the group walk");
    if (trials == 0) trials = 3;
    static const int kBpl[] = {1, 2, 4};
    static const int kLeaf[] = {2, 4, 8};
    static const int kBlock[] = {64, 256};  // besides the default 128 of the first sweep
    bh_tune_result best{};
    best.walk_ms = 1e30f;
    cudaEvent_t e0, e1;
    BH_CUDA(s, cudaEventCreate(&e0));
    BH_CUDA(s, cudaEventCreate(&e1));
    int count = 0;
    const bh_config saved = s->cfg;
    // Average walk time of the handle's current shape over `trials` launches.
    auto time_walk = [&](float* out) -> int {
        float total = 0.f;
        for (uint32_t t = 0; t <= trials; ++t) {  // trial 0 warms up
            enqueue_tree(s, [](int) {});
            cudaEventRecord(e0, s->stream);
            launch_walk_any(s, walk_params(s, bh::kWalkForces));
            cudaEventRecord(e1, s->stream);
            BH_CUDA(s, cudaEventSynchronize(e1));
            float ms = 0.f;
            BH_CUDA(s, cudaEventElapsedTime(&ms, e0, e1));
            if (t > 0) total += ms;
        }
        *out = total / (float)trials;
        return BH_OK;
    };
    // Groups and buckets first (block of 128 threads), then the block shape
    // for the best of them.
    for (int bpl : kBpl) {
        for (int leaf : kLeaf) {
            if (s->b.n == 0) break;
            s->cfg.bodies_per_lane = bpl;
            s->cfg.leaf_size = leaf;
            s->cfg.walk_block = 128;
            s->b.group_max = 32u * (uint32_t)bpl;
            float avg = 0.f;
            const int rc = time_walk(&avg);
            if (rc != BH_OK) return rc;
            ++count;
            if (avg < best.walk_ms) {
                best.walk_ms = avg;
                best.bodies_per_lane = bpl;
                best.leaf_size = leaf;
                best.walk_block = 128;
            }
        }
    }
    for (int block : kBlock) {
        if (s->b.n == 0) break;
        if (block > bh::walk_group_max_block(best.bodies_per_lane)) continue;
        s->cfg.bodies_per_lane = best.bodies_per_lane;
        s->cfg.leaf_size = best.leaf_size;
        s->cfg.walk_block = block;
        s->b.group_max = 32u * (uint32_t)best.bodies_per_lane;
        float avg = 0.f;
        const int rc = time_walk(&avg);
        if (rc != BH_OK) return rc;
        ++count;
        if (avg < best.walk_ms) {
            best.walk_ms = avg;
            best.walk_block = block;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s->cfg = saved;
    if (count > 0) {
        s->cfg.bodies_per_lane = best.bodies_per_lane;
        s->cfg.leaf_size = best.leaf_size;
        s->cfg.walk_block = best.walk_block;
    }
    s->b.group_max = 32u * (uint32_t)(s->cfg.bodies_per_lane > 0 ? s->cfg.bodies_per_lane : 2);
    destroy_graphs(s);  // captured steps carry the old walk parameters
    s->acc_valid = false;
    best.candidates = count;
    if (out) *out = best;
    return check_device_errors(s);
}

extern "C" int bh_get_config(bh_sim* s, bh_config* out) {
    if (!s || !out) return fail(s, BH_ERR_INVALID_ARGUMENT, "null argument");
    *out = s->cfg;
    return BH_OK;
}

extern "C" int bh_kernels_per_step(bh_sim* s, uint32_t* out) {
    if (!s || !out) return fail(s, BH_ERR_INVALID_ARGUMENT, "null argument");
    uint32_t k = 0;
    if (s->cfg.integrator == BH_INTEGRATOR_LEAPFROG_KDK) k += 1;  // kick + drift
    k += 1;                                                         // scratch reset
    if (needs_bbox(s) || s->b.num_systems) k += 1;                 // bbox (per system)
    k += 1;                                                         // encode
    k += (uint32_t)bh::sort_passes(s->b);                          // sort passes
    k += bh::split_build(s->b.n, s->b.debug_flags) ? 2 : 1;                           // build + fill (+ frontier climb)
    k += 1;                                                         // walk + integrate
    *out = s->b.n ? k : 0;
    return BH_OK;
}

// ---- errors ----------------------------------------------------------------------------

extern "C" const char* bh_last_error(bh_sim* s) { return s ? s->err.c_str() : g_err.c_str(); }
extern "C" const char* bh_global_last_error(void) { return g_err.c_str(); }
extern "C" const char* bh_version(void) { return "bh-b200 0.1.0 (sm_100a)"; }
