// ref_harness.cpp -- runs the mechanically translated reference shaders
// (oracle/_ref/ref_lbvh.inc, ref_barnes_hut.inc) on the CPU.
//
// TEST INFRASTRUCTURE ONLY: builds oracle/_ref/libref_wgsl.so, used to pin
// the oracle restatement, to generate tests/golden/ fixtures, and as the
// timed CPU baseline of the benchmark (the reference's own shader logic).
//
// It allocates the buffers of src/simulation.ts:82-91, writes the 32-byte
// metadata of simulation.ts:212-225 (offset chosen by the caller instead of
// Math.random), and per step dispatches the entry points in the order of
// simulation.ts:393-420 with ceil(N/64) workgroups of 64 invocations, one
// invocation after another (global_invocation_id.x = 0, 1, ...).  The sort
// stage is the third-party webgpu-radix-sort@1.0.7, which is not vendored;
// its place is taken by the stable sort of (key, id) by key.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#include <parallel/algorithm>
#endif

#include "wgsl_prelude.h"
#include "ref_lbvh.inc"
#include "ref_barnes_hut.inc"

static_assert(sizeof(ref_lbvh::NodeData) == 48 && sizeof(ref_barnes_hut::NodeData) == 48,
              "NodeData is 12 words (simulation.ts:90)");

static void dispatch(void (*entry)(wgsl::vec3u), uint32_t workgroups) {
    for (uint32_t g = 0; g < workgroups * 64u; ++g) {
        wgsl::vec3u id;
        id.x = g;
        entry(id);
    }
}

// Invocations that touch disjoint outputs (Morton encode, build, velocity
// and position steps) may run on all host threads; the result is the same as
// one at a time.  The fill is always serial: run concurrently, its
// fence-free arrival counters are the race the reference's README describes.
static void dispatch_par(void (*entry)(wgsl::vec3u), uint32_t workgroups, int parallel) {
    if (!parallel) {
        dispatch(entry, workgroups);
        return;
    }
    const int64_t total = (int64_t)workgroups * 64;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t g = 0; g < total; ++g) {
        wgsl::vec3u id;
        id.x = (uint32_t)g;
        entry(id);
    }
}

static double omp_now() {
#ifdef _OPENMP
    return omp_get_wtime();
#else
    return 0.0;
#endif
}

extern "C" int ref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// The buffers of simulation.ts:82-91 and the metadata of :212-225, bound to
// the translated shaders' globals.
struct RefState {
    uint32_t n = 0;
    std::vector<float> m;
    std::vector<wgsl::vec2f> p, v;
    std::vector<uint32_t> codes, ids, status, order, tk, ti;
    std::vector<ref_lbvh::NodeData> nodes;

    RefState(uint32_t n_, const float* mass, const float* pos, const float* vel, float G, float dt,
             float eps_mult, float theta, uint32_t offset)
        : n(n_), m(mass, mass + n_), p(n_), v(n_), codes(n_), ids(n_),
          status(2 * (size_t)n_ - 1, 0u), order(n_), tk(n_), ti(n_), nodes(2 * (size_t)n_ - 1) {
        for (uint32_t i = 0; i < n; ++i) {
            p[i] = wgsl::vec2f(pos[2 * i], pos[2 * i + 1]);
            v[i] = wgsl::vec2f(vel[2 * i], vel[2 * i + 1]);
        }
        ref_lbvh::metadata.num_bodies = n;
        ref_lbvh::metadata.grav_constant = G;
        ref_lbvh::metadata.delta_time = dt;
        ref_lbvh::metadata.epsilon_multiplier = eps_mult;
        ref_lbvh::metadata.bh_theta = theta;
        ref_lbvh::metadata.offset = offset % n;
        ref_barnes_hut::metadata.num_bodies = n;
        ref_barnes_hut::metadata.grav_constant = G;
        ref_barnes_hut::metadata.delta_time = dt;
        ref_barnes_hut::metadata.epsilon_multiplier = eps_mult;
        ref_barnes_hut::metadata.bh_theta = theta;
        ref_lbvh::mass_buf = m.data();
        ref_lbvh::pos_buf = p.data();
        ref_lbvh::node_data = nodes.data();
        ref_lbvh::node_status = status.data();
        ref_barnes_hut::mass_buf = m.data();
        ref_barnes_hut::pos_buf = p.data();
        ref_barnes_hut::vel_buf = v.data();
        ref_barnes_hut::node_data = reinterpret_cast<ref_barnes_hut::NodeData*>(nodes.data());
        bind_sorted();
    }
    void bind_sorted() {
        ref_lbvh::morton_codes = codes.data();
        ref_lbvh::body_indices = ids.data();
        ref_barnes_hut::body_indices = ids.data();
    }
    // The third-party sort's contract: the stable sort of (key, id) by key.
    void sort(int parallel) {
        std::iota(order.begin(), order.end(), 0u);
        auto by_key = [&](uint32_t a, uint32_t b) { return codes[a] < codes[b]; };
#ifdef _OPENMP
        if (parallel) __gnu_parallel::stable_sort(order.begin(), order.end(), by_key);
        else std::stable_sort(order.begin(), order.end(), by_key);
#else
        std::stable_sort(order.begin(), order.end(), by_key);
#endif
        for (uint32_t i = 0; i < n; ++i) {
            tk[i] = codes[order[i]];
            ti[i] = ids[order[i]];
        }
        codes.swap(tk);
        ids.swap(ti);
        bind_sorted();
    }
};

// Every `stride`-th invocation of an entry point (a bounded sample of a
// dispatch whose invocations are independent).
static void dispatch_sampled(void (*entry)(wgsl::vec3u), uint32_t n, uint32_t stride, int parallel) {
    const int64_t count = ((int64_t)n + stride - 1) / stride;
#pragma omp parallel for schedule(dynamic, 64) if (parallel)
    for (int64_t k = 0; k < count; ++k) {
        wgsl::vec3u id;
        id.x = (uint32_t)(k * stride);
        entry(id);
    }
}

extern "C" int ref_run(uint32_t n, const float* mass, const float* pos, const float* vel, float G,
                       float dt, float eps_mult, float theta, uint32_t offset, uint32_t steps,
                       int parallel, float* pos_out, float* vel_out, uint32_t* codes_out,
                       uint32_t* ids_out, uint32_t* left_out, uint32_t* right_out,
                       uint32_t* parent_out, float* com_out, float* mass_out, float* aabb_out,
                       float* length_out) {
    if (n == 0) return 0;
    RefState S(n, mass, pos, vel, G, dt, eps_mult, theta, offset);
    std::vector<wgsl::vec2f>& p = S.p;
    std::vector<wgsl::vec2f>& v = S.v;
    std::vector<uint32_t>& codes = S.codes;
    std::vector<uint32_t>& ids = S.ids;
    std::vector<ref_lbvh::NodeData>& nodes = S.nodes;
    const uint32_t wg = (n + 63u) / 64u;
    for (uint32_t s = 0; s < steps; ++s) {
        dispatch_par(ref_lbvh::compute_morton_codes_main, wg, parallel);
        S.sort(parallel);
        dispatch_par(ref_lbvh::build_lbvh_main, wg, parallel);
        dispatch(ref_lbvh::fill_lbvh_main, wg);
        dispatch_par(ref_barnes_hut::bh_vel_step_main, wg, parallel);
        dispatch_par(ref_barnes_hut::bh_pos_step_main, wg, parallel);
    }
    for (uint32_t i = 0; i < n; ++i) {
        if (pos_out) { pos_out[2 * i] = p[i].x; pos_out[2 * i + 1] = p[i].y; }
        if (vel_out) { vel_out[2 * i] = v[i].x; vel_out[2 * i + 1] = v[i].y; }
        if (codes_out) codes_out[i] = codes[i];
        if (ids_out) ids_out[i] = ids[i];
    }
    for (size_t k = 0; k < 2 * (size_t)n - 1; ++k) {
        const auto& nd = nodes[k];
        if (left_out) left_out[k] = nd.left_child;
        if (right_out) right_out[k] = nd.right_child;
        if (parent_out) parent_out[k] = nd.parent;
        if (com_out) { com_out[2 * k] = nd.center_of_mass.x; com_out[2 * k + 1] = nd.center_of_mass.y; }
        if (mass_out) mass_out[k] = nd.total_mass;
        if (aabb_out) {
            aabb_out[4 * k] = nd.aabb_min.x; aabb_out[4 * k + 1] = nd.aabb_min.y;
            aabb_out[4 * k + 2] = nd.aabb_max.x; aabb_out[4 * k + 3] = nd.aabb_max.y;
        }
        if (length_out) length_out[k] = nd.length;
    }
    return 0;
}

// Timing sample of the pipeline: `steps` steps with the wall time of each
// stage summed into stage_s[5] = {Morton, sort, build + fill, velocity step,
// position step}.  The velocity step (the walk) runs only for every
// `walk_stride`-th sorted slot, a bounded sample whose time the caller
// scales by walk_stride; the other stages run whole.  With walk_stride 1
// this is ref_run's pipeline.
extern "C" int ref_run_timed(uint32_t n, const float* mass, const float* pos, const float* vel,
                             float G, float dt, float eps_mult, float theta, uint32_t steps,
                             uint32_t walk_stride, int parallel, double* stage_s) {
    if (n == 0 || walk_stride == 0) return 1;
    RefState S(n, mass, pos, vel, G, dt, eps_mult, theta, 0u);
    const uint32_t wg = (n + 63u) / 64u;
    for (int k = 0; k < 5; ++k) stage_s[k] = 0.0;
    for (uint32_t s = 0; s < steps; ++s) {
        double t0 = omp_now();
        dispatch_par(ref_lbvh::compute_morton_codes_main, wg, parallel);
        double t1 = omp_now();
        S.sort(parallel);
        double t2 = omp_now();
        dispatch_par(ref_lbvh::build_lbvh_main, wg, parallel);
        dispatch(ref_lbvh::fill_lbvh_main, wg);
        double t3 = omp_now();
        if (walk_stride == 1) dispatch_par(ref_barnes_hut::bh_vel_step_main, wg, parallel);
        else dispatch_sampled(ref_barnes_hut::bh_vel_step_main, n, walk_stride, parallel);
        double t4 = omp_now();
        dispatch_par(ref_barnes_hut::bh_pos_step_main, wg, parallel);
        double t5 = omp_now();
        stage_s[0] += t1 - t0;
        stage_s[1] += t2 - t1;
        stage_s[2] += t3 - t2;
        stage_s[3] += t4 - t3;
        stage_s[4] += t5 - t4;
    }
    return 0;
}
