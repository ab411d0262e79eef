// tree_kernel.cuh -- the fused bottom-up hierarchy build + mass / centre-of-mass
// / AABB fill kernel (included by tree.cu, which launches it for the engine).
//
// Reference: build_lbvh_main (lbvh.wgsl:85-165, Karras 2012 fig. 4) followed by
// fill_lbvh_main (lbvh.wgsl:168-232).  The reference builds top-down with one
// thread per internal node and binary searches, then climbs from the leaves
// with arrival counters but no memory fences, which its README calls a race.
//
// Here one thread per sorted slot climbs from its leaf and creates each
// internal node when it is the second child to arrive (agglomerative build,
// Apetrei 2014), using the same delta(i, j) as lbvh.wgsl:72-83:
//   delta = clz(k_i ^ k_j), or key_bits + clz(i ^ j) for equal keys, -1 outside.
// A node covering sorted slots [l, r] is the left child of its parent when
// delta(r, r+1) > delta(l-1, l), and the parent's split is then r; otherwise it
// is the right child and the split is l-1.  Karras numbers an internal node by
// the end of its range next to its parent's split (a left child by its last
// slot, a right child by its first slot, the root is 0), and its children are
// gamma / gamma+1, or the leaves n-1+gamma / n+gamma when a side holds one slot
// (lbvh.wgsl:141-152).  Computing those indices here gives the same
// left/right/parent arrays as the reference's top-down build, bit for bit.
//
// Synchronisation: the two children of a split gamma meet at bound[gamma] with
// an atomic exchange of their far range ends; the first arriver stops.  The
// exchange is acq_rel at device scope: it releases the node record this
// thread wrote and acquires the sibling's, which the second arriver then reads
// through L2 (__ldcg), so no stale data is ever combined.  There are no spins.
// bound[] holds kSentinel between steps: the second arriver restores it.
//
// Two phases per climb.  A CTA owns 256 consecutive slots.  A node whose
// range lies inside those slots ("local") is combined through shared memory:
// its split's exchange slot is a shared-memory word, the sibling's record is
// read from shared memory, and block-scope fences suffice.  Which splits are
// local follows from the boundary deltas alone: the node split at boundary g
// spans from just after the nearest boundary on its left with a smaller
// delta to the nearest one on its right with a smaller delta (the hierarchy
// is the Cartesian tree of the boundary deltas, whose values are distinct
// between two smaller ones), so it is local when both of those boundaries
// are among the CTA's own, i.e. when the prefix and suffix minima of the
// CTA's deltas around g are below delta(g).  A climb leaves the local phase
// at the first split that is not local and continues with the device-scope
// protocol above.  Local nodes hold < 256 bodies, so they all take the f32
// path below.
//
// Mass / COM: small nodes use the reference's f32 formula
//   M = m_l + m_r;  com = (c_l m_l + c_r m_r) / M  (0 if M <= 0)   (lbvh.wgsl:216-224)
// and nodes of >= kFp64MinBodies bodies aggregate {m, m x, m y} in FP64.
// AABB and length = longest side are exact (lbvh.wgsl:212-213,227-228).
#pragma once

#include <cuda/atomic>

#include "bh_internal.cuh"

namespace bh {

template <typename K>
__device__ __forceinline__ int delta_at(const K* __restrict__ keys, uint32_t i, uint32_t j) {
    K a = __ldg(&keys[i]), b = __ldg(&keys[j]);
    if (a == b) return (int)(8 * sizeof(K)) + __clz((int)(i ^ j));
    if (sizeof(K) == 8) return __clzll((long long)(a ^ b));
    return __clz((int)(uint32_t)(a ^ b));
}

template <typename K>
__device__ __forceinline__ int delta_keys(K a, K b, uint32_t i, uint32_t j) {
    if (a == b) return (int)(8 * sizeof(K)) + __clz((int)(i ^ j));
    if (sizeof(K) == 8) return __clzll((long long)(a ^ b));
    return __clz((int)(uint32_t)(a ^ b));
}

// Kernel arguments (device pointers; gnode / groups / group_count are null
// when the caller needs no group-walk records).
template <typename K>
struct BuildArgs {
    const K* keys;
    const uint32_t* ids;
    const float* mass;
    const float2* pos;
    float4* node4;
    uint2* children;
    uint32_t* parent;
    float4* aabb;
    uint2* range;
    double2* big;
    uint32_t* bound;
    uint32_t n;
    int fp64;
    GNode* gnode;
    uint2* groups;
    unsigned int* group_count;
    uint32_t gmax;
};

// One thread per sorted slot climbs from its leaf; the lanes of a warp start
// at adjacent leaves, so the low levels they create are adjacent in memory.
// (A persistent variant that hands each finished lane a new leaf measured
// slower at 16M bodies: its lanes drift apart and its node writes scatter.)
constexpr int kBuildBlock = 256;
static_assert(kFp64MinBodies > kBuildBlock, "local nodes must all take the f32 path");

template <typename K>
__global__ void __launch_bounds__(kBuildBlock)
build_fill_kernel(const BuildArgs<K> A) {
    constexpr int B = kBuildBlock;
    __shared__ K s_key[B + 2];            // keys of slots B0-1 .. B0+B
    __shared__ int s_d[B + 1];            // delta at boundary g = B0-1+q (between slots g, g+1)
    __shared__ int s_wmin[2][B / 32];     // per-warp minima for the two scans
    __shared__ int s_suf[B];              // s_suf[q] = min of s_d[q+1..B]
    __shared__ unsigned char s_local[B + 1];
    __shared__ uint32_t s_bound[B + 1];   // exchange slots of the local splits
    __shared__ float s_leaf[3][B];        // leaf {m, x, y} by slot - B0
    __shared__ float s_rec[10][B];        // local internal node {m, cx, cy, box, S} by index - B0

    const uint32_t n = A.n;
    const int t = (int)threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t B0 = blockIdx.x * (uint32_t)B;
    const uint32_t i = B0 + (uint32_t)t;
    if (n == 1) {
        if (t == 0) {
            const uint32_t body = __ldg(&A.ids[0]);
            const float2 p = __ldg(&A.pos[body]);
            A.node4[0] = make_float4(p.x, p.y, __ldg(&A.mass[body]), 0.0f);  // lbvh.wgsl:179-187
            // The reference's build has no internal node to run for n == 1
            // (lbvh.wgsl:95-97): the only node keeps its buffer's initial 0.
            A.parent[0] = 0u;
            if (A.groups) {
                A.groups[0] = make_uint2(0u, 1u);
                *A.group_count = 1u;
            }
        }
        return;
    }
    const uint32_t nm1 = n - 1;
    // ---- boundary deltas of the CTA's slots and which splits are local ----
    for (int q = t; q < B + 2; q += B) {
        const long long g = (long long)B0 - 1 + q;
        s_key[q] = (g >= 0 && g < (long long)n) ? __ldg(&A.keys[g]) : (K)0;
    }
    for (int q = t; q <= B; q += B) s_bound[q] = kSentinel;
    __syncthreads();
    for (int q = t; q <= B; q += B) {
        const long long g = (long long)B0 - 1 + q;
        s_d[q] = (g < 0 || g >= (long long)nm1)
                     ? -1
                     : delta_keys<K>(s_key[q], s_key[q + 1], (uint32_t)g, (uint32_t)g + 1u);
    }
    __syncthreads();
    {
        const unsigned FULL = 0xFFFFFFFFu;
        // pm = min of s_d[0..t], sm = min of s_d[t+1..B]
        int pm = s_d[t], sm = s_d[t + 1];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int a = __shfl_up_sync(FULL, pm, o);
            const int c = __shfl_down_sync(FULL, sm, o);
            if (lane >= o) pm = min(pm, a);
            if (lane + o < 32) sm = min(sm, c);
        }
        if (lane == 31) s_wmin[0][warp] = pm;
        if (lane == 0) s_wmin[1][warp] = sm;
        __syncthreads();
        for (int w = 0; w < warp; ++w) pm = min(pm, s_wmin[0][w]);
        for (int w = warp + 1; w < B / 32; ++w) sm = min(sm, s_wmin[1][w]);
        s_suf[t] = sm;
        __syncthreads();
        // Boundary q = t + 1 splits a local node when a smaller delta lies
        // among s_d[0..q-1] (= pm) and among s_d[q+1..B] (= s_suf[q]).
        const int q = t + 1;
        if (q <= B - 1) s_local[q] = (pm < s_d[q] && s_suf[q] < s_d[q]) ? 1 : 0;
        if (t == 0) {
            s_local[0] = 0;
            s_local[B] = 0;
        }
        __syncthreads();
    }
    if (i >= n) return;

    const uint32_t body = __ldg(&A.ids[i]);
    const float m = __ldg(&A.mass[body]);
    const float2 p = __ldg(&A.pos[body]);
    A.node4[nm1 + i] = make_float4(p.x, p.y, m, 0.0f);  // leaf (lbvh.wgsl:179-187)
    s_leaf[0][t] = m;
    s_leaf[1][t] = p.x;
    s_leaf[2][t] = p.y;
    // Running record of the node this thread currently owns.
    float cm = m, cx = p.x, cy = p.y;
    float lox = p.x, loy = p.y, hix = p.x, hiy = p.y;
    double dm = 0.0, dmx = 0.0, dmy = 0.0;  // valid when the node has >= kFp64MinBodies bodies
    float sxx = 0.0f, sxy = 0.0f, syy = 0.0f;  // second moments about the COM (group walk)
    uint32_t l = i, r = i;
    // delta at the two boundaries of the current range (-1 outside [0, n-1]);
    // a parent keeps one of them, so each level computes only one new delta.
    int dl = s_d[t], dr = s_d[t + 1];
    bool local = true;
    volatile float* vrec = &s_rec[0][0];
    volatile float* vleaf = &s_leaf[0][0];
    while (true) {
        const bool is_left = dr > dl;
        const uint32_t gamma = is_left ? r : l - 1;
        const int qg = (int)((long long)gamma - ((long long)B0 - 1));
        local = local && qg >= 1 && qg <= B - 1 && s_local[qg];
        uint32_t other;
        if (local) {
            // Shared-memory exchange: this node's record (in shared memory)
            // is released to the CTA before the slot changes hands.
            __threadfence_block();
            other = atomicExch(&s_bound[qg], is_left ? l : r);
            if (other == kSentinel) return;
            __threadfence_block();
        } else {
            // One acq_rel exchange releases this node's record and acquires
            // the sibling's (release/acquire through bound[gamma]).
            cuda::atomic_ref<uint32_t, cuda::thread_scope_device> slot(A.bound[gamma]);
            other = slot.exchange(is_left ? l : r, cuda::memory_order_acq_rel);
            if (other == kSentinel) return;  // first to arrive: the sibling finishes the parent
            slot.store(kSentinel, cuda::memory_order_relaxed);
        }
        const uint32_t pl = is_left ? l : other;
        const uint32_t pr = is_left ? other : r;
        const uint32_t li = (pl == gamma) ? nm1 + gamma : gamma;
        const uint32_t ri = (pr == gamma + 1) ? nm1 + gamma + 1 : gamma + 1;
        const uint32_t sib = is_left ? ri : li;
        const uint32_t sib_cnt = is_left ? (pr - gamma) : (gamma - pl + 1);
        const uint32_t my_cnt = r - l + 1;
        float4 s4, sb, sq = make_float4(0.f, 0.f, 0.f, 0.f);
        if (local) {
            // Sibling record from shared memory.
            if (sib >= nm1) {
                const int k = (int)(sib - nm1 - B0);
                s4 = make_float4(vleaf[B + k], vleaf[2 * B + k], vleaf[k], 0.f);
                sb = make_float4(s4.x, s4.y, s4.x, s4.y);
            } else {
                const int k = (int)(sib - B0);
                s4 = make_float4(vrec[B + k], vrec[2 * B + k], vrec[k], 0.f);
                sb = make_float4(vrec[3 * B + k], vrec[4 * B + k], vrec[5 * B + k], vrec[6 * B + k]);
                sq = make_float4(vrec[7 * B + k], vrec[8 * B + k], vrec[9 * B + k], 0.f);
            }
        } else if (sib >= nm1) {
            // Sibling record through L2 (written by another thread in this launch).
            s4 = __ldcg(&A.node4[sib]);
            sb = make_float4(s4.x, s4.y, s4.x, s4.y);
        } else if (A.gnode) {
            sb = __ldcg(&A.gnode[sib].box);
            s4 = __ldcg(&A.gnode[sib].mom);
            sq = __ldcg(&A.gnode[sib].quad);
        } else {
            s4 = __ldcg(&A.node4[sib]);
            sb = __ldcg(&A.aabb[sib]);
        }
        lox = fminf(lox, sb.x);
        loy = fminf(loy, sb.y);
        hix = fmaxf(hix, sb.z);
        hiy = fmaxf(hiy, sb.w);
        const uint32_t cnt = pr - pl + 1;
        // Parent's boundary deltas and its own Karras index.
        int dpl, dpr;
        if (is_left) {
            dpl = dl;
            dpr = local ? s_d[(int)(pr - B0 + 1)] : ((pr == nm1) ? -1 : delta_at(A.keys, pr, pr + 1));
        } else {
            dpr = dr;
            dpl = local ? s_d[(int)(pl - B0)] : ((pl == 0) ? -1 : delta_at(A.keys, pl - 1, pl));
        }
        const uint32_t pidx = (pl == 0 && pr == nm1) ? 0u : ((dpr > dpl) ? pr : pl);
        float tm, ncx, ncy;
        if (A.fp64 && cnt >= kFp64MinBodies) {
            double sm, smx, smy;
            if (sib_cnt >= kFp64MinBodies) {
                const double2 s0 = __ldcg(&A.big[2 * (size_t)sib]);
                const double2 s1 = __ldcg(&A.big[2 * (size_t)sib + 1]);
                sm = s0.x; smx = s0.y; smy = s1.x;
            } else {
                sm = (double)s4.z; smx = (double)s4.z * (double)s4.x; smy = (double)s4.z * (double)s4.y;
            }
            if (my_cnt < kFp64MinBodies) {
                dm = (double)cm; dmx = (double)cm * (double)cx; dmy = (double)cm * (double)cy;
            }
            dm += sm;
            dmx += smx;
            dmy += smy;
            tm = (float)dm;
            ncx = dm > 0.0 ? (float)(dmx / dm) : 0.0f;
            ncy = dm > 0.0 ? (float)(dmy / dm) : 0.0f;
            A.big[2 * (size_t)pidx] = make_double2(dm, dmx);
            A.big[2 * (size_t)pidx + 1] = make_double2(dmy, 0.0);
        } else {
            float ml, mr, clx, cly, crx, cry;
            if (is_left) { ml = cm; clx = cx; cly = cy; mr = s4.z; crx = s4.x; cry = s4.y; }
            else { ml = s4.z; clx = s4.x; cly = s4.y; mr = cm; crx = cx; cry = cy; }
            tm = __fadd_rn(ml, mr);
            if (tm > 0.0f) {
                ncx = __fdiv_rn(__fadd_rn(__fmul_rn(clx, ml), __fmul_rn(crx, mr)), tm);
                ncy = __fdiv_rn(__fadd_rn(__fmul_rn(cly, ml), __fmul_rn(cry, mr)), tm);
            } else {
                ncx = 0.0f;
                ncy = 0.0f;
            }
        }
        const float len = fmaxf(__fsub_rn(hix, lox), __fsub_rn(hiy, loy));
        if (A.gnode) {
            // Second moments about the parent COM, left child first:
            // S = sum_c S_c + m_c d_c d_c^T, d_c = c_c - c_parent (leaves: S_c = 0).
            float ml, mr, lxx, lxy, lyy, rxx, rxy, ryy, dlx, dly, drx, dry;
            if (is_left) {
                ml = cm; lxx = sxx; lxy = sxy; lyy = syy; dlx = __fsub_rn(cx, ncx); dly = __fsub_rn(cy, ncy);
                mr = s4.z; rxx = sq.x; rxy = sq.y; ryy = sq.z; drx = __fsub_rn(s4.x, ncx); dry = __fsub_rn(s4.y, ncy);
            } else {
                ml = s4.z; lxx = sq.x; lxy = sq.y; lyy = sq.z; dlx = __fsub_rn(s4.x, ncx); dly = __fsub_rn(s4.y, ncy);
                mr = cm; rxx = sxx; rxy = sxy; ryy = syy; drx = __fsub_rn(cx, ncx); dry = __fsub_rn(cy, ncy);
            }
            sxx = __fadd_rn(__fadd_rn(lxx, __fmul_rn(ml, __fmul_rn(dlx, dlx))),
                            __fadd_rn(rxx, __fmul_rn(mr, __fmul_rn(drx, drx))));
            sxy = __fadd_rn(__fadd_rn(lxy, __fmul_rn(ml, __fmul_rn(dlx, dly))),
                            __fadd_rn(rxy, __fmul_rn(mr, __fmul_rn(drx, dry))));
            syy = __fadd_rn(__fadd_rn(lyy, __fmul_rn(ml, __fmul_rn(dly, dly))),
                            __fadd_rn(ryy, __fmul_rn(mr, __fmul_rn(dry, dry))));
            GNode g;
            g.box = make_float4(lox, loy, hix, hiy);
            g.mom = make_float4(ncx, ncy, tm, len);
            g.quad = make_float4(sxx, sxy, syy, 0.0f);
            g.link = make_uint4(li, ri, pl, cnt);
            A.gnode[pidx] = g;
        }
        if (A.groups) {
            // Walk groups: maximal subtrees of <= gmax bodies.  A child is one
            // when its parent is too big; the whole tree is one when n <= gmax.
            if (cnt > A.gmax) {
                const uint32_t lcnt = gamma - pl + 1, rcnt = pr - gamma;
                if (lcnt <= A.gmax) A.groups[atomicAdd(A.group_count, 1u)] = make_uint2(pl, lcnt);
                if (rcnt <= A.gmax) A.groups[atomicAdd(A.group_count, 1u)] = make_uint2(gamma + 1, rcnt);
            } else if (pidx == 0) {
                A.groups[atomicAdd(A.group_count, 1u)] = make_uint2(0u, n);
            }
        }
        if (!A.gnode) {
            // Reference layout (lbvh.wgsl:12-22, split into hot and cold
            // arrays).  With the packed records it is derived on request
            // (ref_layout_kernel): four scattered 8-16 B writes per node
            // fewer in every step.
            A.node4[pidx] = make_float4(ncx, ncy, tm, len);
            A.aabb[pidx] = make_float4(lox, loy, hix, hiy);
            A.children[pidx] = make_uint2(li, ri);
            A.range[pidx] = make_uint2(pl, pr);
        }
        A.parent[li] = pidx;
        A.parent[ri] = pidx;
        if (pidx == 0) {
            A.parent[0] = kSentinel;  // lbvh.wgsl:159-161
            return;
        }
        if (local) {
            // the new node is local: its record for the sibling that may meet it here
            const int k = (int)(pidx - B0);
            vrec[k] = tm;
            vrec[B + k] = ncx;
            vrec[2 * B + k] = ncy;
            vrec[3 * B + k] = lox;
            vrec[4 * B + k] = loy;
            vrec[5 * B + k] = hix;
            vrec[6 * B + k] = hiy;
            vrec[7 * B + k] = sxx;
            vrec[8 * B + k] = sxy;
            vrec[9 * B + k] = syy;
        }
        cm = tm; cx = ncx; cy = ncy;
        l = pl;
        r = pr;
        dl = dpl;
        dr = dpr;
    }
}

}  // namespace bh
