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
__global__ void __launch_bounds__(256)
build_fill_kernel(const K* __restrict__ keys, const uint32_t* __restrict__ ids,
                  const float* __restrict__ mass, const float2* __restrict__ pos,
                  float4* __restrict__ node4, uint2* __restrict__ children,
                  uint32_t* __restrict__ parent, float4* __restrict__ aabb,
                  uint2* __restrict__ range, double2* __restrict__ big,
                  uint32_t* __restrict__ bound, uint32_t n, int fp64,
                  GNode* __restrict__ gnode, uint2* __restrict__ groups,
                  unsigned int* __restrict__ group_count, uint32_t gmax) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t nm1 = n - 1;
    const uint32_t body = __ldg(&ids[i]);
    const float m = __ldg(&mass[body]);
    const float2 p = __ldg(&pos[body]);
    node4[nm1 + i] = make_float4(p.x, p.y, m, 0.0f);  // leaf (lbvh.wgsl:179-187)
    if (n == 1) {
        // The reference's build has no internal node to run for n == 1
        // (lbvh.wgsl:95-97): the only node keeps its buffer's initial 0.
        parent[0] = 0u;
        if (groups) {
            groups[0] = make_uint2(0u, 1u);
            *group_count = 1u;
        }
        return;
    }
    // Running record of the node this thread currently owns.
    float cm = m, cx = p.x, cy = p.y;
    float lox = p.x, loy = p.y, hix = p.x, hiy = p.y;
    double dm = 0.0, dmx = 0.0, dmy = 0.0;  // valid when the node has >= kFp64MinBodies bodies
    float sxx = 0.0f, sxy = 0.0f, syy = 0.0f;  // second moments about the COM (group walk)
    uint32_t l = i, r = i;
    // delta at the two boundaries of the current range (-1 outside [0, n-1]);
    // a parent keeps one of them, so each level computes only one new delta.
    int dl = (l == 0) ? -1 : delta_at(keys, l - 1, l);
    int dr = (r == nm1) ? -1 : delta_at(keys, r, r + 1);
    while (true) {
        const bool is_left = dr > dl;
        const uint32_t gamma = is_left ? r : l - 1;
        // One acq_rel exchange releases this node's record and acquires the
        // sibling's (release/acquire through bound[gamma]).
        cuda::atomic_ref<uint32_t, cuda::thread_scope_device> slot(bound[gamma]);
        const uint32_t other = slot.exchange(is_left ? l : r, cuda::memory_order_acq_rel);
        if (other == kSentinel) return;  // first to arrive: the sibling finishes the parent
        slot.store(kSentinel, cuda::memory_order_relaxed);
        const uint32_t pl = is_left ? l : other;
        const uint32_t pr = is_left ? other : r;
        const uint32_t li = (pl == gamma) ? nm1 + gamma : gamma;
        const uint32_t ri = (pr == gamma + 1) ? nm1 + gamma + 1 : gamma + 1;
        const uint32_t sib = is_left ? ri : li;
        const uint32_t sib_cnt = is_left ? (pr - gamma) : (gamma - pl + 1);
        const uint32_t my_cnt = r - l + 1;
        // Sibling record through L2 (written by another thread in this launch).
        float4 s4, sb, sq = make_float4(0.f, 0.f, 0.f, 0.f);
        if (sib >= nm1) {
            s4 = __ldcg(&node4[sib]);
            sb = make_float4(s4.x, s4.y, s4.x, s4.y);
        } else if (gnode) {
            sb = __ldcg(&gnode[sib].box);
            s4 = __ldcg(&gnode[sib].mom);
            sq = __ldcg(&gnode[sib].quad);
        } else {
            s4 = __ldcg(&node4[sib]);
            sb = __ldcg(&aabb[sib]);
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
            dpr = (pr == nm1) ? -1 : delta_at(keys, pr, pr + 1);
        } else {
            dpr = dr;
            dpl = (pl == 0) ? -1 : delta_at(keys, pl - 1, pl);
        }
        const uint32_t pidx = (pl == 0 && pr == nm1) ? 0u : ((dpr > dpl) ? pr : pl);
        float tm, ncx, ncy;
        if (fp64 && cnt >= kFp64MinBodies) {
            double sm, smx, smy;
            if (sib_cnt >= kFp64MinBodies) {
                const double2 s0 = __ldcg(&big[2 * (size_t)sib]);
                const double2 s1 = __ldcg(&big[2 * (size_t)sib + 1]);
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
            big[2 * (size_t)pidx] = make_double2(dm, dmx);
            big[2 * (size_t)pidx + 1] = make_double2(dmy, 0.0);
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
        if (gnode) {
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
            gnode[pidx] = g;
        }
        if (groups) {
            // Walk groups: maximal subtrees of <= gmax bodies.  A child is one
            // when its parent is too big; the whole tree is one when n <= gmax.
            if (cnt > gmax) {
                const uint32_t lcnt = gamma - pl + 1, rcnt = pr - gamma;
                if (lcnt <= gmax) groups[atomicAdd(group_count, 1u)] = make_uint2(pl, lcnt);
                if (rcnt <= gmax) groups[atomicAdd(group_count, 1u)] = make_uint2(gamma + 1, rcnt);
            } else if (pidx == 0) {
                groups[atomicAdd(group_count, 1u)] = make_uint2(0u, n);
            }
        }
        node4[pidx] = make_float4(ncx, ncy, tm, len);
        aabb[pidx] = make_float4(lox, loy, hix, hiy);
        children[pidx] = make_uint2(li, ri);
        range[pidx] = make_uint2(pl, pr);
        parent[li] = pidx;
        parent[ri] = pidx;
        if (pidx == 0) {
            parent[0] = kSentinel;  // lbvh.wgsl:159-161
            return;
        }
        cm = tm; cx = ncx; cy = ncy;
        l = pl;
        r = pr;
        dl = dpl;
        dr = dpr;
    }
}

}  // namespace bh
