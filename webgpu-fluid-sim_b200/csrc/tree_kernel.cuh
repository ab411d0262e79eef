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
// Two phases per climb.  A CTA owns B consecutive slots (128 in the fused
// build, 512 in the split build's local phase).  A node whose
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
// protocol above.  Local nodes hold < B < 1024 bodies, so they all take the
// f32 path below.
//
// Mass / COM: small nodes use the reference's f32 formula
//   M = m_l + m_r;  com = (c_l m_l + c_r m_r) / M  (0 if M <= 0)   (lbvh.wgsl:216-224)
// and nodes of >= kFp64MinBodies bodies aggregate {m, m x, m y} in FP64.
// AABB and length = longest side are exact (lbvh.wgsl:212-213,227-228).
#pragma once

#include <cuda/atomic>

#include "bh_internal.cuh"

namespace bh {

// a / b correctly rounded, given r = 1/b correctly rounded (__frcp_rn): one
// correction of the product a r by its exact residual a - b (a r) (an FMA),
// P. Markstein's final step for IEEE division (IBM J. Res. Dev. 34(1), 1990):
// with r within half an ulp of 1/b and q within an ulp of a/b, q + (a - b q) r
// rounds to a/b.  Operands here are normal-range masses and mass moments
// (b > 0); the build divides two numerators by one mass, so the reciprocal
// is shared and each quotient costs a multiply and two FMAs.
__device__ __forceinline__ float div_by(float a, float b, float r) {
    const float q = __fmul_rn(a, r);
    const float e = __fmaf_rn(-q, b, a);
    return __fmaf_rn(e, r, q);
}

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
    // Split build only: nodes whose parent split is not local, as {first
    // slot, last slot}, and their count (zero before the local phase).
    uint2* frontier = nullptr;
    unsigned int* frontier_count = nullptr;
    // {x, y, m, 0} per body in original order, when the encode wrote them:
    // one gather per slot instead of a position and a mass
    const float4* xm = nullptr;
    // The step's device error word: when an earlier stage of the step failed
    // (kErrSkipMask), the build does nothing.  Null: no such check.
    const uint32_t* err = nullptr;
};

// One thread per sorted slot climbs from its leaf; the lanes of a warp start
// at adjacent leaves, so the low levels they create are adjacent in memory.
// (A persistent variant that hands each finished lane a new leaf measured
// slower at 16M bodies: its lanes drift apart and its node writes scatter.)
// Slots per CTA (measured, B200): the fused build is fastest with small CTAs
// (800k bodies: 128 -> 0.137 ms, 256 -> 0.140, 512 -> 0.150), the local phase
// of the split build with large ones (16.8M: 128 -> 2.11 ms, 256 -> 1.83,
// 512 -> 1.72).  The frontier climb keeps 256 threads per CTA.
#ifndef BH_BUILD_BLOCK_FUSED
#define BH_BUILD_BLOCK_FUSED 128
#endif
#ifndef BH_BUILD_BLOCK_SPLIT
#define BH_BUILD_BLOCK_SPLIT 512
#endif
constexpr int kBuildBlockFused = BH_BUILD_BLOCK_FUSED;
constexpr int kBuildBlockSplit = BH_BUILD_BLOCK_SPLIT;
constexpr int kClimbBlock = 256;
template <bool SPLIT>
constexpr int build_block() { return SPLIT ? kBuildBlockSplit : kBuildBlockFused; }
// Resident CTAs per SM the launch bounds ask for.  The split build's local
// phase issues in only ~60% of its cycles with 2 CTAs of 512 threads (47
// registers); asking for 3 gives 40 registers with 16 B of spills and a
// faster build (16.8M bodies: 1.86 -> 1.71 ms).  The fused build keeps the
// compiler's choice (0: no minimum): 10 or 12 resident CTAs of 128 threads
// (42-51 registers, spills) made it slower at 800k bodies (0.137 -> 0.143 /
// 0.150 ms).
#ifndef BH_BUILD_MIN_BLOCKS_SPLIT
#define BH_BUILD_MIN_BLOCKS_SPLIT 3
#endif
template <bool SPLIT>
constexpr int build_min_blocks() { return SPLIT ? BH_BUILD_MIN_BLOCKS_SPLIT : 0; }
static_assert(kFp64MinBodies > kBuildBlockFused && kFp64MinBodies > kBuildBlockSplit,
              "local nodes must all take the f32 path");

// The block-local shared state of the local phase (B slots per CTA).
template <typename K, int B>
struct BuildShared {
    K key[B + 2];           // keys of slots B0-1 .. B0+B
    int d[B + 1];           // delta at boundary g = B0-1+q (between slots g, g+1)
    int wmin[2][B / 32];    // per-warp minima for the two scans
    int suf[B];             // suf[q] = min of d[q+1..B]
    unsigned char local[B + 1];
    uint32_t bound[B + 1];  // exchange slots of the local splits
    // Leaves by slot - B0 and local internal nodes by index - B0: float4
    // records ({x, y, m, 0}; {cx, cy, m, 0}, box, {S, 0}) for the split
    // build's large CTAs, separate float arrays ([3][B] {m, x, y}; [10][B]
    // {m, cx, cy, box, S}) for the fused build's small ones -- each measured
    // the faster layout for its kernel.
    static constexpr bool kVec = B >= 256;
    alignas(16) float leaf[kVec ? 4 * B : 3 * B];
    alignas(16) float rec[kVec ? 12 * B : 10 * B];
};

// Record access in either layout of BuildShared.  Reads follow the block
// fence after the exchange and writes precede the next one, which orders
// them (the fence is also a compiler barrier); the separate arrays are read
// and written through volatile pointers as before.
template <typename K, int B>
__device__ __forceinline__ float4 shared_leaf(BuildShared<K, B>* S, int k) {
    if constexpr (BuildShared<K, B>::kVec) return reinterpret_cast<const float4*>(S->leaf)[k];
    const volatile float* v = S->leaf;
    return make_float4(v[B + k], v[2 * B + k], v[k], 0.f);
}
template <typename K, int B>
__device__ __forceinline__ void put_leaf(BuildShared<K, B>* S, int k, float4 r) {
    if constexpr (BuildShared<K, B>::kVec) {
        reinterpret_cast<float4*>(S->leaf)[k] = r;
    } else {
        S->leaf[k] = r.z;
        S->leaf[B + k] = r.x;
        S->leaf[2 * B + k] = r.y;
    }
}
template <typename K, int B>
__device__ __forceinline__ void shared_rec(BuildShared<K, B>* S, int k, float4& mom, float4& box,
                                           float4& quad) {
    if constexpr (BuildShared<K, B>::kVec) {
        const float4* r = reinterpret_cast<const float4*>(S->rec);
        mom = r[k];
        box = r[B + k];
        quad = r[2 * B + k];
    } else {
        const volatile float* v = S->rec;
        mom = make_float4(v[B + k], v[2 * B + k], v[k], 0.f);
        box = make_float4(v[3 * B + k], v[4 * B + k], v[5 * B + k], v[6 * B + k]);
        quad = make_float4(v[7 * B + k], v[8 * B + k], v[9 * B + k], 0.f);
    }
}
template <typename K, int B>
__device__ __forceinline__ void put_rec(BuildShared<K, B>* S, int k, float4 mom, float4 box,
                                        float4 quad) {
    if constexpr (BuildShared<K, B>::kVec) {
        float4* r = reinterpret_cast<float4*>(S->rec);
        r[k] = mom;
        r[B + k] = box;
        r[2 * B + k] = quad;
    } else {
        volatile float* v = S->rec;
        v[k] = mom.z;
        v[B + k] = mom.x;
        v[2 * B + k] = mom.y;
        v[3 * B + k] = box.x;
        v[4 * B + k] = box.y;
        v[5 * B + k] = box.z;
        v[6 * B + k] = box.w;
        v[7 * B + k] = quad.x;
        v[8 * B + k] = quad.y;
        v[9 * B + k] = quad.z;
    }
}

// The node a climbing thread currently owns: its slot range, the deltas at
// the range's two boundaries, and its record.
struct Climb {
    uint32_t l, r;
    int dl, dr;
    float cm, cx, cy;
    float lox, loy, hix, hiy;
    float sxx, sxy, syy;       // second moments about the COM (group walk)
    double dm, dmx, dmy;       // valid when the node has >= kFp64MinBodies bodies
    bool local;                // still in the block-local phase
};

// One level of the climb from the node in `c`: returns false when this thread
// is the first to arrive at the split (it stops; the sibling's thread goes
// on) or has created the root, else true with `c` holding the parent.
//   LOCAL: the thread starts in the block-local phase (shared memory `S` of
//          the CTA owning slots [B0, B0 + B)).
//   STOP:  at the first split that is not local, record the node in the
//          frontier list and stop (the split build's first kernel); else go
//          on with the device-scope protocol (fused build, second kernel).
template <typename K, int B, bool LOCAL, bool STOP>
__device__ __forceinline__ bool climb_step(const BuildArgs<K>& A, Climb& c, BuildShared<K, B>* S,
                                           uint32_t B0) {
    const uint32_t n = A.n, nm1 = n - 1;
    bool local = LOCAL && c.local;
    {
        const bool is_left = c.dr > c.dl;
        const uint32_t gamma = is_left ? c.r : c.l - 1;
        int qg = 0;
        if (LOCAL) {
            qg = (int)((long long)gamma - ((long long)B0 - 1));
            local = local && qg >= 1 && qg <= B - 1 && S->local[qg];
            c.local = local;
        }
        if (STOP && !local) {
            // The parent split lies outside this CTA: leave it to the climb kernel.
            A.frontier[atomicAdd(A.frontier_count, 1u)] = make_uint2(c.l, c.r);
            return false;
        }
        // Past the stop test a split build's first kernel is always local;
        // its nodes hold fewer than B bodies, so never take FP64.
        const bool IN_LOCAL = LOCAL && (STOP || local);
        uint32_t other;
        if (IN_LOCAL) {
            // Shared-memory exchange: this node's record (in shared memory)
            // is released to the CTA before the slot changes hands.
            __threadfence_block();
            other = atomicExch(&S->bound[qg], is_left ? c.l : c.r);
            if (other == kSentinel) return false;
            __threadfence_block();
        } else {
            // One acq_rel exchange releases this node's record and acquires
            // the sibling's (release/acquire through bound[gamma]).
            cuda::atomic_ref<uint32_t, cuda::thread_scope_device> slot(A.bound[gamma]);
            other = slot.exchange(is_left ? c.l : c.r, cuda::memory_order_acq_rel);
            if (other == kSentinel) return false;  // first to arrive: the sibling finishes the parent
            slot.store(kSentinel, cuda::memory_order_relaxed);
        }
        const uint32_t pl = is_left ? c.l : other;
        const uint32_t pr = is_left ? other : c.r;
        const uint32_t li = (pl == gamma) ? nm1 + gamma : gamma;
        const uint32_t ri = (pr == gamma + 1) ? nm1 + gamma + 1 : gamma + 1;
        const uint32_t sib = is_left ? ri : li;
        const uint32_t sib_cnt = is_left ? (pr - gamma) : (gamma - pl + 1);
        const uint32_t my_cnt = c.r - c.l + 1;
        float4 s4, sb, sq = make_float4(0.f, 0.f, 0.f, 0.f);
        if (IN_LOCAL) {
            // Sibling record from shared memory.
            if (sib >= nm1) {
                const int k = (int)(sib - nm1 - B0);
                s4 = shared_leaf(S, k);
                sb = make_float4(s4.x, s4.y, s4.x, s4.y);
            } else {
                const int k = (int)(sib - B0);
                shared_rec(S, k, s4, sb, sq);
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
        c.lox = fminf(c.lox, sb.x);
        c.loy = fminf(c.loy, sb.y);
        c.hix = fmaxf(c.hix, sb.z);
        c.hiy = fmaxf(c.hiy, sb.w);
        const uint32_t cnt = pr - pl + 1;
        // Parent's boundary deltas and its own Karras index.
        int dpl, dpr;
        if (is_left) {
            dpl = c.dl;
            dpr = (IN_LOCAL) ? S->d[(int)(pr - B0 + 1)]
                                   : ((pr == nm1) ? -1 : delta_at(A.keys, pr, pr + 1));
        } else {
            dpr = c.dr;
            dpl = (IN_LOCAL) ? S->d[(int)(pl - B0)]
                                   : ((pl == 0) ? -1 : delta_at(A.keys, pl - 1, pl));
        }
        const uint32_t pidx = (pl == 0 && pr == nm1) ? 0u : ((dpr > dpl) ? pr : pl);
        float tm, ncx, ncy;
        if (!STOP && A.fp64 && cnt >= kFp64MinBodies) {
            double sm, smx, smy;
            if (sib_cnt >= kFp64MinBodies) {
                const double2 s0 = __ldcg(&A.big[2 * (size_t)sib]);
                const double2 s1 = __ldcg(&A.big[2 * (size_t)sib + 1]);
                sm = s0.x; smx = s0.y; smy = s1.x;
            } else {
                sm = (double)s4.z; smx = (double)s4.z * (double)s4.x; smy = (double)s4.z * (double)s4.y;
            }
            if (my_cnt < kFp64MinBodies) {
                c.dm = (double)c.cm; c.dmx = (double)c.cm * (double)c.cx; c.dmy = (double)c.cm * (double)c.cy;
            }
            c.dm += sm;
            c.dmx += smx;
            c.dmy += smy;
            tm = (float)c.dm;
            const double inv = c.dm > 0.0 ? 1.0 / c.dm : 0.0;
            ncx = (float)(c.dmx * inv);
            ncy = (float)(c.dmy * inv);
            A.big[2 * (size_t)pidx] = make_double2(c.dm, c.dmx);
            A.big[2 * (size_t)pidx + 1] = make_double2(c.dmy, 0.0);
        } else {
            // (c_l m_l + c_r m_r) / (m_l + m_r).  Each sum is one IEEE addition
            // of two terms, which is commutative, so this node's and the
            // sibling's terms may be summed in either order with the same
            // result; the split build's kernels (B >= 256) skip the left/right
            // selects (16.8M-case build 5% faster), the fused build keeps
            // them (measured 2.5% faster at 800k with them).
            float ml = c.cm, mr = s4.z, clx = c.cx, cly = c.cy, crx = s4.x, cry = s4.y;
            if (B < 256 && !is_left) {
                ml = s4.z; clx = s4.x; cly = s4.y; mr = c.cm; crx = c.cx; cry = c.cy;
            }
            tm = __fadd_rn(ml, mr);
            if (tm > 0.0f) {
                const float inv = __frcp_rn(tm);
                ncx = div_by(__fadd_rn(__fmul_rn(clx, ml), __fmul_rn(crx, mr)), tm, inv);
                ncy = div_by(__fadd_rn(__fmul_rn(cly, ml), __fmul_rn(cry, mr)), tm, inv);
            } else {
                ncx = 0.0f;
                ncy = 0.0f;
            }
        }
        const float len = fmaxf(__fsub_rn(c.hix, c.lox), __fsub_rn(c.hiy, c.loy));
        if (A.gnode) {
            // Second moments about the parent COM:
            // S = sum_c S_c + m_c d_c d_c^T, d_c = c_c - c_parent (leaves: S_c = 0),
            // the two children's terms joined by one (commutative) addition;
            // a and b are this node and its sibling, or (fused build) the
            // left and the right child, as for the centre above.
            float ma = c.cm, mb = s4.z, sax = c.sxx, say = c.sxy, saz = c.syy;
            float sbx = sq.x, sby = sq.y, sbz = sq.z, pax = c.cx, pay = c.cy, pbx = s4.x, pby = s4.y;
            if (B < 256 && !is_left) {
                ma = s4.z; sax = sq.x; say = sq.y; saz = sq.z; pax = s4.x; pay = s4.y;
                mb = c.cm; sbx = c.sxx; sby = c.sxy; sbz = c.syy; pbx = c.cx; pby = c.cy;
            }
            const float dax = __fsub_rn(pax, ncx), day = __fsub_rn(pay, ncy);
            const float dbx = __fsub_rn(pbx, ncx), dby = __fsub_rn(pby, ncy);
            const float madx = __fmul_rn(ma, dax), mady = __fmul_rn(ma, day);
            const float mbdx = __fmul_rn(mb, dbx), mbdy = __fmul_rn(mb, dby);
            c.sxx = __fadd_rn(__fmaf_rn(madx, dax, sax), __fmaf_rn(mbdx, dbx, sbx));
            c.sxy = __fadd_rn(__fmaf_rn(madx, day, say), __fmaf_rn(mbdx, dby, sby));
            c.syy = __fadd_rn(__fmaf_rn(mady, day, saz), __fmaf_rn(mbdy, dby, sbz));
            GNode g;
            g.box = make_float4(c.lox, c.loy, c.hix, c.hiy);
            g.mom = make_float4(ncx, ncy, tm, len);
            g.quad = make_float4(c.sxx, c.sxy, c.syy, 0.0f);
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
            A.aabb[pidx] = make_float4(c.lox, c.loy, c.hix, c.hiy);
            A.children[pidx] = make_uint2(li, ri);
            A.range[pidx] = make_uint2(pl, pr);
        }
        A.parent[li] = pidx;
        A.parent[ri] = pidx;
        if (pidx == 0) {
            A.parent[0] = kSentinel;  // lbvh.wgsl:159-161
            return false;
        }
        if (IN_LOCAL) {
            // the new node is local: its record for the sibling that may meet it here
            const int k = (int)(pidx - B0);
            put_rec(S, k, make_float4(ncx, ncy, tm, 0.0f), make_float4(c.lox, c.loy, c.hix, c.hiy),
                    make_float4(c.sxx, c.sxy, c.syy, 0.0f));
        }
        c.cm = tm; c.cx = ncx; c.cy = ncy;
        c.l = pl;
        c.r = pr;
        c.dl = dpl;
        c.dr = dpr;
    }
    return true;
}

// The whole climb of one thread.
template <typename K, int B, bool LOCAL, bool STOP>
__device__ __forceinline__ void climb(const BuildArgs<K>& A, Climb& c, BuildShared<K, B>* S,
                                      uint32_t B0) {
    while (climb_step<K, B, LOCAL, STOP>(A, c, S, B0)) {
    }
}

// Hierarchy build + fill, one thread per sorted slot.  SPLIT = false: the
// whole climb (fused build, one kernel).  SPLIT = true: only the block-local
// phase; threads that reach a split outside their CTA list their node in the
// frontier and exit, and build_climb_kernel finishes the tree.  A CTA of the
// fused build stays resident while one or two of its threads climb the
// device-scope levels (a few L2 round trips each); the split build frees it
// at the end of its local phase and climbs all frontier nodes side by side,
// which pays off from a few million bodies up (measured: 2.14 -> 1.87 ms at
// 16.8M bodies; at 800k the extra launch costs about as much as it saves).
// (Climbing the local phase in CTA-wide rounds that pack the remaining
// nodes into the lowest warps measured slower.  Nor do the random leaf
// gathers set the pace: with the bodies uploaded in the previous step's
// sorted order, so the gathers run nearly in sequence, the 16.8M-body build
// took 1.80 against 1.84 ms.)
template <typename K, bool SPLIT>
__global__ void __launch_bounds__(build_block<SPLIT>(), build_min_blocks<SPLIT>())
build_fill_kernel(const BuildArgs<K> A) {
    constexpr int B = build_block<SPLIT>();
    // dynamic: sizeof(BuildShared<K, B>) bytes (more than 48 KB for large B)
    extern __shared__ __align__(16) unsigned char build_smem[];
    BuildShared<K, B>& S = *reinterpret_cast<BuildShared<K, B>*>(build_smem);

    const uint32_t n = A.n;
    if (step_failed(A.err)) return;  // uniform over the block
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
        S.key[q] = (g >= 0 && g < (long long)n) ? __ldg(&A.keys[g]) : (K)0;
    }
    for (int q = t; q <= B; q += B) S.bound[q] = kSentinel;
    __syncthreads();
    for (int q = t; q <= B; q += B) {
        const long long g = (long long)B0 - 1 + q;
        S.d[q] = (g < 0 || g >= (long long)nm1)
                     ? -1
                     : delta_keys<K>(S.key[q], S.key[q + 1], (uint32_t)g, (uint32_t)g + 1u);
    }
    __syncthreads();
    {
        const unsigned FULL = 0xFFFFFFFFu;
        // pm = min of d[0..t], sm = min of d[t+1..B]
        int pm = S.d[t], sm = S.d[t + 1];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int a = __shfl_up_sync(FULL, pm, o);
            const int c = __shfl_down_sync(FULL, sm, o);
            if (lane >= o) pm = min(pm, a);
            if (lane + o < 32) sm = min(sm, c);
        }
        if (lane == 31) S.wmin[0][warp] = pm;
        if (lane == 0) S.wmin[1][warp] = sm;
        __syncthreads();
        for (int w = 0; w < warp; ++w) pm = min(pm, S.wmin[0][w]);
        for (int w = warp + 1; w < B / 32; ++w) sm = min(sm, S.wmin[1][w]);
        S.suf[t] = sm;
        __syncthreads();
        // Boundary q = t + 1 splits a local node when a smaller delta lies
        // among d[0..q-1] (= pm) and among d[q+1..B] (= suf[q]).
        const int q = t + 1;
        if (q <= B - 1) S.local[q] = (pm < S.d[q] && S.suf[q] < S.d[q]) ? 1 : 0;
        if (t == 0) {
            S.local[0] = 0;
            S.local[B] = 0;
        }
        __syncthreads();
    }
    if (i >= n) return;

    const uint32_t body = __ldg(&A.ids[i]);
    float m;
    float2 p;
    if (A.xm) {
        const float4 r = __ldg(&A.xm[body]);
        m = r.z;
        p = make_float2(r.x, r.y);
    } else {
        m = __ldg(&A.mass[body]);
        p = __ldg(&A.pos[body]);
    }
    A.node4[nm1 + i] = make_float4(p.x, p.y, m, 0.0f);  // leaf (lbvh.wgsl:179-187)
    put_leaf(&S, t, make_float4(p.x, p.y, m, 0.0f));
    Climb c;
    c.l = i;
    c.r = i;
    // delta at the two boundaries of the current range (-1 outside [0, n-1]);
    // a parent keeps one of them, so each level computes only one new delta.
    c.dl = S.d[t];
    c.dr = S.d[t + 1];
    c.cm = m; c.cx = p.x; c.cy = p.y;
    c.lox = p.x; c.loy = p.y; c.hix = p.x; c.hiy = p.y;
    c.sxx = 0.0f; c.sxy = 0.0f; c.syy = 0.0f;
    c.dm = 0.0; c.dmx = 0.0; c.dmy = 0.0;
    c.local = true;
    climb<K, B, true, SPLIT>(A, c, &S, B0);
}

// Second kernel of the split build: one thread per frontier node (a node
// made in the local phase, or a leaf, whose parent split is outside its
// CTA) continues the climb with the device-scope protocol.  The node's
// record is read back from the tree arrays the first kernel wrote; no
// frontier node is large enough for the FP64 path (local nodes hold fewer
// than kBuildBlockSplit < kFp64MinBodies bodies).  Each climb ends without
// waiting for any other thread, so a thread may take several entries.
template <typename K>
__global__ void __launch_bounds__(kClimbBlock)
build_climb_kernel(const BuildArgs<K> A) {
    if (step_failed(A.err)) return;
    const uint32_t count = *A.frontier_count;
    const uint32_t n = A.n, nm1 = n - 1;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < count; e += gridDim.x * blockDim.x) {
        const uint2 f = A.frontier[e];
        Climb c;
        c.l = f.x;
        c.r = f.y;
        c.dl = (c.l == 0) ? -1 : delta_at(A.keys, c.l - 1, c.l);
        c.dr = (c.r == nm1) ? -1 : delta_at(A.keys, c.r, c.r + 1);
        c.sxx = 0.0f; c.sxy = 0.0f; c.syy = 0.0f;
        c.dm = 0.0; c.dmx = 0.0; c.dmy = 0.0;
        c.local = false;
        if (c.l == c.r) {
            const float4 leaf = A.node4[nm1 + c.l];
            c.cm = leaf.z; c.cx = leaf.x; c.cy = leaf.y;
            c.lox = leaf.x; c.loy = leaf.y; c.hix = leaf.x; c.hiy = leaf.y;
        } else {
            // Karras index: the range end next to the parent's split.
            const uint32_t idx = (c.dr > c.dl) ? c.r : c.l;
            float4 box, mom;
            if (A.gnode) {
                box = A.gnode[idx].box;
                mom = A.gnode[idx].mom;
                const float4 q = A.gnode[idx].quad;
                c.sxx = q.x; c.sxy = q.y; c.syy = q.z;
            } else {
                box = A.aabb[idx];
                mom = A.node4[idx];
            }
            c.cm = mom.z; c.cx = mom.x; c.cy = mom.y;
            c.lox = box.x; c.loy = box.y; c.hix = box.z; c.hiy = box.w;
        }
        climb<K, kBuildBlockSplit, false, false>(A, c, nullptr, 0u);
    }
}

}  // namespace bh
