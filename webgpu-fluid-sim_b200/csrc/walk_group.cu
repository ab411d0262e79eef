// walk_group.cu -- group tree walk with quadrupole moments (extension).
//
// No reference counterpart as a whole: it replaces bh_vel_step_main
// (barnes_hut.wgsl:48-111) + bh_pos_step_main (:113-120) when the
// configuration asks for the group walk.  The reference's per-body monopole
// walk has a median relative force error of order 1e-2 at theta = 0.5 in 2D;
// this walk reaches <= 1e-3 at the same theta.
//
// One warp owns a group: a maximal subtree of at most G = 32 x BPL bodies, so
// its bodies are contiguous sorted slots inside one Morton cell (the build
// kernel lists the groups).  Fixed runs of G slots would not do: a run that
// straddles a jump of the Z curve has a box spanning far-apart regions and
// opens nearly every node.  (Cutting maximal 2G-body subtrees into G-slot
// runs fills more lanes but opens more nodes; measured slower.  So did
// stack entries that stand for both children of an opened node -- adjacent
// in the Karras numbering, one round trip for the pair -- which halve the
// dependent steps but double the emission work per step and the registers.)  The group
// accepts a node when
//     L^2 < theta^2 d^2,  L = longest side of the node's box,
//     d = distance from the group's box to the node's COM,
// and the node's box lies apart from the group's box (group_accepts); then
// every body of the group meets the per-body test length / |com - x| <
// theta.  Other nodes are opened.  Accepted nodes act through their monopole and
// (multipole order 2) quadrupole about the COM,
//     a = G [ M r/|r|^3 - Q'r/|r|^5 + 5/2 (r.Q'r) r/|r|^7 ],  Q' = 3S - tr(S) I,
// with r = com - x and |r|^2 = r.r + eps^2 (S = second moments about the COM).
// Leaves, and opened nodes of <= leaf_size bodies, are summed body by body.
//
// Traversal: a per-warp stack in shared memory.  Every step each lane takes
// one of the top 32 stack entries, loads its whole 64-B record in one round
// trip, evaluates it, and the warp compacts the outcomes (ballots and a
// warp scan) into a node list, a body-slot list and the stack.  Lists are
// evaluated when they hold >= 32 entries: every lane runs every entry for its
// BPL bodies (shared-memory broadcasts, no divergence); body records are
// first loaded 32 at a time by the 32 lanes in parallel.
// Above kGroupDfsAt entries the warp pops one node per step (plain DFS), which
// keeps the stack below kGroupStack for any tree of depth <= 96; a push that
// would not fit raises kErrGroupStack instead of writing out of bounds.
// Groups are taken from an atomic counter (the walk is persistent).
//
// Packed arithmetic: with BPL >= 2 each lane evaluates its bodies in pairs
// with the sm_100 packed FP32 instructions (add/sub/mul/fma .rn.f32x2), one
// instruction for both bodies.  Node-list entries are stored in shared memory
// with every value duplicated ({cx,cx,cy,cy}, ...), so a 128-bit shared load
// yields ready operand pairs, and with the quadrupole negated so every
// accumulation is a plain fused multiply-add.  With eps^2 > 0 a body's own
// leaf adds exactly zero (r = 0), so no self test is needed.
//
// Far field (far_alpha > 0, extension): an accepted node whose COM lies far
// from the group compared with the group's size (r_g < far_alpha R, r_g the
// group box's half-diagonal, R the distance from the box centre to the COM)
// is not evaluated body by body.  Lanes turn 32 such nodes at a time into
// the coefficients of a local expansion about the box centre, each lane
// summing its own in registers; at the end of the group the lanes' sums are
// reduced and every body evaluates the expansion once (far_field.cuh).
#include "bh_internal.cuh"
#include "far_field.cuh"
#include "packed.cuh"

namespace bh {

// Per-warp stack entries.  Shared memory and L1 share each SM's 256 KB, so
// every byte of stack is L1 the node records lose: 320 entries instead of
// 384 put 6 far-field blocks per SM in a 196 KB carve-out instead of 228
// (16.8M bodies: walk 7.67 -> 7.50 ms).  256 entries were slower (0.391 ->
// 0.407 ms at 800k): more warps reach the one-node-per-step depth guard.
constexpr int kWalkStack = 320;
constexpr int kWalkDfsAt = kWalkStack - 128;  // >= 32 + 96 below the capacity

constexpr int kSlotList = 32 + 32 * kGroupMaxLeaf;  // body slots: < 32 kept + one step's adds
// Node list entries.  Without the far field the multipole list is flushed
// at 32 entries, so it holds < 64 after any step.  With it, multipole
// entries grow from the bottom and far entries from the top; both lists are
// flushed at 32 entries, so before a step each holds < 32 and one step adds
// at most 32 in all: < 96 together.
template <bool FAR>
struct GroupSmem {
    static constexpr int kListCap = FAR ? 96 : kGroupList;
    uint32_t stack[kWalkStack];
    // node entry j: ent[j][0] = {cx, cx, cy, cy}, ent[j][1] = {m, m, -Q'xx, -Q'xx},
    //               ent[j][2] = {-Q'xy, -Q'xy, -Q'yy, -Q'yy}
    // far entry j (at kListCap - 1 - j): {cx, cy, m, Sxx}, {Sxy, Syy, 0, 0}
    float4 ent[kListCap][3];
    uint32_t slot[kSlotList];  // sorted slots of bodies to sum one by one
    float4 body[32][2];        // 32 staged leaf records as pairs {x,x,y,y}, {m,m,0,0}
};

// Far list: the top `cnt` (<= 32) far entries of `nf_total`, one per lane,
// added to the lane's local-expansion sums.  Not inlined: the coefficient
// arithmetic is the walk's register peak, and as a call (the caller's live
// values saved around it, the sums in a 56-B stack frame) the 128-body
// far-field walk fits 6 blocks per SM in 80 registers instead of 5 in 96.
// A call costs little once per 32 far nodes (800k bodies: walk 0.399 ->
// 0.392 ms; 16.8M: 7.87 -> 7.69 ms).
__device__ __noinline__ void far_batch(GroupSmem<true>& S, float (&cacc)[kFarCoeffs], int lane,
                                          int nf_total, int cnt, float gcx, float gcy, float lam,
                                          float eps2) {
    constexpr int cap = GroupSmem<true>::kListCap;
    if (lane < cnt) {
        const int j = nf_total - cnt + lane;
        const float4 a = S.ent[cap - 1 - j][0];
        const float4 b = S.ent[cap - 1 - j][1];
        far_node_coeffs(cacc, __fsub_rn(gcx, a.x), __fsub_rn(gcy, a.y), a.z, a.w, b.x, b.y, lam,
                        eps2);
    }
    __syncwarp();
}

// Register budget: launch bounds for blocks of up to 256 threads with 3
// resident per SM for groups of <= 64 bodies (at most 85 registers, the
// budget of 6 resident 128-thread blocks); for 128-body groups blocks of up
// to 128 threads with 6 resident (at most 85: 80 for the far-field walk with
// its coefficient routine called, not inlined).  The bound does not depend
// on the block shape chosen at launch (walk_block: 64, 128 or, for groups of
// <= 64 bodies, 256 threads), so the shape leaves the warps resident per SM
// unchanged.  (An explicit register cap of 72 in place of these bounds gave
// a 65-register build of the 64-body walk that ran 12% slower.)
constexpr int walk_max_threads(int bpl) { return bpl >= 4 ? 128 : 256; }
#ifndef BH_WALK_MIN_BLOCKS_128
#define BH_WALK_MIN_BLOCKS_128 6
#endif
constexpr int walk_min_blocks(int bpl) { return bpl >= 4 ? BH_WALK_MIN_BLOCKS_128 : 3; }

// FAR: the far-field variant (Plummer softening, quadrupoles); the other
// instantiations carry none of its code or registers.  COUNT: the
// instrumented walk of bh_walk_stats, which also counts node visits and
// interactions; the stepping walk carries no counters (as a runtime switch
// their four 64-bit sums held 8 registers through the whole traversal and
// cost 5% at 800k and 16.8M bodies, 8% for 64-body groups).  Shared memory:
// one GroupSmem<FAR> per warp, dynamic (the block shape is chosen at
// launch).
template <int BPL, int MP, bool PLUMMER, bool FAR, bool COUNT>
__global__ void __launch_bounds__(walk_max_threads(BPL), walk_min_blocks(BPL))
walk_group_kernel(const GNode* __restrict__ gnode, const float4* __restrict__ node4,
                  const uint2* __restrict__ groups, const uint32_t* __restrict__ ids,
                  float2* __restrict__ pos, float2* __restrict__ vel, float2* __restrict__ acc,
                  const WalkParams P, uint32_t* __restrict__ err) {
    constexpr int NP = BPL / 2;  // packed pairs per lane (BPL >= 2)
    extern __shared__ __align__(16) unsigned char walk_smem[];
    GroupSmem<FAR>* smem = reinterpret_cast<GroupSmem<FAR>*>(walk_smem);
    if (step_failed(err)) return;  // the tree of this step was not built
    const int lane = threadIdx.x & 31;
    GroupSmem<FAR>& S = smem[threadIdx.x >> 5];
    const unsigned FULL = 0xFFFFFFFFu;
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t n = P.n, nm1 = n - 1;
    const uint32_t ngroups = P.group_ctr[1];  // written by the build kernel
    const float th2 = __fmul_rn(P.theta, P.theta);
    const float eps2 = P.eps2, ecoef = P.eps_coef;
    // With a positive softening the own-leaf term is exactly zero.
    const bool self_test = !(PLUMMER && eps2 > 0.0f);
    constexpr bool counting = COUNT;
    unsigned long long c_vis = 0, c_node = 0, c_body = 0, c_far = 0;
    const int stack_cap = (P.stack_cap > 0 && P.stack_cap < kWalkStack) ? P.stack_cap : kWalkStack;

    while (true) {
        uint32_t g = 0;
        if (lane == 0) g = atomicAdd(P.group_ctr, 1u);
        g = __shfl_sync(FULL, g, 0);
        if (g >= ngroups) break;
        // A group is a subtree of <= 32 x BPL bodies: contiguous sorted slots
        // inside one Morton cell, so its box stays compact.
        const uint2 grp = __ldg(&groups[g]);
        if (grp.x < P.slot_lo || grp.x >= P.slot_hi) continue;  // another shard's group
        const uint32_t base = grp.x, nvalid = grp.y;
        const int kmax = (int)((nvalid + 31u) / 32u);  // sub-slots in use (uniform)
        // Ensemble: the slot range of this group's system (systems stay
        // contiguous in sorted order because the system id tops every key).
        uint32_t sys_lo = 0, sys_hi = n;
        if (P.num_systems > 0) {
            uint32_t lo = 0, hi = P.num_systems;  // sys_off[lo] <= base < sys_off[hi]
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (__ldg(&P.sys_off[mid]) <= base) lo = mid;
                else hi = mid;
            }
            sys_lo = __ldg(&P.sys_off[lo]);
            sys_hi = __ldg(&P.sys_off[lo + 1]);
        }
        float bx[BPL], by[BPL], bm[BPL];
        float glox = INFINITY, gloy = INFINITY, ghix = -INFINITY, ghiy = -INFINITY;
#pragma unroll
        for (int k = 0; k < BPL; ++k) {
            float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
            if ((uint32_t)k * 32u + (uint32_t)lane < nvalid) {
                r = __ldg(&node4[nm1 + base + (uint32_t)k * 32u + (uint32_t)lane]);
                glox = fminf(glox, r.x); gloy = fminf(gloy, r.y);
                ghix = fmaxf(ghix, r.x); ghiy = fmaxf(ghiy, r.y);
            }
            bx[k] = r.x; by[k] = r.y; bm[k] = r.z;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            glox = fminf(glox, __shfl_xor_sync(FULL, glox, o));
            gloy = fminf(gloy, __shfl_xor_sync(FULL, gloy, o));
            ghix = fmaxf(ghix, __shfl_xor_sync(FULL, ghix, o));
            ghiy = fmaxf(ghiy, __shfl_xor_sync(FULL, ghiy, o));
        }
        // Far field: box centre, squared half-diagonal and its square root
        // (the expansion's length scale); off for a group of coincident bodies.
        const float gcx = __fmul_rn(0.5f, __fadd_rn(glox, ghix));
        const float gcy = __fmul_rn(0.5f, __fadd_rn(gloy, ghiy));
        const float ghx = __fsub_rn(ghix, glox), ghy = __fsub_rn(ghiy, gloy);
        const float rg2 = __fmul_rn(0.25f, __fadd_rn(__fmul_rn(ghx, ghx), __fmul_rn(ghy, ghy)));
        const bool far_on = FAR && PLUMMER && P.far_alpha2 > 0.0f && rg2 > 0.0f;
        const float lam = far_on ? __fsqrt_rn(rg2) : 1.0f;
        bool far_used = false;
        float cacc[kFarCoeffs];  // this lane's local-expansion sums
#pragma unroll
        for (int k = 0; k < kFarCoeffs; ++k) cacc[k] = 0.0f;
        // Accumulators: packed pairs (BPL >= 2) or scalars (BPL == 1).
        f2x X[NP > 0 ? NP : 1], Y[NP > 0 ? NP : 1], AX[NP > 0 ? NP : 1], AY[NP > 0 ? NP : 1];
        float ax1 = 0.f, ay1 = 0.f;
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            X[q] = pk(bx[2 * q], bx[2 * q + 1]);
            Y[q] = pk(by[2 * q], by[2 * q + 1]);
            AX[q] = pk(0.f, 0.f);
            AY[q] = pk(0.f, 0.f);
        }
        const f2x E2 = pk(eps2, eps2);
        const f2x M25 = pk(-2.5f, -2.5f);

        auto soft_pair = [&](int q, float m2) -> f2x {
            if (PLUMMER) return E2;
            return pk(ecoef * fmaxf(bm[2 * q], m2), ecoef * fmaxf(bm[2 * q + 1], m2));
        };

        // Node list: multipole interactions.
        auto eval_nodes = [&](int cnt) {
#pragma unroll 4  // four independent entries in flight per lane (measured best)
            for (int j = 0; j < cnt; ++j) {
                const float4 e0 = S.ent[j][0], e1 = S.ent[j][1];
                float4 e2 = make_float4(0.f, 0.f, 0.f, 0.f);
                if (MP >= 2) e2 = S.ent[j][2];
                if (NP > 0) {
                    const f2x CX = ld_pair(e0, 0), CY = ld_pair(e0, 1), M = ld_pair(e1, 0);
#pragma unroll
                    for (int q = 0; q < NP; ++q) {
                        if (2 * q >= kmax) break;
                        const f2x rx = sub2(CX, X[q]), ry = sub2(CY, Y[q]);
                        const f2x r2 = fma2(rx, rx, fma2(ry, ry, soft_pair(q, e1.x)));
                        const f2x inv = rsqrt2(r2);
                        const f2x inv2 = mul2(inv, inv);
                        const f2x inv3 = mul2(inv, inv2);
                        if (MP >= 2) {
                            const f2x NQXX = ld_pair(e1, 1), NQXY = ld_pair(e2, 0), NQYY = ld_pair(e2, 1);
                            const f2x nqrx = fma2(NQXX, rx, mul2(NQXY, ry));  // -(Q'r)_x
                            const f2x nqry = fma2(NQXY, rx, mul2(NQYY, ry));  // -(Q'r)_y
                            const f2x nrqr = fma2(rx, nqrx, mul2(ry, nqry)); // -r.Q'r
                            const f2x inv5 = mul2(inv3, inv2);
                            // f = m / |r|^3 + 5/2 r.Q'r / |r|^7
                            const f2x f = fma2(mul2(nrqr, M25), mul2(inv5, inv2), mul2(M, inv3));
                            AX[q] = fma2(nqrx, inv5, fma2(f, rx, AX[q]));
                            AY[q] = fma2(nqry, inv5, fma2(f, ry, AY[q]));
                        } else {
                            const f2x mi3 = mul2(M, inv3);
                            AX[q] = fma2(mi3, rx, AX[q]);
                            AY[q] = fma2(mi3, ry, AY[q]);
                        }
                    }
                } else {
                    const float rx = e0.x - bx[0], ry = e0.z - by[0];
                    const float es = PLUMMER ? eps2 : ecoef * fmaxf(bm[0], e1.x);
                    const float inv = rsqrt_ftz(fmaf(rx, rx, fmaf(ry, ry, es)));
                    const float inv2 = inv * inv, inv3 = inv * inv2;
                    const float mi3 = e1.x * inv3;
                    if (MP >= 2) {
                        const float nqrx = fmaf(e1.z, rx, e2.x * ry);
                        const float nqry = fmaf(e2.x, rx, e2.z * ry);
                        const float nrqr = fmaf(rx, nqrx, ry * nqry);
                        const float inv5 = inv3 * inv2;
                        const float f = fmaf(-2.5f * nrqr, inv5 * inv2, mi3);
                        ax1 = fmaf(nqrx, inv5, fmaf(f, rx, ax1));
                        ay1 = fmaf(nqry, inv5, fmaf(f, ry, ay1));
                    } else {
                        ax1 = fmaf(mi3, rx, ax1);
                        ay1 = fmaf(mi3, ry, ay1);
                    }
                }
            }
        };
        // Body list: point masses.  32 leaf records at a time are loaded by the
        // 32 lanes in parallel into shared memory, then every lane sums them.
        auto eval_bodies = [&](int cnt) {
            for (int c0 = 0; c0 < cnt; c0 += 32) {
                const int mcnt = (cnt - c0) < 32 ? (cnt - c0) : 32;
                __syncwarp();
                if (lane < mcnt) {
                    const float4 o = __ldg(&node4[nm1 + S.slot[c0 + lane]]);
                    S.body[lane][0] = make_float4(o.x, o.x, o.y, o.y);
                    S.body[lane][1] = make_float4(o.z, o.z, 0.f, 0.f);
                }
                __syncwarp();
                for (int j = 0; j < mcnt; ++j) {
                    const float4 p0 = S.body[j][0], p1 = S.body[j][1];
                    const uint32_t s = self_test ? S.slot[c0 + j] : 0u;
                    if (NP > 0) {
                        const f2x OX = ld_pair(p0, 0), OY = ld_pair(p0, 1), OM = ld_pair(p1, 0);
#pragma unroll
                        for (int q = 0; q < NP; ++q) {
                            if (2 * q >= kmax) break;
                            const f2x rx = sub2(OX, X[q]), ry = sub2(OY, Y[q]);
                            const f2x r2 = fma2(rx, rx, fma2(ry, ry, soft_pair(q, p1.x)));
                            const f2x inv = rsqrt2(r2);
                            f2x f = mul2(OM, mul2(inv, mul2(inv, inv)));
                            if (self_test) {
                                const uint32_t s0 = base + (uint32_t)(2 * q) * 32u + (uint32_t)lane;
                                float f0, f1;
                                upk(f, f0, f1);
                                f = pk(s == s0 ? 0.0f : f0, s == s0 + 32u ? 0.0f : f1);
                            }
                            AX[q] = fma2(f, rx, AX[q]);
                            AY[q] = fma2(f, ry, AY[q]);
                        }
                    } else {
                        const float rx = p0.x - bx[0], ry = p0.z - by[0];
                        const float es = PLUMMER ? eps2 : ecoef * fmaxf(bm[0], p1.x);
                        const float inv = rsqrt_ftz(fmaf(rx, rx, fmaf(ry, ry, es)));
                        float f = p1.x * (inv * inv * inv);
                        if (self_test) f = (s == base + (uint32_t)lane) ? 0.0f : f;
                        ax1 = fmaf(f, rx, ax1);
                        ay1 = fmaf(f, ry, ay1);
                    }
                }
            }
            __syncwarp();
        };
        int sp = 0, nn = 0, ns = 0, nf = 0;
        if (n > 1) {
            if (lane == 0) S.stack[0] = 0u;
            sp = 1;
        }
        __syncwarp();
        while (sp > 0) {
            int k = sp < 32 ? sp : 32;
            if (sp > kWalkDfsAt) k = 1;
            const bool has = lane < k;
            const uint32_t v = has ? S.stack[sp - k + lane] : 0u;
            sp -= k;
            __syncwarp();
            bool emit_node = false, emit_range = false, push = false;
            uint32_t r0 = 0, r1 = 0;
            float4 mom = make_float4(0.f, 0.f, 0.f, 0.f), sq = mom;
            if (has) {
                if (v >= nm1) {
                    emit_range = (v - nm1) >= sys_lo && (v - nm1) < sys_hi;
                    r0 = v - nm1;
                    r1 = 1;
                } else {
                    // the whole 64-B record in one round trip
                    const GNode* gp = &gnode[v];
                    const float4 box = __ldg(&gp->box);
                    const float4 m4 = __ldg(&gp->mom);
                    const float4 q4 = __ldg(&gp->quad);
                    const uint4 lk = __ldg(&gp->link);
                    const uint32_t f = lk.z, e = lk.z + lk.w;
                    if (e <= sys_lo || f >= sys_hi) {
                        // another system's subtree: no interaction
                    } else if (f < sys_lo || e > sys_hi) {
                        push = true;  // spans several systems: always open
                        r0 = lk.x;
                        r1 = lk.y;
                    } else if (group_accepts(box, m4.x, m4.y, glox, gloy, ghix, ghiy, th2)) {
                        emit_node = true;
                        mom = m4;
                        sq = q4;
                    } else if (lk.w <= (uint32_t)P.leaf_size) {
                        emit_range = true;
                        r0 = lk.z;
                        r1 = lk.w;
                    } else {
                        push = true;
                        r0 = lk.x;
                        r1 = lk.y;
                    }
                }
            }
            // Far field: an accepted node far from the group goes to the far list.
            bool emit_far = false;
            if (far_on && emit_node) {
                const float rx = __fsub_rn(mom.x, gcx), ry = __fsub_rn(mom.y, gcy);
                const float R2 = __fadd_rn(__fmul_rn(rx, rx), __fmul_rn(ry, ry));
                emit_far = rg2 < __fmul_rn(P.far_alpha2, R2);
                emit_node = !emit_far;
            }
            if (FAR && far_on) {
                const unsigned mf = __ballot_sync(FULL, emit_far);
                if (emit_far) {
                    const int q = GroupSmem<FAR>::kListCap - 1 - (nf + __popc(mf & lt));
                    const bool quad = MP >= 2;
                    S.ent[q][0] = make_float4(mom.x, mom.y, mom.z, quad ? sq.x : 0.f);
                    S.ent[q][1] = make_float4(quad ? sq.y : 0.f, quad ? sq.z : 0.f, 0.f, 0.f);
                }
                nf += __popc(mf);
            }
            const unsigned mn = __ballot_sync(FULL, emit_node);
            if (emit_node) {
                const int p = nn + __popc(mn & lt);
                S.ent[p][0] = make_float4(mom.x, mom.x, mom.y, mom.y);
                if (MP >= 2) {
                    // -Q' = tr(S) I - 3S
                    const float tr = sq.x + sq.z;
                    const float nxx = tr - 3.0f * sq.x, nxy = -3.0f * sq.y, nyy = tr - 3.0f * sq.z;
                    S.ent[p][1] = make_float4(mom.z, mom.z, nxx, nxx);
                    S.ent[p][2] = make_float4(nxy, nxy, nyy, nyy);
                } else {
                    S.ent[p][1] = make_float4(mom.z, mom.z, 0.f, 0.f);
                }
            }
            nn += __popc(mn);
            {
                // Append this step's body slots: exclusive scan of the counts.
                const uint32_t c = emit_range ? r1 : 0u;
                uint32_t incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t t = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += t;
                }
                const uint32_t total = __shfl_sync(FULL, incl, 31);
                const uint32_t at = (uint32_t)ns + incl - c;
                for (uint32_t u = 0; u < c; ++u) S.slot[at + u] = r0 + u;
                ns += (int)total;
            }
            const unsigned mp = __ballot_sync(FULL, push);
            const int npush = 2 * __popc(mp);
            if (sp + npush <= stack_cap) {
                if (push) {
                    const int p = sp + 2 * __popc(mp & lt);
                    S.stack[p] = r1;      // right child
                    S.stack[p + 1] = r0;  // left child on top
                }
                sp += npush;
            } else if (lane == 0) {
                atomicOr(err, kErrGroupStack);
            }
            if (counting) c_vis += (unsigned long long)k;
            __syncwarp();
            // Lists are evaluated when full, and whatever they hold once the
            // stack is empty; one call site each keeps the kernel's code
            // (and its instruction-cache footprint) small.
            const bool last = sp == 0;
            if (nn >= 32 || (last && nn > 0)) {
                eval_nodes(nn);
                if (counting) c_node += (unsigned long long)nn * nvalid;
                nn = 0;
                __syncwarp();
            }
            if (ns >= 32 || (last && ns > 0)) {
                if (counting) c_body += (unsigned long long)ns * nvalid;
                eval_bodies(ns);
                ns = 0;
            }
            if constexpr (FAR) {
                while (nf >= 32 || (last && nf > 0)) {
                    const int cnt = nf < 32 ? nf : 32;
                    far_batch(S, cacc, lane, nf, cnt, gcx, gcy, lam, eps2);
                    if (counting) c_far += (unsigned long long)cnt;
                    nf -= cnt;
                    far_used = true;
                }
            }
        }
        if (counting && n > 1) c_body -= nvalid;  // each body met its own leaf once
        __syncwarp();
        // Far field: reduce the lane columns (every lane gets the sums) and
        // evaluate the local expansion at each of the lane's bodies.
        float fx[BPL], fy[BPL];
#pragma unroll
        for (int k = 0; k < BPL; ++k) {
            fx[k] = 0.0f;
            fy[k] = 0.0f;
        }
        if (far_used) {
            float c[kFarCoeffs];
#pragma unroll
            for (int k = 0; k < kFarCoeffs; ++k) {
                float v = cacc[k];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
                c[k] = v;
            }
            const float inv_lam = __fdiv_rn(1.0f, lam);
#pragma unroll
            for (int k = 0; k < BPL; ++k) {
                if ((uint32_t)k * 32u + (uint32_t)lane >= nvalid) continue;
                const float dx = __fmul_rn(__fsub_rn(bx[k], gcx), inv_lam);
                const float dy = __fmul_rn(__fsub_rn(by[k], gcy), inv_lam);
                float ex, ey;
                far_eval(c, dx, dy, ex, ey);
                fx[k] = -__fmul_rn(ex, inv_lam);
                fy[k] = -__fmul_rn(ey, inv_lam);
            }
        }
        __syncwarp();

        // Integrate (same modes as the exact walk).
        float ax[BPL], ay[BPL];
        if (NP > 0) {
#pragma unroll
            for (int q = 0; q < NP; ++q) {
                upk(AX[q], ax[2 * q], ax[2 * q + 1]);
                upk(AY[q], ay[2 * q], ay[2 * q + 1]);
            }
        } else {
            ax[0] = ax1;
            ay[0] = ay1;
        }
#pragma unroll
        for (int k = 0; k < BPL; ++k) {
            const uint32_t s = base + (uint32_t)k * 32u + (uint32_t)lane;
            if ((uint32_t)k * 32u + (uint32_t)lane >= nvalid) continue;
            const float axk = far_used ? __fadd_rn(ax[k], fx[k]) : ax[k];
            const float ayk = far_used ? __fadd_rn(ay[k], fy[k]) : ay[k];
            const float gx = P.g * axk, gy = P.g * ayk;
            const uint32_t b = __ldg(&ids[s]);
            if (P.mode == kWalkForces) {
                acc[b] = make_float2(gx, gy);
            } else if (P.mode == kWalkEulerKickDrift) {
                float2 vv = vel[b];
                vv.x = __fadd_rn(vv.x, __fmul_rn(gx, P.dt));
                vv.y = __fadd_rn(vv.y, __fmul_rn(gy, P.dt));
                vel[b] = vv;
                pos[b] = make_float2(__fadd_rn(bx[k], __fmul_rn(vv.x, P.dt)),
                                     __fadd_rn(by[k], __fmul_rn(vv.y, P.dt)));
            } else {
                const float hdt = 0.5f * P.dt;
                float2 vv = vel[b];
                vv.x = __fadd_rn(vv.x, __fmul_rn(gx, hdt));
                vv.y = __fadd_rn(vv.y, __fmul_rn(gy, hdt));
                vel[b] = vv;
                acc[b] = make_float2(gx, gy);
            }
        }
    }
    if (counting && lane == 0) {
        atomicAdd(&P.counters[0], c_vis);
        atomicAdd(&P.counters[1], c_node);
        atomicAdd(&P.counters[2], c_body);
        atomicAdd(&P.counters[3], c_far);
    }
}

// Warps per block the group walk may run with (walk_block / 32).
constexpr int kWalkShapes[3] = {2, 4, 8};
constexpr int kWalkDefaultWarps = 4;

static int shape_index(int warps) { return warps == 2 ? 0 : (warps == 8 ? 2 : 1); }

template <int BPL, int MP, bool PL, bool FAR>
static cudaError_t set_walk_attributes() {
    const int smem = (int)(walk_max_threads(BPL) / 32 * sizeof(GroupSmem<FAR>));
    cudaError_t e = cudaFuncSetAttribute(walk_group_kernel<BPL, MP, PL, FAR, false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(walk_group_kernel<BPL, MP, PL, FAR, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

// Largest walk block for bodies_per_lane `bpl` (its launch bound).
int walk_group_max_block(int bpl) { return walk_max_threads(bpl >= 4 ? 4 : 2); }

template <int BPL, int MP, bool PL, bool FAR, bool COUNT>
static void launch_c(const DeviceBuffers& b, const WalkParams& p, int warps, cudaStream_t s) {
    static int blocks_per_sm[64][3] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t smem = (size_t)warps * sizeof(GroupSmem<FAR>);
    int& bps = blocks_per_sm[dev & 63][shape_index(warps)];
    if (bps == 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &bps, walk_group_kernel<BPL, MP, PL, FAR, COUNT>, warps * 32, smem);
        if (bps < 1) bps = 1;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // Persistent grid; the number of groups (<= n) is only known on the device.
    uint32_t blocks = (uint32_t)(sms * bps);
    const uint32_t need = (b.n + warps - 1) / warps;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    walk_group_kernel<BPL, MP, PL, FAR, COUNT><<<blocks, warps * 32, smem, s>>>(
        b.gnode, b.node4, b.groups, b.ids, b.pos, b.vel, b.acc, p, b.err);
}

// The counting walk only when bh_walk_stats asks for it (p.count).
template <int BPL, int MP, bool PL, bool FAR = false>
static void launch_t(const DeviceBuffers& b, const WalkParams& p, int warps, cudaStream_t s) {
    if (p.count) launch_c<BPL, MP, PL, FAR, true>(b, p, warps, s);
    else launch_c<BPL, MP, PL, FAR, false>(b, p, warps, s);
}

template <int BPL>
static void launch_bpl(const DeviceBuffers& b, const WalkParams& p, int warps, cudaStream_t s) {
    if (p.multipole >= 2) {
        if (p.plummer && p.far_alpha2 > 0.0f) launch_t<BPL, 2, true, true>(b, p, warps, s);
        else if (p.plummer) launch_t<BPL, 2, true>(b, p, warps, s);
        else launch_t<BPL, 2, false>(b, p, warps, s);
    } else {
        if (p.plummer) launch_t<BPL, 1, true>(b, p, warps, s);
        else launch_t<BPL, 1, false>(b, p, warps, s);
    }
}

template <int BPL>
static cudaError_t set_bpl_attributes() {
    cudaError_t e;
    if ((e = set_walk_attributes<BPL, 2, true, true>()) != cudaSuccess) return e;
    if ((e = set_walk_attributes<BPL, 2, true, false>()) != cudaSuccess) return e;
    if ((e = set_walk_attributes<BPL, 2, false, false>()) != cudaSuccess) return e;
    if ((e = set_walk_attributes<BPL, 1, true, false>()) != cudaSuccess) return e;
    return set_walk_attributes<BPL, 1, false, false>();
}

// Allow every walk variant the dynamic shared memory of its largest block
// shape on the current device (once per device, before any launch or
// capture).
cudaError_t walk_init_attributes() {
    cudaError_t e;
    if ((e = set_bpl_attributes<1>()) != cudaSuccess) return e;
    if ((e = set_bpl_attributes<2>()) != cudaSuccess) return e;
    return set_bpl_attributes<4>();
}

void launch_walk_group(const DeviceBuffers& b, const WalkParams& p, int block, cudaStream_t s) {
    if (b.n == 0) return;
    int warps = block / 32;
    if (warps != 2 && warps != 4 && warps != 8) warps = kWalkDefaultWarps;
    if (warps * 32 > walk_group_max_block(p.bpl)) warps = walk_group_max_block(p.bpl) / 32;
    switch (p.bpl) {
        case 1: launch_bpl<1>(b, p, warps, s); break;
        case 4: launch_bpl<4>(b, p, warps, s); break;
        default: launch_bpl<2>(b, p, warps, s); break;
    }
}

}  // namespace bh
