// walk_group.cu -- group tree walk with quadrupole moments (extension).
//
// No reference counterpart as a whole: it replaces bh_vel_step_main
// (barnes_hut.wgsl:48-111) + bh_pos_step_main (:113-120) when the
// configuration asks for the group walk.  The reference's per-body monopole
// walk has a median relative force error of order 1e-2 at theta = 0.5 in 2D;
// this walk reaches <= 1e-3 at the same theta.
//
// One warp owns a group: a maximal subtree of at most 32 x BPL bodies, i.e.
// contiguous sorted slots inside one Morton cell (listed by the build
// kernel).  Fixed runs of 32 x BPL slots would not do: a run that straddles a
// jump of the Z curve has a box spanning far-apart regions and opens nearly
// every node.  The group opens a node unless
//     L^2 < theta^2 d^2,  L = longest side of the node's box,
//     d = distance between the group's box and the node's box,
// which is stricter for every body of the group than the per-body test
// length / |com - x| < theta.  Accepted nodes act through their monopole and
// (multipole order 2) quadrupole about the COM,
//     a = G [ M r/|r|^3 - Q'r/|r|^5 + 5/2 (r.Q'r) r/|r|^7 ],  Q' = 3S - tr(S) I,
// with r = com - x and |r|^2 = r.r + eps^2 (S = second moments about the COM).
// Leaves, and opened nodes of <= leaf_size bodies, are summed body by body.
//
// Traversal: a per-warp stack in shared memory.  Every step each lane takes
// one of the top 32 stack entries, evaluates its node, and the warp compacts
// the outcomes with ballots into a node list, a body-range list and the
// stack.  Lists are evaluated when they hold >= 32 entries: every lane runs
// every entry for its BPL bodies (shared-memory broadcasts, no divergence).
// Above kGroupDfsAt entries the warp pops one node per step (plain DFS), which
// keeps the stack below kGroupStack for any tree of depth <= 96; a push that
// would not fit raises kErrGroupStack instead of writing out of bounds.
// Groups are taken from an atomic counter (the walk is persistent).
#include "bh_internal.cuh"

namespace bh {

constexpr int kGroupWarps = 4;

struct GroupSmem {
    uint32_t stack[kGroupStack];
    float4 mom[kGroupList];   // {com.x, com.y, mass, 0}
    float4 quad[kGroupList];  // {Q'xx, Q'xy, Q'yy, 0}
    uint2 range[kGroupList];  // {first slot, count}
};

template <int BPL, int MP, bool PLUMMER>
__global__ void __launch_bounds__(kGroupWarps * 32)
walk_group_kernel(const GNode* __restrict__ gnode, const float4* __restrict__ node4,
                  const uint2* __restrict__ groups, const uint32_t* __restrict__ ids,
                  float2* __restrict__ pos, float2* __restrict__ vel, float2* __restrict__ acc,
                  const WalkParams P, uint32_t* __restrict__ err) {
    __shared__ GroupSmem smem[kGroupWarps];
    const int lane = threadIdx.x & 31;
    GroupSmem& S = smem[threadIdx.x >> 5];
    const unsigned FULL = 0xFFFFFFFFu;
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t n = P.n, nm1 = n - 1;
    const uint32_t ngroups = P.group_ctr[1];  // written by the build kernel
    const float th2 = __fmul_rn(P.theta, P.theta);
    const float eps2 = P.eps2, ecoef = P.eps_coef;
    const bool counting = P.count != 0;
    unsigned long long c_vis = 0, c_node = 0, c_body = 0;

    while (true) {
        uint32_t g = 0;
        if (lane == 0) g = atomicAdd(P.group_ctr, 1u);
        g = __shfl_sync(FULL, g, 0);
        if (g >= ngroups) break;
        // A group is a subtree of <= 32 x BPL bodies: contiguous sorted slots
        // inside one Morton cell, so its box stays compact.
        const uint2 grp = __ldg(&groups[g]);
        const uint32_t base = grp.x, nvalid = grp.y;
        const int kmax = (int)((nvalid + 31u) / 32u);  // sub-slots in use (uniform)
        float bx[BPL], by[BPL], bm[BPL], ax[BPL], ay[BPL];
        float glox = INFINITY, gloy = INFINITY, ghix = -INFINITY, ghiy = -INFINITY;
#pragma unroll
        for (int k = 0; k < BPL; ++k) {
            const uint32_t s = base + (uint32_t)k * 32u + (uint32_t)lane;
            float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
            if ((uint32_t)k * 32u + (uint32_t)lane < nvalid) {
                r = __ldg(&node4[nm1 + s]);
                glox = fminf(glox, r.x); gloy = fminf(gloy, r.y);
                ghix = fmaxf(ghix, r.x); ghiy = fmaxf(ghiy, r.y);
            }
            bx[k] = r.x; by[k] = r.y; bm[k] = r.z;
            ax[k] = 0.f; ay[k] = 0.f;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            glox = fminf(glox, __shfl_xor_sync(FULL, glox, o));
            gloy = fminf(gloy, __shfl_xor_sync(FULL, gloy, o));
            ghix = fmaxf(ghix, __shfl_xor_sync(FULL, ghix, o));
            ghiy = fmaxf(ghiy, __shfl_xor_sync(FULL, ghiy, o));
        }

        // Evaluate the node list (multipoles) for this lane's bodies.
        auto eval_nodes = [&](int cnt) {
#pragma unroll 2
            for (int j = 0; j < cnt; ++j) {
                const float4 a = S.mom[j];
                float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
                if (MP >= 2) q = S.quad[j];
#pragma unroll
                for (int k = 0; k < BPL; ++k) {
                    if (k >= kmax) break;
                    const float rx = a.x - bx[k], ry = a.y - by[k];
                    const float e2 = PLUMMER ? eps2 : ecoef * fmaxf(bm[k], a.z);
                    const float r2 = fmaf(rx, rx, fmaf(ry, ry, e2));
                    const float inv = rsqrtf(r2);
                    const float inv2 = inv * inv;
                    const float inv3 = inv * inv2;
                    if (MP >= 2) {
                        const float qrx = fmaf(q.x, rx, q.y * ry);
                        const float qry = fmaf(q.y, rx, q.z * ry);
                        const float rqr = fmaf(rx, qrx, ry * qry);
                        const float inv5 = inv3 * inv2;
                        const float f = fmaf(2.5f * rqr, inv5 * inv2, a.z * inv3);
                        ax[k] = fmaf(-qrx, inv5, fmaf(f, rx, ax[k]));
                        ay[k] = fmaf(-qry, inv5, fmaf(f, ry, ay[k]));
                    } else {
                        const float f = a.z * inv3;
                        ax[k] = fmaf(f, rx, ax[k]);
                        ay[k] = fmaf(f, ry, ay[k]);
                    }
                }
            }
        };
        // Evaluate the body-range list (point masses, own slot skipped).
        auto eval_ranges = [&](int cnt) {
            for (int j = 0; j < cnt; ++j) {
                const uint2 rg = S.range[j];
                for (uint32_t s = rg.x; s < rg.x + rg.y; ++s) {
                    const float4 o = __ldg(&node4[nm1 + s]);
#pragma unroll
                    for (int k = 0; k < BPL; ++k) {
                        if (k >= kmax) break;
                        const float rx = o.x - bx[k], ry = o.y - by[k];
                        const float e2 = PLUMMER ? eps2 : ecoef * fmaxf(bm[k], o.z);
                        const float r2 = fmaf(rx, rx, fmaf(ry, ry, e2));
                        const float inv = rsqrtf(r2);
                        float f = o.z * (inv * inv * inv);
                        f = (s == base + (uint32_t)k * 32u + (uint32_t)lane) ? 0.0f : f;
                        ax[k] = fmaf(f, rx, ax[k]);
                        ay[k] = fmaf(f, ry, ay[k]);
                    }
                }
            }
        };

        int sp = 0, nn = 0, nr = 0;
        if (n > 1) {
            if (lane == 0) S.stack[0] = 0u;
            sp = 1;
        }
        __syncwarp();
        while (sp > 0) {
            int k = sp < 32 ? sp : 32;
            if (sp > kGroupDfsAt) k = 1;
            const bool has = lane < k;
            const uint32_t v = has ? S.stack[sp - k + lane] : 0u;
            sp -= k;
            __syncwarp();
            bool emit_node = false, emit_range = false, push = false;
            uint32_t r0 = 0, r1 = 0;
            float4 mom = make_float4(0.f, 0.f, 0.f, 0.f), sq = mom;
            if (has) {
                if (v >= nm1) {
                    emit_range = true;
                    r0 = v - nm1;
                    r1 = 1;
                } else {
                    const float4 box = __ldg(&gnode[v].box);
                    const float dx = fmaxf(0.0f, fmaxf(__fsub_rn(box.x, ghix), __fsub_rn(glox, box.z)));
                    const float dy = fmaxf(0.0f, fmaxf(__fsub_rn(box.y, ghiy), __fsub_rn(gloy, box.w)));
                    const float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
                    const float L = fmaxf(__fsub_rn(box.z, box.x), __fsub_rn(box.w, box.y));
                    if (__fmul_rn(L, L) < __fmul_rn(th2, d2)) {
                        emit_node = true;
                        mom = __ldg(&gnode[v].mom);
                        if (MP >= 2) sq = __ldg(&gnode[v].quad);
                    } else {
                        const uint4 lk = __ldg(&gnode[v].link);
                        if (lk.w <= (uint32_t)P.leaf_size) {
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
            }
            const unsigned mn = __ballot_sync(FULL, emit_node);
            if (emit_node) {
                const int p = nn + __popc(mn & lt);
                S.mom[p] = make_float4(mom.x, mom.y, mom.z, 0.0f);
                if (MP >= 2) {
                    const float tr = sq.x + sq.z;
                    S.quad[p] = make_float4(3.0f * sq.x - tr, 3.0f * sq.y, 3.0f * sq.z - tr, 0.0f);
                }
            }
            nn += __popc(mn);
            const unsigned mr = __ballot_sync(FULL, emit_range);
            if (emit_range) S.range[nr + __popc(mr & lt)] = make_uint2(r0, r1);
            nr += __popc(mr);
            const unsigned mp = __ballot_sync(FULL, push);
            const int npush = 2 * __popc(mp);
            if (sp + npush <= kGroupStack) {
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
            if (nn >= 32) {
                eval_nodes(nn);
                if (counting) c_node += (unsigned long long)nn * nvalid;
                nn = 0;
                __syncwarp();
            }
            if (nr >= 32) {
                if (counting)
                    for (int j = 0; j < nr; ++j) c_body += (unsigned long long)S.range[j].y * nvalid;
                eval_ranges(nr);
                nr = 0;
                __syncwarp();
            }
        }
        if (nn > 0) {
            eval_nodes(nn);
            if (counting) c_node += (unsigned long long)nn * nvalid;
        }
        if (nr > 0) {
            if (counting)
                for (int j = 0; j < nr; ++j) c_body += (unsigned long long)S.range[j].y * nvalid;
            eval_ranges(nr);
        }
        if (counting && n > 1) c_body -= nvalid;  // each body met its own leaf once
        __syncwarp();

        // Integrate (same modes as the exact walk).
#pragma unroll
        for (int k = 0; k < BPL; ++k) {
            const uint32_t s = base + (uint32_t)k * 32u + (uint32_t)lane;
            if ((uint32_t)k * 32u + (uint32_t)lane >= nvalid) continue;
            const float gx = P.g * ax[k], gy = P.g * ay[k];
            const uint32_t b = __ldg(&ids[s]);
            if (P.mode == kWalkForces) {
                acc[b] = make_float2(gx, gy);
            } else if (P.mode == kWalkEulerKickDrift) {
                float2 v = vel[b];
                v.x = __fadd_rn(v.x, __fmul_rn(gx, P.dt));
                v.y = __fadd_rn(v.y, __fmul_rn(gy, P.dt));
                vel[b] = v;
                pos[b] = make_float2(__fadd_rn(bx[k], __fmul_rn(v.x, P.dt)),
                                     __fadd_rn(by[k], __fmul_rn(v.y, P.dt)));
            } else {
                const float hdt = 0.5f * P.dt;
                float2 v = vel[b];
                v.x = __fadd_rn(v.x, __fmul_rn(gx, hdt));
                v.y = __fadd_rn(v.y, __fmul_rn(gy, hdt));
                vel[b] = v;
                acc[b] = make_float2(gx, gy);
            }
        }
    }
    if (counting && lane == 0) {
        atomicAdd(&P.counters[0], c_vis);
        atomicAdd(&P.counters[1], c_node);
        atomicAdd(&P.counters[2], c_body);
    }
}

template <int BPL, int MP, bool PL>
static void launch_t(const DeviceBuffers& b, const WalkParams& p, cudaStream_t s) {
    static int blocks_per_sm[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    int& bps = blocks_per_sm[dev & 63];
    if (bps == 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, walk_group_kernel<BPL, MP, PL>,
                                                      kGroupWarps * 32, 0);
        if (bps < 1) bps = 1;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // Persistent grid; the number of groups (<= n) is only known on the device.
    uint32_t blocks = (uint32_t)(sms * bps);
    const uint32_t need = (b.n + kGroupWarps - 1) / kGroupWarps;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    walk_group_kernel<BPL, MP, PL><<<blocks, kGroupWarps * 32, 0, s>>>(
        b.gnode, b.node4, b.groups, b.ids, b.pos, b.vel, b.acc, p, b.err);
}

template <int BPL>
static void launch_bpl(const DeviceBuffers& b, const WalkParams& p, cudaStream_t s) {
    if (p.multipole >= 2) {
        if (p.plummer) launch_t<BPL, 2, true>(b, p, s); else launch_t<BPL, 2, false>(b, p, s);
    } else {
        if (p.plummer) launch_t<BPL, 1, true>(b, p, s); else launch_t<BPL, 1, false>(b, p, s);
    }
}

void launch_walk_group(const DeviceBuffers& b, const WalkParams& p, int block, cudaStream_t s) {
    (void)block;
    if (b.n == 0) return;
    switch (p.bpl) {
        case 1: launch_bpl<1>(b, p, s); break;
        case 4: launch_bpl<4>(b, p, s); break;
        default: launch_bpl<2>(b, p, s); break;
    }
}

}  // namespace bh
