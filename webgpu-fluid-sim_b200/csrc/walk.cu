// walk.cu -- theta-criterion tree walk with the integrator fused in.
//
// Reference: bh_vel_step_main (barnes_hut.wgsl:48-111) + bh_pos_step_main
// (barnes_hut.wgsl:113-120).  Per body the reference pops nodes from a private
// 256-entry stack (right child on top, so right subtrees go first), skips its
// own leaf, softens with eps = epsMult*sqrt(G*max(m1,m2)*dt), and accepts a
// node when it is a leaf or length/sqrt(d^2+eps^2) < theta; otherwise it
// pushes left then right (dropped if the stack is full).
//
// Warp-cooperative form: the 32 lanes of a warp hold 32 consecutive sorted
// slots (spatially coherent after the Morton sort) and share one stack in
// shared memory whose entries carry the set of lanes that still need the
// node.  A popped node is fetched once for the warp; each lane applies its own
// criterion, and the node's children are pushed with the mask of the lanes
// that opened it.  Each lane therefore visits exactly the nodes its own
// per-body walk would, in the same right-first depth-first order, so its
// interaction list and summation order equal the reference's.
//
// Own-body data comes from the sorted leaf records (node4[n-1+slot]), which
// the fill wrote from pos/mass at the start of the step, so the drift can
// write pos[] in the same kernel without racing other warps' reads.
//
// Extension: leaf buckets.  With leaf_size L > 1 an opened node of <= L bodies
// is summed directly over its contiguous sorted slots instead of being
// descended (more accurate than the monopoles it would otherwise accept).
#include "bh_internal.cuh"

namespace bh {

template <int MODE, bool PLUMMER, bool BUCKETS>
__global__ void __launch_bounds__(256)
walk_kernel(const float4* __restrict__ node4, const uint2* __restrict__ children,
            const uint2* __restrict__ range, const uint32_t* __restrict__ ids,
            float2* __restrict__ pos, float2* __restrict__ vel, float2* __restrict__ acc,
            const WalkParams P, uint32_t* __restrict__ err) {
    constexpr int kWarps = 256 / 32;
    __shared__ uint2 s_stack[kWarps][kStackSize];
    if (step_failed(err)) return;  // the tree of this step was not built
    const int stack_cap = (P.stack_cap > 0 && P.stack_cap < kStackSize) ? P.stack_cap : kStackSize;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t n = P.n, nm1 = n - 1;
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = slot < n;
    const unsigned act = __ballot_sync(0xFFFFFFFFu, active);
    if (act == 0u) return;
    const uint32_t my_leaf = nm1 + slot;
    const float4 me = active ? __ldg(&node4[my_leaf]) : make_float4(0.f, 0.f, 0.f, 0.f);
    float ax = 0.0f, ay = 0.0f;
    const bool counting = MODE == kWalkForces && P.count;
    uint32_t n_vis = 0, n_node = 0, n_body = 0;  // instrumented launch only
    uint2* stk = s_stack[w];
    if (lane == 0) stk[0] = make_uint2(0u, act);
    int sp = 1;
    __syncwarp();
    while (sp > 0) {
        --sp;
        const uint2 e = stk[sp];
        const uint32_t node = e.x;
        const bool in = (e.y >> lane) & 1u;
        const float4 nd = __ldg(&node4[node]);
        const bool leaf = node >= nm1;
        const float rx = nd.x - me.x, ry = nd.y - me.y;
        const float d2 = rx * rx + ry * ry;
        const float e2 = PLUMMER ? P.eps2 : P.eps_coef * fmaxf(me.z, nd.z);
        const float inv = rsqrtf(d2 + e2);
        const bool far = leaf || (nd.w * inv < P.theta);
        if (counting) {
            n_vis += in;
            n_node += in && far && !leaf;
            n_body += in && leaf && node != my_leaf;
        }
        if (in && far && node != my_leaf) {
            const float f = P.g * nd.z * (inv * inv * inv);
            ax = fmaf(f, rx, ax);
            ay = fmaf(f, ry, ay);
        }
        const unsigned open = __ballot_sync(0xFFFFFFFFu, in && !far);
        if (open) {
            if (BUCKETS) {
                const uint2 rg = __ldg(&range[node]);
                if (rg.y - rg.x < (uint32_t)P.leaf_size) {
                    const bool mine = (open >> lane) & 1u;
                    for (uint32_t s = rg.x; s <= rg.y; ++s) {
                        const float4 bj = __ldg(&node4[nm1 + s]);
                        const float qx = bj.x - me.x, qy = bj.y - me.y;
                        const float q2 = qx * qx + qy * qy;
                        const float f2 = PLUMMER ? P.eps2 : P.eps_coef * fmaxf(me.z, bj.z);
                        const float iv = rsqrtf(q2 + f2);
                        if (counting) n_body += mine && s != slot;
                        if (mine && s != slot) {
                            const float f = P.g * bj.z * (iv * iv * iv);
                            ax = fmaf(f, qx, ax);
                            ay = fmaf(f, qy, ay);
                        }
                    }
                    continue;
                }
            }
            if (sp < stack_cap - 1) {  // barnes_hut.wgsl:100: stack_ptr + 2 < stack_size
                const uint2 ch = __ldg(&children[node]);
                if (lane == 0) {
                    stk[sp] = make_uint2(ch.x, open);
                    stk[sp + 1] = make_uint2(ch.y, open);
                }
                sp += 2;
            } else if (lane == 0) {
                atomicOr(err, kErrStackOverflow);
            }
        }
        __syncwarp();
    }
    if (counting) {
        unsigned long long v = n_vis, nd = n_node, bd = n_body;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
            nd += __shfl_xor_sync(0xFFFFFFFFu, nd, o);
            bd += __shfl_xor_sync(0xFFFFFFFFu, bd, o);
        }
        if (lane == 0) {
            atomicAdd(&P.counters[0], v);
            atomicAdd(&P.counters[1], nd);
            atomicAdd(&P.counters[2], bd);
        }
    }
    if (!active) return;
    const uint32_t b = __ldg(&ids[slot]);
    if (MODE == kWalkForces) {
        acc[b] = make_float2(ax, ay);
    } else if (MODE == kWalkEulerKickDrift) {
        // barnes_hut.wgsl:110 then :120
        float2 v = vel[b];
        v.x = __fadd_rn(v.x, __fmul_rn(ax, P.dt));
        v.y = __fadd_rn(v.y, __fmul_rn(ay, P.dt));
        vel[b] = v;
        pos[b] = make_float2(__fadd_rn(me.x, __fmul_rn(v.x, P.dt)),
                             __fadd_rn(me.y, __fmul_rn(v.y, P.dt)));
    } else {
        const float hdt = 0.5f * P.dt;
        float2 v = vel[b];
        v.x = __fadd_rn(v.x, __fmul_rn(ax, hdt));
        v.y = __fadd_rn(v.y, __fmul_rn(ay, hdt));
        vel[b] = v;
        acc[b] = make_float2(ax, ay);
    }
}

template <int MODE>
static void launch_mode(const DeviceBuffers& b, const WalkParams& p, int blocks, cudaStream_t s) {
    const bool buckets = p.leaf_size > 1;
#define BH_WALK(PL, BK)                                                                        \
    walk_kernel<MODE, PL, BK><<<blocks, 256, 0, s>>>(b.node4, b.children, b.range, b.ids, b.pos, \
                                                      b.vel, b.acc, p, b.err)
    if (p.plummer) {
        if (buckets) BH_WALK(true, true); else BH_WALK(true, false);
    } else {
        if (buckets) BH_WALK(false, true); else BH_WALK(false, false);
    }
#undef BH_WALK
}

void launch_walk(const DeviceBuffers& b, const WalkParams& p, int block, cudaStream_t s) {
    (void)block;
    if (b.n == 0) return;
    const int blocks = (int)((b.n + 255) / 256);
    switch (p.mode) {
        case kWalkForces: launch_mode<kWalkForces>(b, p, blocks, s); break;
        case kWalkEulerKickDrift: launch_mode<kWalkEulerKickDrift>(b, p, blocks, s); break;
        default: launch_mode<kWalkKdkClose>(b, p, blocks, s); break;
    }
}

}  // namespace bh
