// adjoint.cu -- vector-Jacobian product of the group-walk force and the
// reverse sweep of a kick-drift-kick rollout (extension, no reference
// counterpart).
//
// Force of one interaction (r = c - x, q = r.r + eps^2, s = q^-1/2, G
// applied by the caller):
//     a = m r s^3 - Q'r s^5 + 5/2 (r.Q'r) r s^7          (Q' = 3S - tr(S) I)
// For an upstream adjoint abar (ab) the VJP is
//     mbar  = (ab.r) s^3
//     Q'bar = d(ab.a)/d(q'xx, q'xy, q'yy)
//           = (-ab_x r_x s^5 + 5/2 r_x^2 (ab.r) s^7,
//              -(ab_x r_y + ab_y r_x) s^5 + 5 r_x r_y (ab.r) s^7,
//              -ab_y r_y s^5 + 5/2 r_y^2 (ab.r) s^7)
//     rbar  = m (s^3 ab - 3 s^5 (ab.r) r)
//           - s^5 Q'ab + 5 s^7 (ab.Q'r) r
//           + 5 s^7 (ab.r) Q'r + 5/2 s^7 (r.Q'r) ab - 35/2 s^9 (r.Q'r)(ab.r) r
// and since r = c - x:  xbar -= rbar,  cbar += rbar.  A body-body
// interaction is the monopole case with the source body's position and mass.
//
// Node adjoints go to bodies through the node moments M = sum m_j,
// c = sum m_j x_j / M, S = sum m_j d_j d_j^T (d_j = x_j - c, so dS/dc = 0):
//     xbar_j += m_j cbar_n / M_n + 2 m_j G_n d_jn
//     mbar_j += mbar_n + cbar_n.d_jn / M_n + d_jn^T G_n d_jn
// with G_n the symmetric matrix of dL/dS_n (Sxx, Sxy, Syy from
// Q'xx = 2Sxx - Syy, Q'xy = 3Sxy, Q'yy = 2Syy - Sxx).  Summed over the
// ancestors n of body j these are polynomials in x_j whose coefficients are
// ten path sums; vjp_push_kernel climbs each leaf's ancestors to form them.
#include "bh_internal.cuh"
#include "packed.cuh"

namespace bh {

constexpr int kVjpWarps = 4;
constexpr int kVjpStack = 384;
constexpr int kVjpDfsAt = kVjpStack - 128;
constexpr int kVjpSlots = 32 + 32 * kGroupMaxLeaf;

struct VjpSmem {
    uint32_t stack[kVjpStack];
    // node entry j, every value duplicated so a 64-bit shared load gives an
    // operand pair: {cx, cx, cy, cy}, {m, m, Q'xx, Q'xx}, {Q'xy, Q'xy, Q'yy, Q'yy}
    float4 nd[kGroupList][3];
    uint32_t nd_idx[kGroupList];  // the entry's internal node
    uint32_t slot[kVjpSlots];
    float4 body[32];           // staged leaf records {x, y, m, slot bits}
};

// Warp sums of 8 values by recursive halving: 4 + 2 + 1 exchanges split the
// values between lane halves, 2 more finish the sum.  Afterwards lanes 4k..4k+3
// hold the sum of v[k] (9 shuffles instead of 8 x 5).
__device__ __forceinline__ float warp_reduce_scatter8(float v[8]) {
    const unsigned FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const bool h4 = lane & 16, h3 = lane & 8, h2 = lane & 4;
    float a[4], b[2];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float keep = h4 ? v[j + 4] : v[j], send = h4 ? v[j] : v[j + 4];
        a[j] = keep + __shfl_xor_sync(FULL, send, 16);
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const float keep = h3 ? a[j + 2] : a[j], send = h3 ? a[j] : a[j + 2];
        b[j] = keep + __shfl_xor_sync(FULL, send, 8);
    }
    float c;
    {
        const float keep = h2 ? b[1] : b[0], send = h2 ? b[0] : b[1];
        c = keep + __shfl_xor_sync(FULL, send, 4);
    }
    c += __shfl_xor_sync(FULL, c, 2);
    c += __shfl_xor_sync(FULL, c, 1);
    return c;
}

// Same for 4 values: lanes 8k..8k+7 hold the sum of v[k] (6 shuffles).
__device__ __forceinline__ float warp_reduce_scatter4(float v[4]) {
    const unsigned FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const bool h4 = lane & 16, h3 = lane & 8;
    float a[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const float keep = h4 ? v[j + 2] : v[j], send = h4 ? v[j] : v[j + 2];
        a[j] = keep + __shfl_xor_sync(FULL, send, 16);
    }
    float c;
    {
        const float keep = h3 ? a[1] : a[0], send = h3 ? a[0] : a[1];
        c = keep + __shfl_xor_sync(FULL, send, 8);
    }
    c += __shfl_xor_sync(FULL, c, 4);
    c += __shfl_xor_sync(FULL, c, 2);
    c += __shfl_xor_sync(FULL, c, 1);
    return c;
}

// node_adj: 6 floats per internal node {cbar.x, cbar.y, mbar, Q'bar xx, xy, yy}
template <int BPL, int MP>
__global__ void __launch_bounds__(kVjpWarps * 32)
vjp_group_kernel(const GNode* __restrict__ gnode, const float4* __restrict__ node4,
                 const uint2* __restrict__ groups, const uint32_t* __restrict__ ids,
                 const float2* __restrict__ abar, float* __restrict__ node_adj,
                 float2* __restrict__ xbar_slot, float* __restrict__ mbar_slot,
                 const WalkParams P, uint32_t* __restrict__ err) {
    __shared__ VjpSmem smem[kVjpWarps];
    if (step_failed(err)) return;  // the tree at these positions was not built
    const int lane = threadIdx.x & 31;
    VjpSmem& S = smem[threadIdx.x >> 5];
    const unsigned FULL = 0xFFFFFFFFu;
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t n = P.n, nm1 = n - 1;
    const uint32_t ngroups = P.group_ctr[1];
    const float th2 = __fmul_rn(P.theta, P.theta);
    const float eps2 = P.eps2, G = P.g;

    while (true) {
        uint32_t g = 0;
        if (lane == 0) g = atomicAdd(P.group_ctr, 1u);
        g = __shfl_sync(FULL, g, 0);
        if (g >= ngroups) break;
        const uint2 grp = __ldg(&groups[g]);
        const uint32_t base = grp.x, nvalid = grp.y;
        float bx[BPL], by[BPL], abx[BPL], aby[BPL], xbx[BPL], xby[BPL];
        bool ok[BPL];
        float glox = INFINITY, gloy = INFINITY, ghix = -INFINITY, ghiy = -INFINITY;
#pragma unroll
        for (int k = 0; k < BPL; ++k) {
            const uint32_t rel = (uint32_t)k * 32u + (uint32_t)lane;
            ok[k] = rel < nvalid;
            float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
            float2 a = make_float2(0.f, 0.f);
            if (ok[k]) {
                r = __ldg(&node4[nm1 + base + rel]);
                a = __ldg(&abar[__ldg(&ids[base + rel])]);
                glox = fminf(glox, r.x); gloy = fminf(gloy, r.y);
                ghix = fmaxf(ghix, r.x); ghiy = fmaxf(ghiy, r.y);
            }
            bx[k] = r.x; by[k] = r.y;
            abx[k] = G * a.x; aby[k] = G * a.y;  // the force carries G
            xbx[k] = 0.f; xby[k] = 0.f;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            glox = fminf(glox, __shfl_xor_sync(FULL, glox, o));
            gloy = fminf(gloy, __shfl_xor_sync(FULL, gloy, o));
            ghix = fmaxf(ghix, __shfl_xor_sync(FULL, ghix, o));
            ghiy = fmaxf(ghiy, __shfl_xor_sync(FULL, ghiy, o));
        }

        // Packed pairs of the lane's bodies (BPL >= 2): positions, adjoints
        // and the node-list part of their position adjoints.
        constexpr int NP = BPL / 2;
        f2x PX[NP > 0 ? NP : 1], PY[NP > 0 ? NP : 1], PAX[NP > 0 ? NP : 1], PAY[NP > 0 ? NP : 1];
        f2x PXB[NP > 0 ? NP : 1], PYB[NP > 0 ? NP : 1];
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            PX[q] = pk(bx[2 * q], bx[2 * q + 1]);
            PY[q] = pk(by[2 * q], by[2 * q + 1]);
            PAX[q] = pk(abx[2 * q], abx[2 * q + 1]);
            PAY[q] = pk(aby[2 * q], aby[2 * q + 1]);
            PXB[q] = pk(0.f, 0.f);
            PYB[q] = pk(0.f, 0.f);
        }
        const int kmax = (int)((nvalid + 31u) / 32u);  // sub-slots in use (uniform)

        auto eval_nodes = [&](int cnt) {
#pragma unroll 2
            for (int j = 0; j < cnt; ++j) {
                const float4 e0 = S.nd[j][0], e1 = S.nd[j][1], e2 = S.nd[j][2];
                const uint32_t v = S.nd_idx[j];
                float cbx = 0.f, cby = 0.f, mb = 0.f, gxx = 0.f, gxy = 0.f, gyy = 0.f;
                if (NP > 0) {
                    // Two bodies per instruction.  A slot past the group's end
                    // holds a zero adjoint, so it adds exactly zero everywhere.
                    const f2x CX = ld_pair(e0, 0), CY = ld_pair(e0, 1), M = ld_pair(e1, 0);
                    const f2x QXX = ld_pair(e1, 1), QXY = ld_pair(e2, 0), QYY = ld_pair(e2, 1);
                    const f2x E2 = pk(eps2, eps2), CM3 = pk(-3.0f, -3.0f), CM1 = pk(-1.0f, -1.0f);
                    const f2x C5 = pk(5.0f, 5.0f), C25 = pk(2.5f, 2.5f), CM175 = pk(-17.5f, -17.5f);
                    f2x CB_X = pk(0.f, 0.f), CB_Y = CB_X, MB = CB_X, GXX = CB_X, GXY = CB_X, GYY = CB_X;
#pragma unroll
                    for (int q = 0; q < NP; ++q) {
                        if (2 * q >= kmax) break;
                        const f2x rx = sub2(CX, PX[q]), ry = sub2(CY, PY[q]);
                        const f2x sv = rsqrt2(fma2(rx, rx, fma2(ry, ry, E2)));
                        const f2x s2 = mul2(sv, sv), s3 = mul2(sv, s2), s5 = mul2(s3, s2);
                        const f2x ar = fma2(PAX[q], rx, mul2(PAY[q], ry));
                        const f2x tn = mul2(mul2(s5, ar), CM3);  // -3 s^5 (ab.r)
                        f2x rbx = mul2(M, fma2(s3, PAX[q], mul2(tn, rx)));
                        f2x rby = mul2(M, fma2(s3, PAY[q], mul2(tn, ry)));
                        MB = fma2(ar, s3, MB);
                        if (MP >= 2) {
                            const f2x s7 = mul2(s5, s2), s9 = mul2(s7, s2), s5n = mul2(s5, CM1);
                            const f2x qrx = fma2(QXX, rx, mul2(QXY, ry));
                            const f2x qry = fma2(QXY, rx, mul2(QYY, ry));
                            const f2x qax = fma2(QXX, PAX[q], mul2(QXY, PAY[q]));
                            const f2x qay = fma2(QXY, PAX[q], mul2(QYY, PAY[q]));
                            const f2x rqr = fma2(rx, qrx, mul2(ry, qry));
                            const f2x aqr = fma2(PAX[q], qrx, mul2(PAY[q], qry));
                            const f2x f7 = mul2(C5, s7), h7 = mul2(C25, s7);
                            const f2x c1 = fma2(f7, aqr, mul2(mul2(CM175, s9), mul2(rqr, ar)));
                            const f2x f7ar = mul2(f7, ar), h7ar = mul2(h7, ar), h7rqr = mul2(h7, rqr);
                            rbx = fma2(s5n, qax, rbx);
                            rbx = fma2(c1, rx, rbx);
                            rbx = fma2(f7ar, qrx, rbx);
                            rbx = fma2(h7rqr, PAX[q], rbx);
                            rby = fma2(s5n, qay, rby);
                            rby = fma2(c1, ry, rby);
                            rby = fma2(f7ar, qry, rby);
                            rby = fma2(h7rqr, PAY[q], rby);
                            GXX = fma2(mul2(PAX[q], rx), s5n, fma2(mul2(rx, rx), h7ar, GXX));
                            GXY = fma2(fma2(PAX[q], ry, mul2(PAY[q], rx)), s5n,
                                       fma2(mul2(rx, ry), f7ar, GXY));
                            GYY = fma2(mul2(PAY[q], ry), s5n, fma2(mul2(ry, ry), h7ar, GYY));
                        }
                        PXB[q] = sub2(PXB[q], rbx);
                        PYB[q] = sub2(PYB[q], rby);
                        CB_X = add2(CB_X, rbx);
                        CB_Y = add2(CB_Y, rby);
                    }
                    cbx = sum_halves(CB_X);
                    cby = sum_halves(CB_Y);
                    mb = sum_halves(MB);
                    if (MP >= 2) {
                        gxx = sum_halves(GXX);
                        gxy = sum_halves(GXY);
                        gyy = sum_halves(GYY);
                    }
                } else {
                    const float cxn = e0.x, cyn = e0.z, mn = e1.x;
                    const float qxx = e1.z, qxy = e2.x, qyy = e2.z;
#pragma unroll
                    for (int k = 0; k < BPL; ++k) {
                        if (!ok[k]) continue;
                        const float rx = cxn - bx[k], ry = cyn - by[k];
                        const float s = rsqrt_ftz(fmaf(rx, rx, fmaf(ry, ry, eps2)));
                        const float s2 = s * s, s3 = s * s2, s5 = s3 * s2;
                        const float ar = abx[k] * rx + aby[k] * ry;
                        float rbx = mn * (s3 * abx[k] - 3.0f * s5 * ar * rx);
                        float rby = mn * (s3 * aby[k] - 3.0f * s5 * ar * ry);
                        mb += ar * s3;
                        if (MP >= 2) {
                            const float s7 = s5 * s2, s9 = s7 * s2;
                            const float qrx = qxx * rx + qxy * ry, qry = qxy * rx + qyy * ry;
                            const float qax = qxx * abx[k] + qxy * aby[k], qay = qxy * abx[k] + qyy * aby[k];
                            const float rqr = rx * qrx + ry * qry;
                            const float aqr = abx[k] * qrx + aby[k] * qry;
                            const float c1 = 5.0f * s7 * aqr - 17.5f * s9 * rqr * ar;
                            rbx += -s5 * qax + c1 * rx + 5.0f * s7 * ar * qrx + 2.5f * s7 * rqr * abx[k];
                            rby += -s5 * qay + c1 * ry + 5.0f * s7 * ar * qry + 2.5f * s7 * rqr * aby[k];
                            gxx += -abx[k] * rx * s5 + 2.5f * rx * rx * ar * s7;
                            gxy += -(abx[k] * ry + aby[k] * rx) * s5 + 5.0f * rx * ry * ar * s7;
                            gyy += -aby[k] * ry * s5 + 2.5f * ry * ry * ar * s7;
                        }
                        xbx[k] -= rbx;
                        xby[k] -= rby;
                        cbx += rbx;
                        cby += rby;
                    }
                }
                if (MP >= 2) {
                    float vals[8] = {cbx, cby, mb, gxx, gxy, gyy, 0.f, 0.f};
                    const float tot = warp_reduce_scatter8(vals);
                    const int q = lane >> 2;  // lanes 4q hold the sum of vals[q]
                    if ((lane & 3) == 0 && q < 6) atomicAdd(node_adj + 6 * (size_t)v + q, tot);
                } else {
                    float vals[4] = {cbx, cby, mb, 0.f};
                    const float tot = warp_reduce_scatter4(vals);
                    const int q = lane >> 3;  // lanes 8q hold the sum of vals[q]
                    if ((lane & 7) == 0 && q < 3) atomicAdd(node_adj + 6 * (size_t)v + q, tot);
                }
            }
        };
        auto eval_bodies = [&](int cnt) {
            for (int j = 0; j < cnt; ++j) {
                if ((j & 31) == 0) {  // stage the next 32 leaf records in parallel
                    __syncwarp();
                    if (j + lane < cnt) {
                        const uint32_t sl = S.slot[j + lane];
                        float4 r = __ldg(&node4[nm1 + sl]);
                        r.w = __uint_as_float(sl);
                        S.body[lane] = r;
                    }
                    __syncwarp();
                }
                const float4 o = S.body[j & 31];
                const uint32_t sj = __float_as_uint(o.w);
                float cbx = 0.f, cby = 0.f, mb = 0.f;
#pragma unroll
                for (int k = 0; k < BPL; ++k) {
                    if (!ok[k] || sj == base + (uint32_t)k * 32u + (uint32_t)lane) continue;
                    const float rx = o.x - bx[k], ry = o.y - by[k];
                    const float s = rsqrt_ftz(fmaf(rx, rx, fmaf(ry, ry, eps2)));
                    const float s3 = s * s * s, s5 = s3 * s * s;
                    const float ar = abx[k] * rx + aby[k] * ry;
                    const float rbx = o.z * (s3 * abx[k] - 3.0f * s5 * ar * rx);
                    const float rby = o.z * (s3 * aby[k] - 3.0f * s5 * ar * ry);
                    xbx[k] -= rbx;
                    xby[k] -= rby;
                    cbx += rbx;
                    cby += rby;
                    mb += ar * s3;
                }
                {
                    float vals[4] = {cbx, cby, mb, 0.f};
                    const float tot = warp_reduce_scatter4(vals);
                    const int q = lane >> 3;  // lanes 8q hold the sum of vals[q]
                    if ((lane & 7) == 0 && q < 3)
                        atomicAdd(q == 2 ? &mbar_slot[sj] : (q == 0 ? &xbar_slot[sj].x : &xbar_slot[sj].y), tot);
                }
            }
        };

        // Same traversal as walk_group_kernel: identical interaction lists.
        int sp = 0, nn = 0, ns = 0;
        if (n > 1) {
            if (lane == 0) S.stack[0] = 0u;
            sp = 1;
        }
        __syncwarp();
        while (sp > 0) {
            int k = sp < 32 ? sp : 32;
            if (sp > kVjpDfsAt) k = 1;
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
                    const uint4 lk = __ldg(&gnode[v].link);
                    mom = __ldg(&gnode[v].mom);
                    if (MP >= 2) sq = __ldg(&gnode[v].quad);
                    if (group_accepts(box, mom.x, mom.y, glox, gloy, ghix, ghiy, th2)) {
                        emit_node = true;
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
            const unsigned mn = __ballot_sync(FULL, emit_node);
            if (emit_node) {
                const int p = nn + __popc(mn & lt);
                const float tr = sq.x + sq.z;  // Q' = 3S - tr(S) I
                const float qxx = 3.0f * sq.x - tr, qxy = 3.0f * sq.y, qyy = 3.0f * sq.z - tr;
                S.nd[p][0] = make_float4(mom.x, mom.x, mom.y, mom.y);
                S.nd[p][1] = make_float4(mom.z, mom.z, qxx, qxx);
                S.nd[p][2] = make_float4(qxy, qxy, qyy, qyy);
                S.nd_idx[p] = v;
            }
            nn += __popc(mn);
            {
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
            if (sp + npush <= kVjpStack) {
                if (push) {
                    const int p = sp + 2 * __popc(mp & lt);
                    S.stack[p] = r1;
                    S.stack[p + 1] = r0;
                }
                sp += npush;
            } else if (lane == 0) {
                atomicOr(err, kErrGroupStack);
            }
            __syncwarp();
            if (nn >= 32) {
                eval_nodes(nn);
                nn = 0;
                __syncwarp();
            }
            if (ns >= 32) {
                eval_bodies(ns);
                ns = 0;
                __syncwarp();
            }
        }
        if (nn > 0) eval_nodes(nn);
        if (ns > 0) eval_bodies(ns);
        __syncwarp();
#pragma unroll
        for (int q = 0; q < NP; ++q) {  // node-list part of the packed bodies
            float lo, hi;
            upk(PXB[q], lo, hi);
            xbx[2 * q] += lo;
            xbx[2 * q + 1] += hi;
            upk(PYB[q], lo, hi);
            xby[2 * q] += lo;
            xby[2 * q + 1] += hi;
        }
#pragma unroll
        for (int k = 0; k < BPL; ++k) {
            if (!ok[k]) continue;
            const uint32_t s = base + (uint32_t)k * 32u + (uint32_t)lane;
            atomicAdd(&xbar_slot[s].x, xbx[k]);
            atomicAdd(&xbar_slot[s].y, xby[k]);
        }
    }
}

// Push node adjoints down to bodies and add the per-slot adjoints; writes
// xbar/mbar in original body order (accumulating: +=).
__global__ void __launch_bounds__(256)
vjp_push_kernel(const GNode* __restrict__ gnode, const float4* __restrict__ node4,
                const uint32_t* __restrict__ parent, const uint32_t* __restrict__ ids,
                const float* __restrict__ node_adj, const float2* __restrict__ xbar_slot,
                const float* __restrict__ mbar_slot, float2* __restrict__ xbar,
                float* __restrict__ mbar, uint32_t n, int mp) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t nm1 = n - 1;
    // path sums over the ancestors
    double sm = 0, ux = 0, uy = 0, w = 0, gxx = 0, gxy = 0, gyy = 0, gcx = 0, gcy = 0, cgc = 0;
    uint32_t v = (n > 1) ? __ldg(&parent[nm1 + j]) : kSentinel;
    uint32_t guard = 0;
    while (v != kSentinel && v < nm1 && guard++ < 4096u) {
        const float4 mom = __ldg(&gnode[v].mom);
        const float* na = node_adj + 6 * (size_t)v;
        const double cx = mom.x, cy = mom.y, M = mom.z;
        sm += na[2];
        if (M > 0.0) {
            ux += na[0] / M;
            uy += na[1] / M;
            w += (na[0] * cx + na[1] * cy) / M;
        }
        if (mp >= 2) {
            // dL/dS from dL/dQ': Q'xx = 2Sxx - Syy, Q'xy = 3Sxy, Q'yy = 2Syy - Sxx
            const double sxx = 2.0 * na[3] - na[5], sxy = 3.0 * na[4], syy = 2.0 * na[5] - na[3];
            // G = [[sxx, sxy/2], [sxy/2, syy]]
            const double hxy = 0.5 * sxy;
            gxx += sxx;
            gxy += hxy;
            gyy += syy;
            const double tx = sxx * cx + hxy * cy, ty = hxy * cx + syy * cy;
            gcx += tx;
            gcy += ty;
            cgc += cx * tx + cy * ty;
        }
        v = __ldg(&parent[v]);
    }
    const float4 me = __ldg(&node4[nm1 + j]);
    const double x = me.x, y = me.y, m = me.z;
    const double gx = gxx * x + gxy * y - gcx, gy = gxy * x + gyy * y - gcy;  // G x - G c
    const double xb_x = m * ux + 2.0 * m * gx;
    const double xb_y = m * uy + 2.0 * m * gy;
    const double mb = sm + (x * ux + y * uy - w) + (x * (gxx * x + gxy * y) + y * (gxy * x + gyy * y)) -
                      2.0 * (x * gcx + y * gcy) + cgc;
    const uint32_t b = __ldg(&ids[j]);
    const float2 xs = xbar_slot[j];
    float2 acc = xbar[b];
    acc.x += (float)(xb_x + xs.x);
    acc.y += (float)(xb_y + xs.y);
    xbar[b] = acc;
    mbar[b] += (float)(mb + mbar_slot[j]);
}

// ---- elementwise steps of the reverse sweep (original body order) ---------
__global__ void adj_init_kernel(const float2* __restrict__ pos, const float2* __restrict__ target,
                                uint32_t n, float2* __restrict__ xbar, float2* __restrict__ vbar,
                                float* __restrict__ mbar, float2* __restrict__ apend,
                                double* __restrict__ loss) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double part = 0.0;
    if (i < n) {
        const float dx = pos[i].x - target[i].x, dy = pos[i].y - target[i].y;
        const float sc = 2.0f / (float)n;
        xbar[i] = make_float2(sc * dx, sc * dy);
        vbar[i] = make_float2(0.f, 0.f);
        mbar[i] = 0.f;
        apend[i] = make_float2(0.f, 0.f);
        part = ((double)dx * dx + (double)dy * dy) / (double)n;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xFFFFFFFFu, part, o);
    if ((threadIdx.x & 31) == 0 && part != 0.0) atomicAdd(loss, part);
}

// abar = apend + h vbar   (closing kick of the step that ends at this point)
__global__ void adj_pre_kernel(const float2* __restrict__ apend, const float2* __restrict__ vbar,
                               float h, uint32_t n, float2* __restrict__ abar) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    abar[i] = make_float2(apend[i].x + h * vbar[i].x, apend[i].y + h * vbar[i].y);
}

// drift and opening kick: vbar += dt xbar; apend = h vbar
__global__ void adj_post_kernel(const float2* __restrict__ xbar, float2* __restrict__ vbar,
                                float2* __restrict__ apend, float dt, float h, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float2 v = vbar[i];
    v.x += dt * xbar[i].x;
    v.y += dt * xbar[i].y;
    vbar[i] = v;
    apend[i] = make_float2(h * v.x, h * v.y);
}

// ---- launchers -----------------------------------------------------------------
template <int BPL, int MP>
static void vjp_launch_t(const DeviceBuffers& b, const WalkParams& p, const float2* abar,
                         float* node_adj, float2* xbar_slot, float* mbar_slot, cudaStream_t s) {
    static int bps_cache[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    int& bps = bps_cache[dev & 63];
    if (bps == 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, vjp_group_kernel<BPL, MP>,
                                                      kVjpWarps * 32, 0);
        if (bps < 1) bps = 1;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint32_t blocks = (uint32_t)(sms * bps);
    const uint32_t need = (b.n + kVjpWarps - 1) / kVjpWarps;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    vjp_group_kernel<BPL, MP><<<blocks, kVjpWarps * 32, 0, s>>>(
        b.gnode, b.node4, b.groups, b.ids, abar, node_adj, xbar_slot, mbar_slot, p, b.err);
}

void launch_force_vjp(const DeviceBuffers& b, const WalkParams& p, const float2* abar,
                      float* node_adj, float2* xbar_slot, float* mbar_slot, float2* xbar,
                      float* mbar, cudaStream_t s) {
    if (b.n == 0) return;
    if (b.n > 1) cudaMemsetAsync(node_adj, 0, sizeof(float) * 6 * (size_t)(b.n - 1), s);
    cudaMemsetAsync(xbar_slot, 0, sizeof(float2) * (size_t)b.n, s);
    cudaMemsetAsync(mbar_slot, 0, sizeof(float) * (size_t)b.n, s);
    const bool quad = p.multipole >= 2;
    switch (p.bpl) {
        case 1:
            if (quad) vjp_launch_t<1, 2>(b, p, abar, node_adj, xbar_slot, mbar_slot, s);
            else vjp_launch_t<1, 1>(b, p, abar, node_adj, xbar_slot, mbar_slot, s);
            break;
        case 4:
            if (quad) vjp_launch_t<4, 2>(b, p, abar, node_adj, xbar_slot, mbar_slot, s);
            else vjp_launch_t<4, 1>(b, p, abar, node_adj, xbar_slot, mbar_slot, s);
            break;
        default:
            if (quad) vjp_launch_t<2, 2>(b, p, abar, node_adj, xbar_slot, mbar_slot, s);
            else vjp_launch_t<2, 1>(b, p, abar, node_adj, xbar_slot, mbar_slot, s);
            break;
    }
    const int blocks = (int)((b.n + 255) / 256);
    vjp_push_kernel<<<blocks, 256, 0, s>>>(b.gnode, b.node4, b.parent, b.ids, node_adj, xbar_slot,
                                          mbar_slot, xbar, mbar, b.n, p.multipole);
}

void launch_adj_init(const float2* pos, const float2* target, uint32_t n, float2* xbar,
                     float2* vbar, float* mbar, float2* apend, double* loss, cudaStream_t s) {
    cudaMemsetAsync(loss, 0, sizeof(double), s);
    adj_init_kernel<<<(n + 255) / 256, 256, 0, s>>>(pos, target, n, xbar, vbar, mbar, apend, loss);
}

void launch_adj_pre(const float2* apend, const float2* vbar, float h, uint32_t n, float2* abar,
                    cudaStream_t s) {
    adj_pre_kernel<<<(n + 255) / 256, 256, 0, s>>>(apend, vbar, h, n, abar);
}

void launch_adj_post(const float2* xbar, float2* vbar, float2* apend, float dt, float h, uint32_t n,
                     cudaStream_t s) {
    adj_post_kernel<<<(n + 255) / 256, 256, 0, s>>>(xbar, vbar, apend, dt, h, n);
}

}  // namespace bh
