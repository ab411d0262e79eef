// far_field.cuh -- local (Taylor) expansions of far multipoles for the group
// walk (extension; no reference counterpart).
//
// The group walk evaluates every accepted node at each of the group's bodies
// (a multipole-to-body interaction per body).  A node that is far from the
// group compared with the group's size -- group half-diagonal r_g < alpha R,
// R = |c - x_g| from the group's centre x_g to the node's COM c -- is instead
// turned once into the coefficients of a local expansion of its potential
// about x_g, summed over all such nodes, and the sum is evaluated at each body
// (Cartesian "multipole-to-local" + "local-to-body").
//
// Potential of a node (mass M, second moments S about its COM; G applied by
// the caller), with the Plummer-softened kernel g(R) = (|R|^2 + eps^2)^-1/2:
//     Phi(x) = -[ M g(R) + 1/2 (Sxx g_xx + 2 Sxy g_xy + Syy g_yy) ],  R = x - c.
// Derivatives of g (Faa di Bruno for g = h(|R|^2), h(u) = (u + eps^2)^-1/2):
//     d^(a,b) g = s^(a+b+1) P_ab(rho),  s = (|R|^2 + eps^2)^-1/2,  rho = s R,
//     P_ab = sum_{i<=a/2, j<=b/2} c(a,i) c(b,j) rho_x^(a-2i) rho_y^(b-2j) w(a+b-i-j),
//     c(a,i) = a! / (i! (a-2i)! 2^i),  w(m) = (-1)^m (2m-1)!!.
// With the length scale lambda = r_g and t = lambda s (< alpha for a far node)
// the scaled coefficients of orders 1..4 (kFarCoeffs of them) are
//     C_ab = lambda^(a+b) d^(a,b) Phi(x_g)
//          = -s t^(a+b) [ M P_ab + 1/2 (S'xx P_(a+2)b + 2 S'xy P_(a+1)(b+1) + S'yy P_a(b+2)) ],
//     S' = s^2 S,
// all bounded by M s (no overflow for close, dense groups).  At a body
// x = x_g + lambda d (|d| <= 1) the force of all far nodes is the gradient of
// the local expansion truncated at order 4 (cubic in d):
//     a_x = -(1/lambda) sum_{a+b<=3} C_(a+1)b d_x^a d_y^b / (a! b!),
//     a_y = -(1/lambda) sum_{a+b<=3} C_a(b+1) d_x^a d_y^b / (a! b!).
// The truncation error of a node's force is about (r_g / R)^4 of it; with
// alpha = 0.25 a prototype on the 100k colliding disks moved the median
// force error against the FP64 direct sum from 3.8e-4 to 4.2e-4 while 64% of
// the accepted nodes took this path.
#pragma once

#include "bh_internal.cuh"

namespace bh {

constexpr int kFarCoeffs = 14;  // potential coefficients of orders 1..4

// Coefficient index of (a, b), 1 <= a + b <= 4: by order, then by b.
__host__ __device__ constexpr int far_idx(int a, int b) {
    return (a + b - 1) * (a + b + 2) / 2 + b;
}
__host__ __device__ constexpr float far_c(int a, int i) {
    // a! / (i! (a - 2i)! 2^i)
    float num = 1.f;
    for (int k = 2; k <= a; ++k) num *= (float)k;
    float den = 1.f;
    for (int k = 2; k <= i; ++k) den *= (float)k;
    for (int k = 2; k <= a - 2 * i; ++k) den *= (float)k;
    for (int k = 0; k < i; ++k) den *= 2.f;
    return num / den;
}
__host__ __device__ constexpr float far_w(int m) {
    // (-1)^m (2m - 1)!!
    float v = 1.f;
    for (int k = 1; k <= m; ++k) v *= -(float)(2 * k - 1);
    return v;
}

// P_ab(rho) from the powers ex[k] = rho_x^k, ey[k] = rho_y^k (k <= 6).
template <int A, int B>
__device__ __forceinline__ float far_poly(const float (&ex)[7], const float (&ey)[7]) {
    float acc = 0.f;
#pragma unroll
    for (int i = 0; 2 * i <= A; ++i)
#pragma unroll
        for (int j = 0; 2 * j <= B; ++j)
            acc = __fmaf_rn(far_c(A, i) * far_c(B, j) * far_w(A + B - i - j),
                            __fmul_rn(ex[A - 2 * i], ey[B - 2 * j]), acc);
    return acc;
}

// One coefficient C_ab of one node, added to acc[far_idx(a, b)].
template <int A, int B>
__device__ __forceinline__ void far_term(float* acc, const float (&ex)[7], const float (&ey)[7],
                                         float m, float sxx, float sxy, float syy,
                                         const float (&st)[5]) {
    const float quad = __fmaf_rn(sxx, far_poly<A + 2, B>(ex, ey),
                        __fmaf_rn(2.f * sxy, far_poly<A + 1, B + 1>(ex, ey),
                                  __fmul_rn(syy, far_poly<A, B + 2>(ex, ey))));
    const float v = __fmaf_rn(m, far_poly<A, B>(ex, ey), __fmul_rn(0.5f, quad));
    acc[far_idx(A, B)] = __fmaf_rn(-st[A + B], v, acc[far_idx(A, B)]);
}

// Add one node's scaled local coefficients (about x_g, length scale lambda)
// to acc[kFarCoeffs].  R = x_g - c.
__device__ __forceinline__ void far_node_coeffs(float (&acc)[kFarCoeffs], float rx, float ry, float m, float sxx,
                                                float sxy, float syy, float lambda, float eps2) {
    const float u = __fadd_rn(__fadd_rn(__fmul_rn(rx, rx), __fmul_rn(ry, ry)), eps2);
    const float s = __frsqrt_rn(u);
    const float s2 = __fmul_rn(s, s);
    float ex[7], ey[7];
    ex[0] = 1.f;
    ey[0] = 1.f;
    ex[1] = __fmul_rn(rx, s);
    ey[1] = __fmul_rn(ry, s);
#pragma unroll
    for (int k = 2; k < 7; ++k) {
        ex[k] = __fmul_rn(ex[k - 1], ex[1]);
        ey[k] = __fmul_rn(ey[k - 1], ey[1]);
    }
    const float t = __fmul_rn(lambda, s);
    float st[5];
    st[0] = s;
#pragma unroll
    for (int k = 1; k < 5; ++k) st[k] = __fmul_rn(st[k - 1], t);
    const float qxx = __fmul_rn(s2, sxx), qxy = __fmul_rn(s2, sxy), qyy = __fmul_rn(s2, syy);
    far_term<1, 0>(acc, ex, ey, m, qxx, qxy, qyy, st);
    far_term<0, 1>(acc, ex, ey, m, qxx, qxy, qyy, st);
    far_term<2, 0>(acc, ex, ey, m, qxx, qxy, qyy, st);
    far_term<1, 1>(acc, ex, ey, m, qxx, qxy, qyy, st);
    far_term<0, 2>(acc, ex, ey, m, qxx, qxy, qyy, st);
    far_term<3, 0>(acc, ex, ey, m, qxx, qxy, qyy, st);
    far_term<2, 1>(acc, ex, ey, m, qxx, qxy, qyy, st);
    far_term<1, 2>(acc, ex, ey, m, qxx, qxy, qyy, st);
    far_term<0, 3>(acc, ex, ey, m, qxx, qxy, qyy, st);
    far_term<4, 0>(acc, ex, ey, m, qxx, qxy, qyy, st);
    far_term<3, 1>(acc, ex, ey, m, qxx, qxy, qyy, st);
    far_term<2, 2>(acc, ex, ey, m, qxx, qxy, qyy, st);
    far_term<1, 3>(acc, ex, ey, m, qxx, qxy, qyy, st);
    far_term<0, 4>(acc, ex, ey, m, qxx, qxy, qyy, st);
}

// Force of the local expansion at offset d = (x - x_g) / lambda:
// (ax, ay) without the factor -1/lambda (the caller applies it).
__device__ __forceinline__ void far_eval(const float* C, float dx, float dy, float& ax, float& ay) {
    const float dxx = __fmul_rn(dx, dx), dxy = __fmul_rn(dx, dy), dyy = __fmul_rn(dy, dy);
    // sum_{a+b<=3} C_(a+1)b d^(a,b) / (a! b!) and C_a(b+1) likewise
    float x = C[far_idx(1, 0)];
    x = __fmaf_rn(C[far_idx(2, 0)], dx, x);
    x = __fmaf_rn(C[far_idx(1, 1)], dy, x);
    x = __fmaf_rn(0.5f * C[far_idx(3, 0)], dxx, x);
    x = __fmaf_rn(C[far_idx(2, 1)], dxy, x);
    x = __fmaf_rn(0.5f * C[far_idx(1, 2)], dyy, x);
    x = __fmaf_rn((1.f / 6.f) * C[far_idx(4, 0)], __fmul_rn(dxx, dx), x);
    x = __fmaf_rn(0.5f * C[far_idx(3, 1)], __fmul_rn(dxx, dy), x);
    x = __fmaf_rn(0.5f * C[far_idx(2, 2)], __fmul_rn(dx, dyy), x);
    x = __fmaf_rn((1.f / 6.f) * C[far_idx(1, 3)], __fmul_rn(dyy, dy), x);
    float y = C[far_idx(0, 1)];
    y = __fmaf_rn(C[far_idx(1, 1)], dx, y);
    y = __fmaf_rn(C[far_idx(0, 2)], dy, y);
    y = __fmaf_rn(0.5f * C[far_idx(2, 1)], dxx, y);
    y = __fmaf_rn(C[far_idx(1, 2)], dxy, y);
    y = __fmaf_rn(0.5f * C[far_idx(0, 3)], dyy, y);
    y = __fmaf_rn((1.f / 6.f) * C[far_idx(3, 1)], __fmul_rn(dxx, dx), y);
    y = __fmaf_rn(0.5f * C[far_idx(2, 2)], __fmul_rn(dxx, dy), y);
    y = __fmaf_rn(0.5f * C[far_idx(1, 3)], __fmul_rn(dx, dyy), y);
    y = __fmaf_rn((1.f / 6.f) * C[far_idx(0, 4)], __fmul_rn(dyy, dy), y);
    ax = x;
    ay = y;
}

}  // namespace bh
