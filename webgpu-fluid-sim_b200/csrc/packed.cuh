// packed.cuh -- packed FP32 pairs for sm_100: one add/sub/mul/fma.rn.f32x2
// instruction on two floats held in one 64-bit register pair.  The group walk
// and its VJP evaluate two bodies per instruction with these.
#pragma once

#include "bh_internal.cuh"

namespace bh {

typedef unsigned long long f2x;
__device__ __forceinline__ f2x pk(float lo, float hi) {
    f2x r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void upk(f2x v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2x sub2(f2x a, f2x b) {
    f2x r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2x mul2(f2x a, f2x b) {
    f2x r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2x fma2(f2x a, f2x b, f2x c) {
    f2x r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
__device__ __forceinline__ f2x rsqrt2(f2x v) {
    float lo, hi;
    upk(v, lo, hi);
    return pk(rsqrt_ftz(lo), rsqrt_ftz(hi));
}
__device__ __forceinline__ f2x ld_pair(const float4& v, int half) {
    // {v.x, v.y} or {v.z, v.w} of a shared-memory float4 as one 64-bit pair
    return reinterpret_cast<const f2x*>(&v)[half];
}

__device__ __forceinline__ f2x add2(f2x a, f2x b) {
    f2x r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ float sum_halves(f2x v) {
    float lo, hi;
    upk(v, lo, hi);
    return lo + hi;
}

}  // namespace bh
