// Packed single-precision pairs for sm_100: the f32x2 forms of add, mul and
// fma issue two IEEE binary32 operations as one instruction, each rounded to
// nearest with subnormals flushed (the library is built with
// --use_fast_math, whose scalar float operations flush the same way), so a
// pair computes exactly what two scalar operations would, in half the issue
// slots.  Used by the rasterizers, whose pixels are evaluated in pairs.
#pragma once

namespace lig {

struct f2 {
    unsigned long long v;
};

__device__ __forceinline__ f2 f2_pack(float lo, float hi) {
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ f2 f2_dup(float x) { return f2_pack(x, x); }
__device__ __forceinline__ f2 f2_zero() { return f2{0ull}; }
__device__ __forceinline__ void f2_unpack(f2 a, float &lo, float &hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
}
__device__ __forceinline__ float f2_sum(f2 a) {
    float lo, hi;
    f2_unpack(a, lo, hi);
    return lo + hi;
}
__device__ __forceinline__ f2 f2_add(f2 a, f2 b) {
    f2 d;
    asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b) {
    f2 d;
    asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c) {
    f2 d;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(d.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return d;
}

}  // namespace lig
