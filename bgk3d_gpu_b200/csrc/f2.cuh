// Two FP32 values advanced together by the packed arithmetic of sm_100
// (FADD2 / FFMA2: one instruction for both lanes, each lane rounded exactly
// like the scalar operation), so that a collision written once for a value
// type V runs on two nodes at the cost of one.
//
// A packed multiply followed by a packed add can be contracted into one fused
// multiply-add by the code generator even when both carry an explicit
// rounding mode (observed on B200 with CUDA 12.9: about a fifth of a*a + b*b
// results one unit off), which would break the bit-exact parity with the
// reference's operation order.  So a product is formed as fma(a, b, z) with
// z = -0 read from constant memory: the compiler cannot know the addend,
// a*b + (-0) rounds exactly like a*b, and the result is an ordinary rounded
// value that a following addition cannot absorb.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace bgk {

static __constant__ float2 k_negzero2 = {-0.0f, -0.0f};

struct F2 {
    float2 v;
    __device__ __forceinline__ F2() {}
    __device__ __forceinline__ explicit F2(float s) : v(make_float2(s, s)) {}
    __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
    __device__ __forceinline__ explicit F2(float2 w) : v(w) {}
};
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 operator-(F2 a) { return F2(make_float2(-a.v.x, -a.v.y)); }
__device__ __forceinline__ F2 operator+(F2 a) { return a; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2(__fadd2_rn(a.v, make_float2(-b.v.x, -b.v.y))); }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2(__ffma2_rn(a.v, b.v, k_negzero2)); }
__device__ __forceinline__ F2 operator/(F2 a, F2 b) {
    return F2(__fdiv_rn(a.v.x, b.v.x), __fdiv_rn(a.v.y, b.v.y));
}
__device__ __forceinline__ F2 fma_c(F2 a, F2 b, F2 c) { return F2(__ffma2_rn(a.v, b.v, c.v)); }
__device__ __forceinline__ F2 rcp_c(F2 a) { return F2(__frcp_rn(a.v.x), __frcp_rn(a.v.y)); }
__device__ __forceinline__ F2 inv_rn(F2 a) { return rcp_c(a); }

// Storage <-> two compute values (storage units), and the 2-element vectors.
template <class S> struct Pack2;
template <> struct Pack2<float> {
    typedef float2 V;
    static __device__ __forceinline__ F2 raw(V w) { return F2(w); }
    static __device__ __forceinline__ V pack(F2 a) { return a.v; }
    static __device__ __forceinline__ float lo(V w) { return w.x; }
    static __device__ __forceinline__ float hi(V w) { return w.y; }
};
template <> struct Pack2<__half> {
    typedef __half2 V;
    static __device__ __forceinline__ F2 raw(V w) { return F2(__half22float2(w)); }
    static __device__ __forceinline__ V pack(F2 a) { return __floats2half2_rn(a.v.x, a.v.y); }
    static __device__ __forceinline__ __half lo(V w) { return __low2half(w); }
    static __device__ __forceinline__ __half hi(V w) { return __high2half(w); }
};
template <> struct Pack2<__nv_bfloat16> {
    typedef __nv_bfloat162 V;
    static __device__ __forceinline__ F2 raw(V w) { return F2(__bfloat1622float2(w)); }
    static __device__ __forceinline__ V pack(F2 a) { return __floats2bfloat162_rn(a.v.x, a.v.y); }
    static __device__ __forceinline__ __nv_bfloat16 lo(V w) { return __low2bfloat16(w); }
    static __device__ __forceinline__ __nv_bfloat16 hi(V w) { return __high2bfloat16(w); }
};

// Bits of a 16-bit storage value, and two packed values <-> one 32-bit word
// (lo = first element in memory).
__device__ __forceinline__ uint32_t s_bits(__half v) { return __half_as_ushort(v); }
__device__ __forceinline__ uint32_t s_bits(__nv_bfloat16 v) { return __bfloat16_as_ushort(v); }
template <class S> __device__ __forceinline__ S bits_s(uint32_t b);
template <> __device__ __forceinline__ __half bits_s<__half>(uint32_t b) { return __ushort_as_half((unsigned short)b); }
template <> __device__ __forceinline__ __nv_bfloat16 bits_s<__nv_bfloat16>(uint32_t b) {
    return __ushort_as_bfloat16((unsigned short)b);
}
template <class S> __device__ __forceinline__ F2 raw_bits(uint32_t w) {
    typename Pack2<S>::V v;
    memcpy(&v, &w, sizeof w);
    return Pack2<S>::raw(v);
}
// The same conversion, written so that the compiler neither merges it with
// another conversion of the same word nor keeps the result alive instead of
// the word (a caller short of registers converts a packed word twice).  Both
// conversions are exact, so the values equal raw_bits's.
template <class S> __device__ __forceinline__ F2 raw_bits_again(uint32_t w);
template <> __device__ __forceinline__ F2 raw_bits_again<__half>(uint32_t w) {
    float a, b;
    asm volatile("{\n\t.reg .b16 lo, hi;\n\tmov.b32 {lo, hi}, %2;\n\tcvt.f32.f16 %0, lo;\n\tcvt.f32.f16 %1, hi;\n\t}"
                 : "=f"(a), "=f"(b) : "r"(w));
    return F2(a, b);
}
template <> __device__ __forceinline__ F2 raw_bits_again<__nv_bfloat16>(uint32_t w) {
    uint32_t a, b;
    asm volatile("{\n\tshl.b32 %0, %2, 16;\n\tand.b32 %1, %2, 0xffff0000;\n\t}" : "=r"(a), "=r"(b) : "r"(w));
    return F2(__uint_as_float(a), __uint_as_float(b));
}
template <class S> __device__ __forceinline__ uint32_t pack_bits(F2 a) {
    const typename Pack2<S>::V v = Pack2<S>::pack(a);
    uint32_t w;
    memcpy(&w, &v, sizeof w);
    return w;
}

}  // namespace bgk
