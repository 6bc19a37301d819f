// f32x2.cuh -- two FP32 lanes computed with sm_100's packed FP32x2 instructions (FADD2 / FMUL2 / FFMA2).
//
// F2 holds the values of one quantity at two neighbouring cells.  Arithmetic maps to __fadd2_rn, __fmul2_rn and
// __ffma2_rn, whose per-lane results are those of __fadd_rn, __fmul_rn and __fmaf_rn.  A product is kept pending
// (P2) so that a*b + c, c + a*b, c - a*b and a*b - c become one fused multiply-add, as the compiler contracts the
// scalar FP32 expressions; a pending product used any other way is rounded first.  Scalars broadcast to both lanes.
#pragma once

#include <cuda_runtime.h>
#include <type_traits>

namespace dfdm {

struct F2 {
    float2 v;
    __device__ __forceinline__ F2() {}
    __device__ __forceinline__ F2(float2 a) : v(a) {}
    template <typename S, typename = typename std::enable_if<std::is_arithmetic<S>::value>::type>
    __device__ __forceinline__ F2(S s) { v.x = (float)s; v.y = (float)s; }
    static __device__ __forceinline__ F2 pair(float a, float b) { F2 r; r.v.x = a; r.v.y = b; return r; }
};

struct P2 {   // pending product a*b
    F2 a, b;
    __device__ __forceinline__ operator F2() const { return F2(__fmul2_rn(a.v, b.v)); }
};

__device__ __forceinline__ F2 neg(F2 a) { return F2::pair(-a.v.x, -a.v.y); }
__device__ __forceinline__ F2 eval(const P2 &p) { return F2(__fmul2_rn(p.a.v, p.b.v)); }

__device__ __forceinline__ P2 operator*(F2 a, F2 b) { return P2{a, b}; }
__device__ __forceinline__ P2 operator*(const P2 &p, F2 c) { return P2{eval(p), c}; }
__device__ __forceinline__ P2 operator*(F2 c, const P2 &p) { return P2{c, eval(p)}; }
__device__ __forceinline__ P2 operator*(const P2 &p, const P2 &q) { return P2{eval(p), eval(q)}; }

__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2(__fadd2_rn(a.v, neg(b).v)); }
__device__ __forceinline__ F2 operator-(F2 a) { return neg(a); }
__device__ __forceinline__ P2 operator-(const P2 &p) { return P2{neg(p.a), p.b}; }

__device__ __forceinline__ F2 operator+(const P2 &p, F2 c) { return F2(__ffma2_rn(p.a.v, p.b.v, c.v)); }
__device__ __forceinline__ F2 operator+(F2 c, const P2 &p) { return F2(__ffma2_rn(p.a.v, p.b.v, c.v)); }
__device__ __forceinline__ F2 operator-(F2 c, const P2 &p) { return F2(__ffma2_rn(neg(p.a).v, p.b.v, c.v)); }
__device__ __forceinline__ F2 operator-(const P2 &p, F2 c) { return F2(__ffma2_rn(p.a.v, p.b.v, neg(c).v)); }
__device__ __forceinline__ F2 operator+(const P2 &p, const P2 &q) { return F2(__ffma2_rn(p.a.v, p.b.v, eval(q).v)); }
__device__ __forceinline__ F2 operator-(const P2 &p, const P2 &q) { return F2(__ffma2_rn(p.a.v, p.b.v, neg(eval(q)).v)); }

// scalar operands (metrics, constants) broadcast
__device__ __forceinline__ P2 operator*(float s, F2 b) { return P2{F2(s), b}; }
__device__ __forceinline__ P2 operator*(F2 a, float s) { return P2{a, F2(s)}; }
__device__ __forceinline__ P2 operator*(const P2 &p, float s) { return P2{eval(p), F2(s)}; }
__device__ __forceinline__ P2 operator*(float s, const P2 &p) { return P2{F2(s), eval(p)}; }
__device__ __forceinline__ F2 operator+(F2 a, float s) { return a + F2(s); }
__device__ __forceinline__ F2 operator+(float s, F2 a) { return F2(s) + a; }
__device__ __forceinline__ F2 operator-(F2 a, float s) { return a - F2(s); }
__device__ __forceinline__ F2 operator-(float s, F2 a) { return F2(s) - a; }
__device__ __forceinline__ F2 operator+(const P2 &p, float s) { return p + F2(s); }
__device__ __forceinline__ F2 operator+(float s, const P2 &p) { return F2(s) + p; }

// the FP32 forms (base profile, difference forms) apply to float and to its packed pairs
template <typename T> struct Fp32Forms { static constexpr bool value = !std::is_same<T, double>::value; };

}  // namespace dfdm
