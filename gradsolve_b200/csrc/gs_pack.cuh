// gs_pack.cuh -- a real type holding two float32 trajectories side by side, evaluated with
// sm_100's packed float32x2 instructions (__ffma2_rn / __fadd2_rn / __fmul2_rn: one
// instruction, two round-to-nearest float operations).
//
// The step helpers and the fields are templated on the real type R and use only +, -, *,
// unary minus and R(constant); instantiating them with F2 runs two trajectories per thread in
// half the float instructions.  Products are kept lazy (P2) so that a product that feeds an
// addition becomes one fused multiply-add, as the compiler contracts the scalar float code:
//   a * b          -> P2{a, b}                 (nothing issued yet)
//   P2 + c, c + P2 -> ffma2(a, b, c)
//   P2 - c         -> ffma2(a, b, -c),  c - P2 -> ffma2(-a, b, c)
//   P2 + P2        -> ffma2(a1, b1, a2 * b2)
//   P2 used as F2  -> fmul2(a, b)
// F1 is the one-trajectory twin: the same lazy products and the same contractions, issued as
// scalar __fmaf_rn / __fadd_rn / __fmul_rn (which the compiler never re-associates or fuses).
// A step evaluated with F1 and either half of the same step evaluated with F2 are therefore
// the same float operations in the same order -- bit for bit alike -- so the float32 route's
// forward, replay and one-per-thread reverse pass (F1) and its two-per-thread reverse pass (F2)
// all see the same states.
#pragma once
#include <cuda_runtime.h>

namespace gs {

struct F2 {
  float2 v;
  F2() = default;
  __device__ __forceinline__ explicit F2(float2 x) : v(x) {}
  __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
  // a constant, broadcast (rounded to float as the scalar float code rounds R(constant))
  __device__ __forceinline__ F2(double c) : v(make_float2((float)c, (float)c)) {}
};

struct P2 {
  F2 a, b;
  __device__ __forceinline__ operator F2() const { return F2(__fmul2_rn(a.v, b.v)); }
};

__device__ __forceinline__ F2 neg(F2 x) { return F2(-x.v.x, -x.v.y); }

__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return F2(__ffma2_rn(a.v, b.v, c.v)); }

__device__ __forceinline__ P2 operator*(F2 a, F2 b) { return P2{a, b}; }
__device__ __forceinline__ P2 operator*(P2 a, F2 b) { return P2{F2(a), b}; }
__device__ __forceinline__ P2 operator*(F2 a, P2 b) { return P2{a, F2(b)}; }
__device__ __forceinline__ P2 operator*(P2 a, P2 b) { return P2{F2(a), F2(b)}; }

__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 operator+(P2 a, F2 c) { return fma2(a.a, a.b, c); }
__device__ __forceinline__ F2 operator+(F2 c, P2 a) { return fma2(a.a, a.b, c); }
__device__ __forceinline__ F2 operator+(P2 a, P2 b) { return fma2(a.a, a.b, F2(b)); }

__device__ __forceinline__ F2 operator-(F2 a) { return neg(a); }
__device__ __forceinline__ P2 operator-(P2 a) { return P2{neg(a.a), a.b}; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2(__fadd2_rn(a.v, neg(b).v)); }
__device__ __forceinline__ F2 operator-(P2 a, F2 c) { return fma2(a.a, a.b, neg(c)); }
__device__ __forceinline__ F2 operator-(F2 c, P2 a) { return fma2(neg(a.a), a.b, c); }
__device__ __forceinline__ F2 operator-(P2 a, P2 b) { return fma2(a.a, a.b, neg(F2(b))); }

// division only appears between constants in the fields (e.g. R(8.0) / R(3.0)), which the
// compiler folds
__device__ __forceinline__ F2 operator/(F2 a, F2 b) { return F2(a.v.x / b.v.x, a.v.y / b.v.y); }

__device__ __forceinline__ F2& operator+=(F2& a, F2 b) { return a = a + b; }
__device__ __forceinline__ F2& operator+=(F2& a, P2 b) { return a = b + a; }
__device__ __forceinline__ F2& operator-=(F2& a, F2 b) { return a = a - b; }
__device__ __forceinline__ F2& operator-=(F2& a, P2 b) { return a = a - b; }
__device__ __forceinline__ F2& operator*=(F2& a, F2 b) { return a = F2(a * b); }

// ---- F1: one trajectory, the same rules in scalar float ---------------------------------
struct F1 {
  float v;
  F1() = default;
  __device__ __forceinline__ F1(float x) : v(x) {}
  // a constant (rounded to float as the scalar float code rounds R(constant))
  __device__ __forceinline__ F1(double c) : v((float)c) {}
};

struct P1 {
  F1 a, b;
  __device__ __forceinline__ operator F1() const { return F1(__fmul_rn(a.v, b.v)); }
};

__device__ __forceinline__ F1 neg(F1 x) { return F1(-x.v); }

__device__ __forceinline__ F1 fma1(F1 a, F1 b, F1 c) { return F1(__fmaf_rn(a.v, b.v, c.v)); }

__device__ __forceinline__ P1 operator*(F1 a, F1 b) { return P1{a, b}; }
__device__ __forceinline__ P1 operator*(P1 a, F1 b) { return P1{F1(a), b}; }
__device__ __forceinline__ P1 operator*(F1 a, P1 b) { return P1{a, F1(b)}; }
__device__ __forceinline__ P1 operator*(P1 a, P1 b) { return P1{F1(a), F1(b)}; }

__device__ __forceinline__ F1 operator+(F1 a, F1 b) { return F1(__fadd_rn(a.v, b.v)); }
__device__ __forceinline__ F1 operator+(P1 a, F1 c) { return fma1(a.a, a.b, c); }
__device__ __forceinline__ F1 operator+(F1 c, P1 a) { return fma1(a.a, a.b, c); }
__device__ __forceinline__ F1 operator+(P1 a, P1 b) { return fma1(a.a, a.b, F1(b)); }

__device__ __forceinline__ F1 operator-(F1 a) { return neg(a); }
__device__ __forceinline__ P1 operator-(P1 a) { return P1{neg(a.a), a.b}; }
__device__ __forceinline__ F1 operator-(F1 a, F1 b) { return F1(__fadd_rn(a.v, neg(b).v)); }
__device__ __forceinline__ F1 operator-(P1 a, F1 c) { return fma1(a.a, a.b, neg(c)); }
__device__ __forceinline__ F1 operator-(F1 c, P1 a) { return fma1(neg(a.a), a.b, c); }
__device__ __forceinline__ F1 operator-(P1 a, P1 b) { return fma1(a.a, a.b, neg(F1(b))); }

__device__ __forceinline__ F1 operator/(F1 a, F1 b) { return F1(a.v / b.v); }

__device__ __forceinline__ F1& operator+=(F1& a, F1 b) { return a = a + b; }
__device__ __forceinline__ F1& operator+=(F1& a, P1 b) { return a = b + a; }
__device__ __forceinline__ F1& operator-=(F1& a, F1 b) { return a = a - b; }
__device__ __forceinline__ F1& operator-=(F1& a, P1 b) { return a = a - b; }
__device__ __forceinline__ F1& operator*=(F1& a, F1 b) { return a = F1(a * b); }

// Fields whose expressions use only the operations above (the built-in nonstiff fields); the
// float32 reverse pass runs them two trajectories per thread.
template <class F>
struct Packable {
  static constexpr bool value = false;
};

}  // namespace gs
