// Packed FP32 pairs for the FP32 Jacobian product.
//
// sm_100 executes FP32 add, multiply and fused multiply-add on pairs of
// values held in one 64-bit register pair (FADD2 / FMUL2 / FFMA2, the
// __fadd2_rn / __fmul2_rn / __ffma2_rn intrinsics), one instruction for two
// results.  The FP32 product is bound by instruction issue, so the pair
// kernel runs two tiles at once: lane x of every value belongs to the first
// tile, lane y to the second, and the templated cell code runs unchanged on
// this type.  Products are kept pending (P2) until they are added, so that
// a * b + c becomes one FFMA2 as the scalar code's contraction would make it
// one FFMA; every lane rounds exactly as a scalar FP32 operation does.
#pragma once

#include <cuda_runtime.h>

namespace sint
{
  struct P2;

  // a parameter type excluded from template argument deduction, so that a
  // pending product (P2) converts to the type deduced from the other arguments
  template <typename T>
  struct nondeduced
  {
    using type = T;
  };
  template <typename T>
  using nd = typename nondeduced<T>::type;

  struct F2
  {
    float2 v;
    F2() = default;
    __host__ __device__ __forceinline__ explicit F2(double d) : v(make_float2(float(d), float(d))) {}
    __host__ __device__ __forceinline__ explicit F2(float d) : v(make_float2(d, d)) {}
    __host__ __device__ __forceinline__ explicit F2(int d) : v(make_float2(float(d), float(d))) {}
    __host__ __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
    __host__ __device__ __forceinline__ explicit F2(float2 x) : v(x) {}
    __device__ __forceinline__ F2(const P2 &p);
  };

  // a pending product a * b (lane-wise)
  struct P2
  {
    float2 a, b;
  };

  __device__ __forceinline__ float2 f2neg(float2 x) { return make_float2(-x.x, -x.y); }
  __device__ __forceinline__ F2::F2(const P2 &p) : v(__fmul2_rn(p.a, p.b)) {}

  __device__ __forceinline__ P2 operator*(const F2 &a, const F2 &b) { return P2{a.v, b.v}; }
  __device__ __forceinline__ P2 operator*(const P2 &a, const F2 &b) { return P2{__fmul2_rn(a.a, a.b), b.v}; }
  __device__ __forceinline__ P2 operator*(const F2 &a, const P2 &b) { return P2{a.v, __fmul2_rn(b.a, b.b)}; }
  __device__ __forceinline__ P2 operator*(const P2 &a, const P2 &b)
  {
    return P2{__fmul2_rn(a.a, a.b), __fmul2_rn(b.a, b.b)};
  }
  __device__ __forceinline__ F2 operator+(const F2 &a, const F2 &b) { return F2(__fadd2_rn(a.v, b.v)); }
  __device__ __forceinline__ F2 operator-(const F2 &a, const F2 &b) { return F2(__fadd2_rn(a.v, f2neg(b.v))); }
  __device__ __forceinline__ F2 operator-(const F2 &a) { return F2(f2neg(a.v)); }
  __device__ __forceinline__ F2 operator+(const P2 &p, const F2 &c) { return F2(__ffma2_rn(p.a, p.b, c.v)); }
  __device__ __forceinline__ F2 operator+(const F2 &c, const P2 &p) { return F2(__ffma2_rn(p.a, p.b, c.v)); }
  __device__ __forceinline__ F2 operator+(const P2 &p, const P2 &q)
  {
    return F2(__ffma2_rn(p.a, p.b, __fmul2_rn(q.a, q.b)));
  }
  __device__ __forceinline__ F2 operator-(const F2 &c, const P2 &p) { return F2(__ffma2_rn(f2neg(p.a), p.b, c.v)); }
  __device__ __forceinline__ F2 operator-(const P2 &p, const F2 &c) { return F2(__ffma2_rn(p.a, p.b, f2neg(c.v))); }
  __device__ __forceinline__ F2 operator-(const P2 &p, const P2 &q)
  {
    return F2(__ffma2_rn(f2neg(q.a), q.b, __fmul2_rn(p.a, p.b)));
  }
  __device__ __forceinline__ P2 operator-(const P2 &p) { return P2{f2neg(p.a), p.b}; }
  __device__ __forceinline__ F2 &operator+=(F2 &a, const F2 &b) { return a = a + b; }
  __device__ __forceinline__ F2 &operator-=(F2 &a, const F2 &b) { return a = a - b; }
  __device__ __forceinline__ F2 &operator+=(F2 &a, const P2 &b) { return a = a + b; }
  __device__ __forceinline__ F2 &operator-=(F2 &a, const P2 &b) { return a = a - b; }
  __device__ __forceinline__ F2 &operator*=(F2 &a, const F2 &b) { return a = F2(a * b); }

  // the scalar overloads stay visible beside the pair ones inside sint
  using ::fmax;
  using ::fmin;

  // lane-wise comparison results and selection
  struct M2
  {
    bool x, y;
  };
  __device__ __forceinline__ M2 operator<(const F2 &a, const F2 &b) { return M2{a.v.x < b.v.x, a.v.y < b.v.y}; }
  __device__ __forceinline__ M2 operator>(const F2 &a, const F2 &b) { return M2{a.v.x > b.v.x, a.v.y > b.v.y}; }
  __device__ __forceinline__ F2 sel(const M2 &m, const F2 &a, const F2 &b)
  {
    return F2(m.x ? a.v.x : b.v.x, m.y ? a.v.y : b.v.y);
  }
  // v with lane x zeroed unless a, lane y unless b (a scalar keeps v when a)
  template <typename R>
  __device__ __forceinline__ R lane_keep(R v, bool a, bool)
  {
    return a ? v : R(0);
  }
  __device__ __forceinline__ F2 lane_keep(F2 v, bool a, bool b) { return F2(a ? v.v.x : 0.f, b ? v.v.y : 0.f); }
  __device__ __forceinline__ F2 fmin(const F2 &a, const F2 &b) { return F2(fminf(a.v.x, b.v.x), fminf(a.v.y, b.v.y)); }
  __device__ __forceinline__ F2 fmax(const F2 &a, const F2 &b) { return F2(fmaxf(a.v.x, b.v.x), fmaxf(a.v.y, b.v.y)); }
} // namespace sint
