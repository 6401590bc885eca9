// Two-lane arithmetic for the collide pass, whose work comes in twins: the
// two directions of an opposite pair (e, -e) and the two staged fields c and
// p share every operation of their stencils. FP32 lanes map to the packed
// f32x2 instructions of sm_100 (one FFMA2 / FADD2 / FMUL2 does both lanes,
// each lane rounded as the scalar operation would be); FP64 lanes are two
// scalar instructions. No operation here contracts a multiply and an add
// unless it is written as fma.
#pragma once
#include <cuda_runtime.h>

namespace fe {

template <class R>
struct V2;

template <>
struct alignas(8) V2<float> {
  float2 v;
  __device__ __forceinline__ V2() {}
  __device__ __forceinline__ V2(float a, float b) : v(make_float2(a, b)) {}
  __device__ __forceinline__ explicit V2(float s) : v(make_float2(s, s)) {}
  __device__ __forceinline__ float x() const { return v.x; }
  __device__ __forceinline__ float y() const { return v.y; }
  __device__ __forceinline__ static V2 raw(float2 f) {
    V2 r;
    r.v = f;
    return r;
  }
};
__device__ __forceinline__ V2<float> operator+(V2<float> a, V2<float> b) { return V2<float>::raw(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ V2<float> operator*(V2<float> a, V2<float> b) { return V2<float>::raw(__fmul2_rn(a.v, b.v)); }
// a - b as b * (-1) + a: the product is exact, so one rounding, as FADD
__device__ __forceinline__ V2<float> operator-(V2<float> a, V2<float> b) {
  return V2<float>::raw(__ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v));
}
__device__ __forceinline__ V2<float> fma2(V2<float> a, V2<float> b, V2<float> c) {
  return V2<float>::raw(__ffma2_rn(a.v, b.v, c.v));
}

template <>
struct alignas(16) V2<double> {
  double a_, b_;
  __device__ __forceinline__ V2() {}
  __device__ __forceinline__ V2(double a, double b) : a_(a), b_(b) {}
  __device__ __forceinline__ explicit V2(double s) : a_(s), b_(s) {}
  __device__ __forceinline__ double x() const { return a_; }
  __device__ __forceinline__ double y() const { return b_; }
};
__device__ __forceinline__ V2<double> operator+(V2<double> a, V2<double> b) {
  return V2<double>(__dadd_rn(a.a_, b.a_), __dadd_rn(a.b_, b.b_));
}
__device__ __forceinline__ V2<double> operator-(V2<double> a, V2<double> b) {
  return V2<double>(__dsub_rn(a.a_, b.a_), __dsub_rn(a.b_, b.b_));
}
__device__ __forceinline__ V2<double> operator*(V2<double> a, V2<double> b) {
  return V2<double>(__dmul_rn(a.a_, b.a_), __dmul_rn(a.b_, b.b_));
}
__device__ __forceinline__ V2<double> fma2(V2<double> a, V2<double> b, V2<double> c) {
  return V2<double>(fma(a.a_, b.a_, c.a_), fma(a.b_, b.b_, c.b_));
}

// lane-wise select with one predicate for both lanes
template <class R>
__device__ __forceinline__ V2<R> sel(bool p, V2<R> a, V2<R> b) {
  return V2<R>(p ? a.x() : b.x(), p ? a.y() : b.y());
}

}  // namespace fe
