// Four consecutive cells along k held by one thread ("quad"), with the
// elementwise arithmetic of the MPDATA formulae.  FP32 quads use one FP32
// instruction per element by default (MPDX_QUAD_PAIRED=1 selects the paired
// float2 add/mul/fma of sm_100 instead; measured slower here because the
// shifted quads of the k-stencils need re-pairing moves); FP64 quads use plain
// double arithmetic (the FP64 translation unit is compiled without FMA
// contraction, so every operation rounds exactly as the reference's does).
#pragma once

#include <cuda_runtime.h>

#include "mpdx_common.cuh"

namespace mpdx {
namespace qd {

template <class T> struct q4;

template <> struct q4<float> {
  float2 a, b;  // elements (a.x, a.y, b.x, b.y)
};
template <> struct q4<double> {
  double x, y, z, w;
};

// element access
__device__ __forceinline__ float e0(const q4<float> &v) { return v.a.x; }
__device__ __forceinline__ float e3(const q4<float> &v) { return v.b.y; }
__device__ __forceinline__ double e0(const q4<double> &v) { return v.x; }
__device__ __forceinline__ double e3(const q4<double> &v) { return v.w; }

__device__ __forceinline__ q4<float> mk(float x, float y, float z, float w) { return {make_float2(x, y), make_float2(z, w)}; }
__device__ __forceinline__ q4<double> mkd(double x, double y, double z, double w) { return {x, y, z, w}; }
template <class T> __device__ __forceinline__ q4<T> bc(T s);
template <> __device__ __forceinline__ q4<float> bc<float>(float s) { return mk(s, s, s, s); }
template <> __device__ __forceinline__ q4<double> bc<double>(double s) { return {s, s, s, s}; }

// shifted quads: (left, x, y, z) and (y, z, w, right)
__device__ __forceinline__ q4<float> shl(const q4<float> &v, float left) { return mk(left, v.a.x, v.a.y, v.b.x); }
__device__ __forceinline__ q4<float> shr(const q4<float> &v, float right) { return mk(v.a.y, v.b.x, v.b.y, right); }
__device__ __forceinline__ q4<double> shl(const q4<double> &v, double left) { return {left, v.x, v.y, v.z}; }
__device__ __forceinline__ q4<double> shr(const q4<double> &v, double right) { return {v.y, v.z, v.w, right}; }

// arithmetic (MPDX_QUAD_PAIRED = 0 selects one FP32 instruction per element)
#ifndef MPDX_QUAD_PAIRED
#define MPDX_QUAD_PAIRED 0
#endif
#if MPDX_QUAD_PAIRED
__device__ __forceinline__ q4<float> operator+(const q4<float> &p, const q4<float> &q) { return {__fadd2_rn(p.a, q.a), __fadd2_rn(p.b, q.b)}; }
__device__ __forceinline__ q4<float> operator-(const q4<float> &p, const q4<float> &q) {
  return {__fadd2_rn(p.a, make_float2(-q.a.x, -q.a.y)), __fadd2_rn(p.b, make_float2(-q.b.x, -q.b.y))};
}
__device__ __forceinline__ q4<float> operator*(const q4<float> &p, const q4<float> &q) { return {__fmul2_rn(p.a, q.a), __fmul2_rn(p.b, q.b)}; }
#else
__device__ __forceinline__ q4<float> operator+(const q4<float> &p, const q4<float> &q) {
  return mk(p.a.x + q.a.x, p.a.y + q.a.y, p.b.x + q.b.x, p.b.y + q.b.y);
}
__device__ __forceinline__ q4<float> operator-(const q4<float> &p, const q4<float> &q) {
  return mk(p.a.x - q.a.x, p.a.y - q.a.y, p.b.x - q.b.x, p.b.y - q.b.y);
}
__device__ __forceinline__ q4<float> operator*(const q4<float> &p, const q4<float> &q) {
  return mk(p.a.x * q.a.x, p.a.y * q.a.y, p.b.x * q.b.x, p.b.y * q.b.y);
}
#endif
// FP32 quotients through mpdx::rdivf (correctly rounded, no slow-path branch):
// the denominators of the formulae are sums plus FLT_MIN or FLT_EPSILON
__device__ __forceinline__ q4<float> operator/(const q4<float> &p, const q4<float> &q) {
  return mk(rdivf(p.a.x, q.a.x), rdivf(p.a.y, q.a.y), rdivf(p.b.x, q.b.x), rdivf(p.b.y, q.b.y));
}
__device__ __forceinline__ q4<float> operator-(const q4<float> &p) { return mk(-p.a.x, -p.a.y, -p.b.x, -p.b.y); }
// p * q + r with one rounding per element (FP32 only; the FP64 path never fuses)
__device__ __forceinline__ q4<float> fma(const q4<float> &p, const q4<float> &q, const q4<float> &r) {
#if MPDX_QUAD_PAIRED
  return {__ffma2_rn(p.a, q.a, r.a), __ffma2_rn(p.b, q.b, r.b)};
#else
  return mk(__fmaf_rn(p.a.x, q.a.x, r.a.x), __fmaf_rn(p.a.y, q.a.y, r.a.y), __fmaf_rn(p.b.x, q.b.x, r.b.x),
            __fmaf_rn(p.b.y, q.b.y, r.b.y));
#endif
}

__device__ __forceinline__ q4<double> operator+(const q4<double> &p, const q4<double> &q) { return {p.x + q.x, p.y + q.y, p.z + q.z, p.w + q.w}; }
__device__ __forceinline__ q4<double> operator-(const q4<double> &p, const q4<double> &q) { return {p.x - q.x, p.y - q.y, p.z - q.z, p.w - q.w}; }
__device__ __forceinline__ q4<double> operator*(const q4<double> &p, const q4<double> &q) { return {p.x * q.x, p.y * q.y, p.z * q.z, p.w * q.w}; }
__device__ __forceinline__ q4<double> operator/(const q4<double> &p, const q4<double> &q) { return {p.x / q.x, p.y / q.y, p.z / q.z, p.w / q.w}; }
__device__ __forceinline__ q4<double> operator-(const q4<double> &p) { return {-p.x, -p.y, -p.z, -p.w}; }
__device__ __forceinline__ q4<double> fma(const q4<double> &p, const q4<double> &q, const q4<double> &r) { return p * q + r; }

// elementwise functions; min/max/pos/neg agree with std::min/std::max for
// non-NaN operands (the only operands the formulae produce)
#define MPDX_Q_MAP1(NAME, EXPR)                                                                      \
  __device__ __forceinline__ q4<float> NAME(const q4<float> &p) {                                    \
    auto f = [](float x) { return EXPR; };                                                           \
    return mk(f(p.a.x), f(p.a.y), f(p.b.x), f(p.b.y));                                                \
  }                                                                                                  \
  __device__ __forceinline__ q4<double> NAME(const q4<double> &p) {                                  \
    auto f = [](double x) { return EXPR; };                                                          \
    return {f(p.x), f(p.y), f(p.z), f(p.w)};                                                         \
  }
MPDX_Q_MAP1(qabs, fabs(x))
MPDX_Q_MAP1(pos, fmax(decltype(x)(0), x))
MPDX_Q_MAP1(neg, fmin(decltype(x)(0), x))
#undef MPDX_Q_MAP1

#define MPDX_Q_MAP2(NAME, EXPR)                                                                      \
  __device__ __forceinline__ q4<float> NAME(const q4<float> &p, const q4<float> &q) {                \
    auto f = [](float x, float y) { return EXPR; };                                                  \
    return mk(f(p.a.x, q.a.x), f(p.a.y, q.a.y), f(p.b.x, q.b.x), f(p.b.y, q.b.y));                   \
  }                                                                                                  \
  __device__ __forceinline__ q4<double> NAME(const q4<double> &p, const q4<double> &q) {             \
    auto f = [](double x, double y) { return EXPR; };                                                \
    return {f(p.x, q.x), f(p.y, q.y), f(p.z, q.z), f(p.w, q.w)};                                     \
  }
MPDX_Q_MAP2(qmin, fmin(x, y))
MPDX_Q_MAP2(qmax, fmax(x, y))
#undef MPDX_Q_MAP2

// FCT limiter factor of GC_mono: C > 0 ? min(1, bd_l, bu_r) : min(1, bu_l, bd_r)
template <class T>
__device__ __forceinline__ T lim1(T C, T bdl, T bur, T bul, T bdr) {
  const bool p = C > T(0);
  return fmin(T(1), fmin(p ? bdl : bul, p ? bur : bdr));
}
// elementwise C > 0 ? a : b
template <class T> __device__ __forceinline__ T sel1(T c, T a, T b) { return c > T(0) ? a : b; }
__device__ __forceinline__ q4<float> sel_pos(const q4<float> &c, const q4<float> &a, const q4<float> &b) {
  return mk(sel1(c.a.x, a.a.x, b.a.x), sel1(c.a.y, a.a.y, b.a.y), sel1(c.b.x, a.b.x, b.b.x), sel1(c.b.y, a.b.y, b.b.y));
}
__device__ __forceinline__ q4<double> sel_pos(const q4<double> &c, const q4<double> &a, const q4<double> &b) {
  return {sel1(c.x, a.x, b.x), sel1(c.y, a.y, b.y), sel1(c.z, a.z, b.z), sel1(c.w, a.w, b.w)};
}
__device__ __forceinline__ q4<float> qlim(const q4<float> &C, const q4<float> &bdl, const q4<float> &bur,
                                          const q4<float> &bul, const q4<float> &bdr) {
  return mk(lim1(C.a.x, bdl.a.x, bur.a.x, bul.a.x, bdr.a.x), lim1(C.a.y, bdl.a.y, bur.a.y, bul.a.y, bdr.a.y),
            lim1(C.b.x, bdl.b.x, bur.b.x, bul.b.x, bdr.b.x), lim1(C.b.y, bdl.b.y, bur.b.y, bul.b.y, bdr.b.y));
}
__device__ __forceinline__ q4<double> qlim(const q4<double> &C, const q4<double> &bdl, const q4<double> &bur,
                                           const q4<double> &bul, const q4<double> &bdr) {
  return {lim1(C.x, bdl.x, bur.x, bul.x, bdr.x), lim1(C.y, bdl.y, bur.y, bul.y, bdr.y),
          lim1(C.z, bdl.z, bur.z, bul.z, bdr.z), lim1(C.w, bdl.w, bur.w, bul.w, bdr.w)};
}

// shared-memory quad load/store (16-byte / 32-byte aligned)
__device__ __forceinline__ q4<float> lds(const float *p) {
  const float4 v = *reinterpret_cast<const float4 *>(p);
  return mk(v.x, v.y, v.z, v.w);
}
__device__ __forceinline__ void sts(float *p, const q4<float> &v) {
  *reinterpret_cast<float4 *>(p) = make_float4(v.a.x, v.a.y, v.b.x, v.b.y);
}
__device__ __forceinline__ q4<double> lds(const double *p) {
  const double2 u = reinterpret_cast<const double2 *>(p)[0], v = reinterpret_cast<const double2 *>(p)[1];
  return {u.x, u.y, v.x, v.y};
}
__device__ __forceinline__ void sts(double *p, const q4<double> &v) {
  reinterpret_cast<double2 *>(p)[0] = make_double2(v.x, v.y);
  reinterpret_cast<double2 *>(p)[1] = make_double2(v.z, v.w);
}

// neighbour quads along k through warp shuffles: lane l holds columns 4l..4l+3
// of its row; a row of 64 columns spans 16 lanes
template <class T>
__device__ __forceinline__ q4<T> km1(const q4<T> &v) {
  const T left = __shfl_up_sync(0xffffffffu, e3(v), 1);
  return shl(v, left);
}
template <class T>
__device__ __forceinline__ q4<T> kp1(const q4<T> &v) {
  const T right = __shfl_down_sync(0xffffffffu, e0(v), 1);
  return shr(v, right);
}

}  // namespace qd
}  // namespace mpdx
