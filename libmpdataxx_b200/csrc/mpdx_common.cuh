// Shared definitions of the libmpdataxx_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "../../include/mpdx.h"

namespace mpdx {

// Named range on the NVTX timeline (the tracing of this library: Nsight Systems
// and Nsight Compute show each entry point and solver phase by name).  NVTX is
// header-only: without a tool attached a range costs one check of a function
// pointer.
struct trace_range {
  explicit trace_range(const char *name) { nvtxRangePushA(name); }
  ~trace_range() { nvtxRangePop(); }
  trace_range(const trace_range &) = delete;
  trace_range &operator=(const trace_range &) = delete;
};

// option bits (libmpdata++/opts.hpp:34-49)
enum : unsigned {
  o_fct = 1u << 0, o_abs = 1u << 1, o_tot = 1u << 2, o_pfc = 1u << 3,
  o_npa = 1u << 4, o_iga = 1u << 5, o_nug = 1u << 6, o_dfl = 1u << 7,
  o_khn = 1u << 8, o_div_2nd = 1u << 9, o_div_3rd = 1u << 10,
  o_div_3rd_dt = 1u << 11, o_fot = 1u << 12
};

struct error : std::runtime_error {
  mpdx_status code;
  error(mpdx_status c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define MPDX_CUDA(call)                                                                     \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      throw ::mpdx::error(MPDX_E_CUDA, std::string(#call ": ") + cudaGetErrorString(e_));   \
  } while (0)

#define MPDX_LAUNCH_CHECK() MPDX_CUDA(cudaGetLastError())

struct rng {
  int f, l;
  int n() const { return l - f + 1; }
};
inline rng ext(rng r, int n) { return {r.f - n, r.l + n}; }  // r^n
inline rng exh(rng r) { return {r.f - 1, r.l}; }             // r^h

// Device view of a field stored with its halo: element (i, j, k) lives at
// o[i*s0 + j*s1 + k*s2]; unused dimensions are pinned to index 0.
#ifdef MPDX_BOUNDS_CHECK
// where the bounds-checked build records the first out-of-range field access
struct oob_info {
  unsigned hit;
  int i, j, k;
};
// one record per device, allocated on first use (the current device's)
inline oob_info *oob_record() {
  static oob_info *rec[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return nullptr;
  if (!rec[dev]) {
    if (cudaMalloc(&rec[dev], sizeof(oob_info)) != cudaSuccess) { rec[dev] = nullptr; return nullptr; }
    cudaMemset(rec[dev], 0, sizeof(oob_info));
  }
  return rec[dev];
}
#endif

template <class T>
struct dfield {
  T *o = nullptr;
  long long s0 = 0, s1 = 0, s2 = 0;
#ifdef MPDX_BOUNDS_CHECK
  // the bounds-checked build (libmpdx_debug.so): the index ranges of the allocation
  // (lo > hi: not checked, as for views built from a bare pointer) and the flag that
  // an access outside them sets instead of touching memory outside the field
  int lo[3] = {1, 1, 1}, hi[3] = {0, 0, 0};
  oob_info *oob = nullptr;
#endif
  __host__ __device__ __forceinline__ T &operator()(int i, int j, int k) const {
#if defined(MPDX_BOUNDS_CHECK) && defined(__CUDA_ARCH__)
    if (oob && lo[0] <= hi[0] &&
        (i < lo[0] || i > hi[0] || j < lo[1] || j > hi[1] || k < lo[2] || k > hi[2])) {
      if (atomicExch(&oob->hit, 1u) == 0u) { oob->i = i; oob->j = j; oob->k = k; }
      return o[lo[0] * s0 + lo[1] * s1 + lo[2] * s2];  // the field's first point: the call fails afterwards
    }
#endif
    return o[i * s0 + j * s1 + k * s2];
  }
};

// Owning device allocation of one field (scalar, or one vector component).
// The fastest-varying dimension is padded so that index 0 of every row sits on
// a 128-byte boundary; rows have a pitch that is a multiple of 128 bytes.
template <class T>
struct field {
  void *base = nullptr;
  size_t bytes = 0;
  int nd = 0;
  rng r[3] = {{0, 0}, {0, 0}, {0, 0}};
  dfield<T> v;
  field() = default;
  field(const field &) = delete;
  field &operator=(const field &) = delete;
  field(field &&o) noexcept { *this = std::move(o); }
  field &operator=(field &&o) noexcept {
    std::swap(base, o.base); std::swap(bytes, o.bytes); nd = o.nd;
    for (int q = 0; q < 3; ++q) r[q] = o.r[q];
    v = o.v; return *this;
  }
  ~field() { if (base) cudaFree(base); }

  // `stream` is the stream every later use of the field is ordered on: the zero fill
  // goes there too (a legacy-stream memset would not be ordered with work on
  // a non-blocking stream)
  void alloc(int nd_, const rng *rr, cudaStream_t stream) {
    nd = nd_;
    for (int q = 0; q < 3; ++q) r[q] = q < nd ? rr[q] : rng{0, 0};
    const int align = int(128 / sizeof(T));
    const int f = nd - 1;  // fastest dimension
    const int front = ((-r[f].f) + align - 1) / align * align;
    const long long pitch = ((long long)front + r[f].l + 1 + align - 1) / align * align;
    long long s[3] = {0, 0, 0};
    s[f] = 1;
    long long acc = pitch;
    for (int q = f - 1; q >= 0; --q) { s[q] = acc; acc *= r[q].n(); }
    bytes = size_t(acc) * sizeof(T);
    MPDX_CUDA(cudaMalloc(&base, bytes));
#ifdef MPDX_POISON
    // the debug build fills new fields with NaN (all bits set), so that a value read
    // before anything wrote it shows in the results
    MPDX_CUDA(cudaMemsetAsync(base, 0xff, bytes, stream));
#else
    MPDX_CUDA(cudaMemsetAsync(base, 0, bytes, stream));
#endif
    long long off = front;
    for (int q = 0; q < f; ++q) off += (long long)(-r[q].f) * s[q];
    v.o = static_cast<T *>(base) + off;
    v.s0 = s[0]; v.s1 = s[1]; v.s2 = s[2];
    // indices of unused dimensions are always 0; give them stride 0
    for (int q = nd; q < 3; ++q) (q == 0 ? v.s0 : q == 1 ? v.s1 : v.s2) = 0;
#ifdef MPDX_BOUNDS_CHECK
    for (int q = 0; q < 3; ++q) {
      v.lo[q] = q < nd ? r[q].f : -2147483647;
      v.hi[q] = q < nd ? r[q].l : 2147483647;
    }
    v.oob = oob_record();
#endif
  }
};

inline unsigned ceil_div(long long a, long long b) { return unsigned((a + b - 1) / b); }

// a / b, correctly rounded, from y = RN(1/b): q = RN(a y), r = a - b q (exact
// with one FMA), result RN(q + r y) -- Markstein's correction step (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000 processor",
// IBM J. Res. Dev. 34(1), 1990).  Equals the IEEE quotient for operands away
// from overflow and underflow (checked against the '/' operator by
// tests/cuda/qdiv_check.cu); a zero numerator gives +0.
template <class T>
__device__ __forceinline__ T qdiv(T a, T b, T y) {
  const T q = a * y;
  const T r = fma(-q, b, a);
  return fma(r, y, q);
}

// a / b in FP32, correctly rounded and without a branch, for normal b whose
// reciprocal is normal and a quotient that neither overflows nor underflows.
// y0 = rcp.approx(b) (relative error below 2^-22), two Newton-Raphson steps
// y <- y + y (1 - b y) leave an error of about 2^-70 relative before the last
// rounding, below the least distance (about 2^-47 relative) of the reciprocal
// of a 24-bit number from a rounding midpoint, so y = RN(1/b); Markstein's
// correction (qdiv) then returns RN(a/b).  Checked against the '/' operator by
// tests/cuda/qdiv_check.cu.
__device__ __forceinline__ float rdivf(float a, float b) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(b));
  y = fmaf(fmaf(-b, y, 1.0f), y, y);
  y = fmaf(fmaf(-b, y, 1.0f), y, y);
  return qdiv(a, b, y);
}

// a / b in FP64 without the division's slow path, for normal b whose reciprocal is
// normal and quotients that neither overflow nor underflow: y0 = rcp.approx.ftz.f64(b),
// two Newton-Raphson steps y <- y + y (1 - b y) (each squares the relative error,
// down to the rounding of y), then Markstein's correction (qdiv).  The result is
// within one ulp of the IEEE quotient (equal to it for all but a small fraction of
// operands; tests/cuda/qdiv_check.cu counts both).
__device__ __forceinline__ double rdivd(double a, double b) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  y = fma(fma(-b, y, 1.0), y, y);
  y = fma(fma(-b, y, 1.0), y, y);
  return qdiv(a, b, y);
}

}  // namespace mpdx
