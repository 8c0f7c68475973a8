// Field statistics without any device allocation.
//
// mpdx_field_stats_noalloc() reduces a caller-owned device array to its FP64
// compensated sum, minimum and maximum, like mpdx_stats() does for a solver's
// advectee, but it never calls cudaMalloc/cudaFree or any allocating library:
// the per-slice partial results live in one file-scope __device__ array of
// fixed size.  It serves callers that cannot allocate device memory at the
// point where they need the numbers -- for example code running under a
// caching or pooled allocator that owns all free memory, or a loop whose
// memory budget is fixed when it starts.
//
// Set-up: the first call on each device, with that device current, looks up
// the device address of the scratch array (cudaGetSymbolAddress); make that
// first call before any stream capture.  Every call on a device shares the
// same array, and the array keeps the previous call's contents: the kernels
// overwrite every slot they read, so nothing has to start at zero, but calls
// that overlap on the GPU (concurrent streams) race on the array and must be
// serialised by the caller.
#include <cfloat>
#include <climits>
#include <cstring>
#include <mutex>

#include "mpdx_common.cuh"

namespace mpdx {
namespace noalloc {

struct nsum {  // Neumaier compensated accumulator
  double s = 0, c = 0;
  __device__ __forceinline__ void add(double x) {
    const double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
  }
  __device__ __forceinline__ double value() const { return s + c; }
};

constexpr int kMaxSlices = 8192;  // largest supported extent along axis 0
constexpr int kSliceVals = 4;     // sum, compensation, min, max per slice
constexpr int kThreads = 256;

// partial results of every x-slice (256 KiB, held by every device that loads the library)
static __device__ __align__(256) double g_scratch[kMaxSlices * kSliceVals];

template <class T>
struct view {
  const T *p;
  long long s0, s1, s2;
  __device__ __forceinline__ T operator()(long long i, long long j, long long k) const { return p[i * s0 + j * s1 + k * s2]; }
};

// one block per x-slice i: Neumaier sum over [0,m1) x [0,m2) (if i < m0),
// min / max over [0,n1) x [0,n2)
template <class T>
__global__ void k_slices(view<T> f, int n1, int n2, int m0, int m1, int m2, double *scratch) {
  __shared__ double ss[kThreads], sc[kThreads], smin[kThreads], smax[kThreads];
  const int i = blockIdx.x;
  nsum acc;
  double mn = DBL_MAX, mx = -DBL_MAX;
  const long long tot = (long long)n1 * n2;
  for (long long q = threadIdx.x; q < tot; q += blockDim.x) {
    const int j = int(q / n2), k = int(q % n2);
    const double v = double(f(i, j, k));
    mn = fmin(mn, v);
    mx = fmax(mx, v);
    if (i < m0 && j < m1 && k < m2) acc.add(v);
  }
  const int t = threadIdx.x;
  ss[t] = acc.s; sc[t] = acc.c; smin[t] = mn; smax[t] = mx;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (t < w) {
      nsum a; a.s = ss[t]; a.c = sc[t];
      a.add(ss[t + w]); a.c += sc[t + w];
      ss[t] = a.s; sc[t] = a.c;
      smin[t] = fmin(smin[t], smin[t + w]);
      smax[t] = fmax(smax[t], smax[t + w]);
    }
    __syncthreads();
  }
  if (t == 0) {
    scratch[kSliceVals * i + 0] = ss[0];
    scratch[kSliceVals * i + 1] = sc[0];
    scratch[kSliceVals * i + 2] = smin[0];
    scratch[kSliceVals * i + 3] = smax[0];
  }
}

// slices combined in index order (deterministic), results to out[0..2]
__global__ void k_total(const double *scratch, int n_slices, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  nsum a;
  double c = 0, mn = DBL_MAX, mx = -DBL_MAX;
  for (int s = 0; s < n_slices; ++s) {
    a.add(scratch[kSliceVals * s]);
    c += scratch[kSliceVals * s + 1];
    mn = fmin(mn, scratch[kSliceVals * s + 2]);
    mx = fmax(mx, scratch[kSliceVals * s + 3]);
  }
  out[0] = a.value() + c;
  out[1] = mn;
  out[2] = mx;
}

constexpr int kMaxDevices = 64;
static std::mutex g_mu;
static double *g_addr[kMaxDevices] = {};

static void set_err(char *err, int errlen, const char *msg) {
  if (err && errlen > 0) {
    std::strncpy(err, msg, size_t(errlen) - 1);
    err[errlen - 1] = 0;
  }
}

}  // namespace noalloc
}  // namespace mpdx

extern "C" mpdx_status mpdx_field_stats_noalloc(const void *dev_field, int dtype, const int64_t *n, const int64_t *strides,
                                                const int64_t *m, double *dev_out, void *stream, char *err, int errlen) {
  using namespace mpdx::noalloc;
  set_err(err, errlen, "");
  if (!dev_field || !n || !strides || !m || !dev_out) {
    set_err(err, errlen, "null argument");
    return MPDX_E_ARG;
  }
  if (dtype != 4 && dtype != 8) {
    set_err(err, errlen, "dtype must be 4 or 8");
    return MPDX_E_ARG;
  }
  for (int d = 0; d < 3; ++d) {
    if (n[d] < 1 || m[d] < 0 || m[d] > n[d]) {
      set_err(err, errlen, "extents must satisfy n >= 1 and 0 <= m <= n along every axis");
      return MPDX_E_ARG;
    }
  }
  if (n[0] > kMaxSlices) {
    set_err(err, errlen, "extent along axis 0 exceeds the no-allocation maximum of 8192 slices");
    return MPDX_E_ARG;
  }
  // the kernels index a slice with int: each extent, and a slice's point count,
  // must stay below 2^31 (checked one extent at a time, so the product cannot overflow)
  if (n[1] > INT_MAX || n[2] > INT_MAX || n[1] * n[2] >= (int64_t(1) << 31)) {
    set_err(err, errlen, "slice size must stay below 2^31 points (n[1], n[2] and n[1]*n[2])");
    return MPDX_E_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_err(err, errlen, "no current CUDA device");
    return MPDX_E_CUDA;
  }
  double *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
      if (e != cudaSuccess) {
        set_err(err, errlen, cudaGetErrorString(e));
        return MPDX_E_CUDA;
      }
      g_addr[dev] = static_cast<double *>(p);
    }
    scratch = g_addr[dev];
  }
  // launched through cudaLaunchKernel, whose return value is this launch's own
  // status: an error left pending by an earlier, unrelated call of the caller is
  // neither reported as this call's failure nor cleared
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int n1 = int(n[1]), n2 = int(n[2]), m0 = int(m[0]), m1 = int(m[1]), m2 = int(m[2]), ns = int(n[0]);
  cudaError_t e = cudaSuccess;
  if (dtype == 8) {
    view<double> v{static_cast<const double *>(dev_field), strides[0], strides[1], strides[2]};
    void *args[] = {&v, &n1, &n2, &m0, &m1, &m2, &scratch};
    e = cudaLaunchKernel((const void *)k_slices<double>, dim3(unsigned(ns)), dim3(kThreads), args, 0, s);
  } else {
    view<float> v{static_cast<const float *>(dev_field), strides[0], strides[1], strides[2]};
    void *args[] = {&v, &n1, &n2, &m0, &m1, &m2, &scratch};
    e = cudaLaunchKernel((const void *)k_slices<float>, dim3(unsigned(ns)), dim3(kThreads), args, 0, s);
  }
  if (e == cudaSuccess) {
    void *args[] = {&scratch, &ns, &dev_out};
    e = cudaLaunchKernel((const void *)k_total, dim3(1), dim3(32), args, 0, s);
  }
  if (e != cudaSuccess) {
    set_err(err, errlen, cudaGetErrorString(e));
    return MPDX_E_CUDA;
  }
  return MPDX_OK;
}
