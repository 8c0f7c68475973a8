// Device reductions for per-step statistics: FP64 compensated (Neumaier) sum,
// min and max of one scalar field.  The reduction tree has a fixed shape (fixed
// grid, fixed per-thread strides, fixed shared-memory tree, one final block),
// so results are bitwise reproducible from run to run, as the reference's
// two-step per-slice-then-total sums are (concurr/detail/sharedmem.hpp:115-199,
// kahan_reduction.hpp:15-58).
#pragma once

#include <cfloat>

#include "state.cuh"

namespace mpdx {

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

constexpr int kStatBlocks = 296;  // fixed: 2 x 148 SMs
constexpr int kStatThreads = 256;

template <class T>
__global__ void k_stats_partial(dfield<T> f, int n0, int n1, int n2, int m0, int m1, int m2, double *part) {
  // sum over the unique cells [0, m) (m = n - 1 along cyclic axes), min/max over all n
  __shared__ double ss[kStatThreads], sc[kStatThreads], smin[kStatThreads], smax[kStatThreads];
  nsum acc;
  double mn = DBL_MAX, mx = -DBL_MAX;
  const long long tot = (long long)n0 * n1 * n2;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += stride) {
    const int k = int(q % n2);
    const long long r = q / n2;
    const int j = int(r % n1), i = int(r / n1);
    const double v = double(f(i, j, k));
    mn = fmin(mn, v);
    mx = fmax(mx, v);
    if (i < m0 && j < m1 && k < m2) acc.add(v);
  }
  const int t = threadIdx.x;
  ss[t] = acc.s; sc[t] = acc.c; smin[t] = mn; smax[t] = mx;
  __syncthreads();
  for (int w = kStatThreads / 2; w > 0; w >>= 1) {
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
    part[4 * blockIdx.x + 0] = ss[0];
    part[4 * blockIdx.x + 1] = sc[0];
    part[4 * blockIdx.x + 2] = smin[0];
    part[4 * blockIdx.x + 3] = smax[0];
  }
}

__global__ void k_stats_final(const double *part, int nb, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  nsum a;
  double c = 0, mn = DBL_MAX, mx = -DBL_MAX;
  for (int b = 0; b < nb; ++b) {
    a.add(part[4 * b]);
    c += part[4 * b + 1];
    mn = fmin(mn, part[4 * b + 2]);
    mx = fmax(mx, part[4 * b + 3]);
  }
  out[0] = a.value() + c;
  out[1] = mn;
  out[2] = mx;
}

template <class T>
struct stats_engine {
  double *part = nullptr, *res = nullptr;
  ~stats_engine() {
    if (part) cudaFree(part);
    if (res) cudaFree(res);
  }
  template <class S>
  void reduce(const S &st, const field<T> &f, mpdx_step_stats *out) {
    if (!part) {
      MPDX_CUDA(cudaMalloc(&part, sizeof(double) * 4 * kStatBlocks));
      MPDX_CUDA(cudaMalloc(&res, sizeof(double) * 4));
    }
    int m[3];
    for (int d = 0; d < 3; ++d) {
      const bool cyc = d < st.nd && st.bcs[d][0] == MPDX_BC_CYCLIC && st.bcs[d][1] == MPDX_BC_CYCLIC && st.n[d] > 1;
      m[d] = cyc ? st.n[d] - 1 : st.n[d];
    }
    k_stats_partial<T><<<kStatBlocks, kStatThreads, 0, st.stream>>>(f.v, st.n[0], st.n[1], st.n[2], m[0], m[1], m[2], part);
    MPDX_LAUNCH_CHECK();
    k_stats_final<<<1, 32, 0, st.stream>>>(part, kStatBlocks, res);
    MPDX_LAUNCH_CHECK();
    double h[3];
    MPDX_CUDA(cudaMemcpyAsync(h, res, sizeof(h), cudaMemcpyDeviceToHost, st.stream));
    MPDX_CUDA(cudaStreamSynchronize(st.stream));
    out->mass = h[0];
    out->min = h[1];
    out->max = h[2];
  }
};

}  // namespace mpdx
