// Boussinesq solver with GCR(k) pressure solve on the device.
//
// The time step follows libmpdata++'s hook chain (paths inside the
// libmpdata++ source tree):
//   hook_ante_loop   mpdata_rhs_vip_prs_common.hpp:130-160 (initial projection,
//                    ini_pressure), mpdata_rhs_vip_common.hpp:283-302, mpdata_rhs.hpp:154-169
//   calc_gc          mpdata_rhs_vip_common.hpp:120-153 (extrp), mpdata_rhs_vip.hpp
//                    (xchng_pres of the stash, intrp, advector halo fills)
//   hook_ante_step   mpdata_rhs_vip_common.hpp:351-364, mpdata_rhs.hpp:171-193
//   advection        general<T>::step() (solver_common.hpp:127-136)
//   hook_post_step   mpdata_rhs.hpp:195-214, boussinesq_expl.hpp:83-126,
//                    mpdata_rhs_vip_prs_common.hpp:162-181
//   pressure solve   mpdata_rhs_vip_prs_common.hpp:47-128, mpdata_rhs_vip_prs_gcrk.hpp:39-97
//
// Pointwise stages that the reference runs as separate array statements are
// fused into one kernel each (the per-point arithmetic and its order are
// unchanged).  The GCR iteration runs as two kernels per inner step:
//   k_gcr_update: err' = err + beta lap_p_v, lap_err = lap(err'), max|err'| and
//                 the alpha sums;
//   k_gcr_direction: Phi += beta p_v (deferred here from the reference's first
//                 half because this kernel reads p_v anyway: same arithmetic,
//                 8 bytes less per point), new search direction and its lap,
//                 and the sums of the next beta.
// lap() is evaluated straight from the interior values: a point outside the
// interior takes the value its pressure halo fill would give it (cyclic copy,
// or rigid one-sided extrapolation), and the gradient component vanishes on a
// rigid wall (set_edges), so no halo-fill kernels run inside the loop.  Sums
// are compensated double-double reductions with a fixed tree (reproducible);
// the last block of each reduction finalises the GCR scalars on the device.
// Convergence is a device flag: bodies are launched in batches and kernels
// return at once after convergence, so the host reads one flag per batch.
// Compiled with --fmad=false: FP64 results follow the reference's rounding.
#include <algorithm>
#include <cfloat>
#include <cstring>
#include <type_traits>

#include "boussinesq.cuh"
#include "precond.cuh"

namespace mpdx {
namespace bq {

struct geom {
  int nd, n[3], bc[3][2];
  int nf, nrows;            // points along the last axis; rows = all other axes
  double dxd[3], rdxd[3];   // spacing and RN(1/spacing), FP64
  float dxf[3], rdxf[3];    // the same in FP32
  long long cells;
  // normalize_vip of the gradient inside lap() (mpdata_rhs_vip_prs_common.hpp:72-74):
  // lap_tmp[d] /= den[d] at every point, den[d] a pressure-type field; norm = 0: none
  int norm = 0;
  const void *den[3] = {nullptr, nullptr, nullptr};
  template <class T> __device__ __forceinline__ T dn(int d, long long q) const { return static_cast<const T *>(den[d])[q]; }
  template <class T> __device__ __forceinline__ T dx(int d) const { if constexpr (sizeof(T) == 4) return dxf[d]; else return dxd[d]; }
  template <class T> __device__ __forceinline__ T rdx(int d) const { if constexpr (sizeof(T) == 4) return rdxf[d]; else return rdxd[d]; }
};

// Every interior point once: threadIdx.x runs along the last (contiguous)
// axis, threadIdx.y and the blocks over the rows of the other axes.
template <class F>
__device__ __forceinline__ void for_interior(const geom &g, F &&fn) {
  for (int row = blockIdx.x * blockDim.y + threadIdx.y; row < g.nrows; row += gridDim.x * blockDim.y) {
    int i = row, j = 0;
    if (g.nd == 3) { i = row / g.n[1]; j = row - i * g.n[1]; }
    for (int f = threadIdx.x; f < g.nf; f += blockDim.x) {
      if (g.nd == 3) fn(i, j, f);
      else fn(i, f, 0);
    }
  }
}

// Field accessors by linear element offset.  Every pressure-type field of a
// solver has the same layout (same halo ranges and padding), so one offset
// addresses the same point in each of them.
template <class T>
struct fld {
  const T *o;
  __device__ __forceinline__ T operator()(long long q) const { return o[q]; }
};
// err + beta * lap_p: the updated error, evaluated where it is read
template <class T>
struct fld_axpy {
  const T *x, *y;
  T b;
  __device__ __forceinline__ T operator()(long long q) const { return x[q] + b * y[q]; }
};

template <class T>
__device__ __forceinline__ long long off3(const dfield<T> &f, int i, int j, int k) {
  return (long long)i * f.s0 + (long long)j * f.s1 + (long long)k * f.s2;
}
template <class T>
__device__ __forceinline__ long long stride(const dfield<T> &f, int d) {
  return d == 0 ? f.s0 : (d == 1 ? f.s1 : f.s2);
}

__device__ __forceinline__ bool rigid_edge(const geom &g, int d, int q) {
  return (q == 0 && g.bc[d][0] == MPDX_BC_RIGID) || (q == g.n[d] - 1 && g.bc[d][1] == MPDX_BC_RIGID);
}

// Where coordinate q along axis d (q in [-2, n+1]) takes its value from under
// the pressure halo fill (cyclic_2d.hpp:35-38 -> fill_halos_sclr; rigid_2d.hpp:
// 26-35, 134-143): the point qa itself, or 2 x (point qa) - (point qb).
__device__ __forceinline__ void pres_src(const geom &g, int d, int q, int &qa, int &qb) {
  const int n = g.n[d];
  qa = q; qb = -1;
  if (q >= 0 && q < n) return;
  const int side = q < 0 ? 0 : 1;
  const int kind = side == 0 ? g.bc[d][0] : g.bc[d][1];
  if (kind == MPDX_BC_CYCLIC) { qa = q < 0 ? q + n - 1 : q - (n - 1); return; }
  qa = side == 0 ? 0 : n - 1;
  qb = side == 0 ? -q : 2 * (n - 1) - q;
}

// A at coordinate q of the line through `base` along d (line element q at base + q * sd)
template <class T, class F>
__device__ __forceinline__ T aval(const F &A, const geom &g, int d, long long base, long long sd, int q) {
  int qa, qb;
  pres_src(g, d, q, qa, qb);
  T v = A(base + qa * sd);
  if (qb >= 0) v = T(2) * v - A(base + qb * sd);
  return v;
}

// grad_d A at interior coordinate q (nabla_formulae.hpp:18-41):
// (x(i+1) - x(i-1)) / dx / 2; halving is exact, so it is a multiplication by 0.5
template <class T, class F>
__device__ __forceinline__ T grad(const F &A, const geom &g, int d, long long base, long long sd, int q) {
  return mpdx::qdiv<T>(aval<T>(A, g, d, base, sd, q + 1) - aval<T>(A, g, d, base, sd, q - 1), g.dx<T>(d), g.rdx<T>(d)) * T(0.5);
}

struct no_u {};
template <class T>
struct vec_u {
  dfield<T> u[3];
};
template <class T> struct is_vec : std::false_type {};
template <class T> struct is_vec<vec_u<T>> : std::true_type {};

// lap_tmp[d] at interior coordinate q: grad, minus u (err_init), zero on a rigid wall (set_edges)
template <class T, class F, class U>
__device__ __forceinline__ T lt(const F &A, const U &u, const geom &g, int d, long long base, long long sd,
                                long long ubase, long long usd, int q) {
  if (rigid_edge(g, d, q)) return T(0);
  T v = grad<T>(A, g, d, base, sd, q);
  if constexpr (is_vec<U>::value) v -= T(u.u[d].o[ubase + q * usd]);
  if (g.norm) v = v / g.dn<T>(d, base + q * sd);
  return v;
}
// lap_tmp[d] at coordinate q in [-1, n] (its own pressure halo fill)
template <class T, class F, class U>
__device__ __forceinline__ T LT(const F &A, const U &u, const geom &g, int d, long long base, long long sd,
                                long long ubase, long long usd, int q) {
  int qa, qb;
  pres_src(g, d, q, qa, qb);
  T v = lt<T>(A, u, g, d, base, sd, ubase, usd, qa);
  if (qb >= 0) v = T(2) * v - lt<T>(A, u, g, d, base, sd, ubase, usd, qb);
  return v;
}
// lap(A) at interior point (i, j, k): div(grad A [- u]) (mpdata_rhs_vip_prs_common.hpp:49-84,
// nabla_formulae.hpp:184-215).  `lay` is the layout shared by A's fields.
template <class T, class F, class U>
__device__ __forceinline__ T lap(const F &A, const dfield<T> &lay, const U &u, const geom &g, int i, int j, int k) {
  const int c[3] = {i, j, k};
  const long long o = off3(lay, i, j, k);
  T r = T(0);
  // Points whose whole stencil (c - 2 .. c + 2 along every axis) is interior: no halo
  // rule and no wall applies, so LT(c +- 1) = grad(c +- 1) [- u(c +- 1)] and aval is a
  // plain read.  Same operations in the same order as the general form below.
  bool inner = true;
#pragma unroll
  for (int d = 0; d < 3; ++d)
    if (d < g.nd) inner = inner && c[d] >= 2 && c[d] <= g.n[d] - 3;
  if (inner) {
    const T a0 = A(o);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (d >= g.nd) break;
      const long long sd = stride(lay, d);
      const T dx = g.dx<T>(d), rdx = g.rdx<T>(d);
      T gp = mpdx::qdiv<T>(A(o + 2 * sd) - a0, dx, rdx) * T(0.5);
      T gm = mpdx::qdiv<T>(a0 - A(o - 2 * sd), dx, rdx) * T(0.5);
      if constexpr (is_vec<U>::value) {
        const long long usd = stride(u.u[d], d), uo = off3(u.u[d], i, j, k);
        gp -= T(u.u[d].o[uo + usd]);
        gm -= T(u.u[d].o[uo - usd]);
      }
      if (g.norm) {
        gp = gp / g.dn<T>(d, o + sd);
        gm = gm / g.dn<T>(d, o - sd);
      }
      const T term = mpdx::qdiv<T>(gp - gm, dx, rdx) * T(0.5);
      r = d == 0 ? term : r + term;
    }
    return r;
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d >= g.nd) break;
    const long long sd = stride(lay, d);
    const long long base = o - c[d] * sd;
    long long ubase = 0, usd = 0;
    if constexpr (is_vec<U>::value) {
      usd = stride(u.u[d], d);
      ubase = off3(u.u[d], i, j, k) - c[d] * usd;
    }
    const T term = mpdx::qdiv<T>(LT<T>(A, u, g, d, base, sd, ubase, usd, c[d] + 1) - LT<T>(A, u, g, d, base, sd, ubase, usd, c[d] - 1),
                                 g.dx<T>(d), g.rdx<T>(d)) * T(0.5);
    r = d == 0 ? term : r + term;
  }
  return r;
}

// ---------------------------------------------------------------------------
// compensated reductions (TwoSum; dd_add is commutative bit for bit)
struct dd {
  double s, c;
};
__device__ __forceinline__ dd dd_add(dd a, dd b) {
  const double s = a.s + b.s;
  const double bp = s - a.s;
  const double e = (a.s - (s - bp)) + (b.s - bp);
  return {s, (a.c + b.c) + e};
}

__device__ __forceinline__ dd warp_sum(dd v) {
  for (int off = 16; off > 0; off >>= 1) {
    dd o{__shfl_down_sync(0xffffffffu, v.s, off), __shfl_down_sync(0xffffffffu, v.c, off)};
    v = dd_add(v, o);
  }
  return v;
}
__device__ __forceinline__ void warp_mm(double &mx, double &mn) {
  for (int off = 16; off > 0; off >>= 1) {
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, off));
  }
}

// Reduces ns sums (and max/min when mm) over the grid.  Returns true in the last
// block to arrive; there tot[] and mx/mn hold the grid results in every thread.
// Fixed tree: per-thread strided sums, warp shuffle tree, warps in order, blocks
// in order -> the same bits on every run.
template <int NS, bool MM>
__device__ __forceinline__ bool grid_reduce(dd (&acc)[NS], double &mx, double &mn, double *part, unsigned *arrive) {
  constexpr int ns = NS;
  constexpr bool mm = MM;
  __shared__ dd wsum[kRedThreads / 32];
  __shared__ double wmx[kRedThreads / 32], wmn[kRedThreads / 32];
  __shared__ bool last;
  __shared__ dd bsum[kRedSlots];
  __shared__ double bmx, bmn;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x, nthr = blockDim.x * blockDim.y;
  const int lane = tid & 31, w = tid >> 5, nw = nthr >> 5;
  double *mine = part + size_t(blockIdx.x) * kRedSlots * 2;
#pragma unroll
  for (int s = 0; s < ns; ++s) {
    const dd v = warp_sum(acc[s]);
    if (lane == 0) wsum[w] = v;
    __syncthreads();
    if (tid == 0) {
      dd t = wsum[0];
      for (int q = 1; q < nw; ++q) t = dd_add(t, wsum[q]);
      mine[2 * s] = t.s;
      mine[2 * s + 1] = t.c;
    }
    __syncthreads();
  }
  if constexpr (mm) {
    warp_mm(mx, mn);
    if (lane == 0) { wmx[w] = mx; wmn[w] = mn; }
    __syncthreads();
    if (tid == 0) {
      double a = wmx[0], b = wmn[0];
      for (int q = 1; q < nw; ++q) { a = fmax(a, wmx[q]); b = fmin(b, wmn[q]); }
      mine[2 * (kRedSlots - 1)] = a;
      mine[2 * (kRedSlots - 1) + 1] = b;
    }
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) last = atomicAdd(arrive, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return false;
  __threadfence();
#pragma unroll
  for (int s = 0; s < ns; ++s) {
    dd v{0.0, 0.0};
    for (int b = tid; b < int(gridDim.x); b += nthr) {
      const double *p = part + size_t(b) * kRedSlots * 2 + 2 * s;
      v = dd_add(v, dd{__ldcg(p), __ldcg(p + 1)});
    }
    v = warp_sum(v);
    if (lane == 0) wsum[w] = v;
    __syncthreads();
    if (tid == 0) {
      dd t = wsum[0];
      for (int q = 1; q < nw; ++q) t = dd_add(t, wsum[q]);
      bsum[s] = t;
    }
    __syncthreads();
  }
  if constexpr (mm) {
    double a = -DBL_MAX, b = DBL_MAX;
    for (int q = tid; q < int(gridDim.x); q += nthr) {
      const double *p = part + size_t(q) * kRedSlots * 2 + 2 * (kRedSlots - 1);
      a = fmax(a, __ldcg(p));
      b = fmin(b, __ldcg(p + 1));
    }
    warp_mm(a, b);
    if (lane == 0) { wmx[w] = a; wmn[w] = b; }
    __syncthreads();
    if (tid == 0) {
      double x = wmx[0], y = wmn[0];
      for (int q = 1; q < nw; ++q) { x = fmax(x, wmx[q]); y = fmin(y, wmn[q]); }
      bmx = x; bmn = y;
    }
    __syncthreads();
    mx = bmx; mn = bmn;
  }
#pragma unroll
  for (int s = 0; s < ns; ++s) acc[s] = bsum[s];
  if (tid == 0) *arrive = 0u;
  return true;
}

__device__ __forceinline__ double ddv(dd a) { return a.s + a.c; }

// ---------------------------------------------------------------------------
// GCR kernels

template <class T>
__global__ void k_gcr_reset(gcr_dev<T> *dv) {
  dv->converged = 0; dv->done = 0; dv->stuck = 0; dv->cur = 0; dv->iters = 0; dv->arrive = 0u; dv->bad = 0;
}
// after the learned corrections: plain GCR continues from the current iterate
template <class T>
__global__ void k_gcr_clear_bad(gcr_dev<T> *dv) { dv->bad = 0; }
template <class T>
__global__ void k_gcr_reset_conv(gcr_dev<T> *dv) { dv->converged = 0; }

// err = lap(Phi) with err_init (u = the velocity being projected)
template <class P, class T>
__global__ void __launch_bounds__(kRedThreads, 4) k_err_init(geom g, dfield<P> phi, vec_u<T> u, dfield<P> err) {
  for_interior(g, [&](int i, int j, int k) {
    err(i, j, k) = lap<P>(fld<P>{phi.o}, phi, u, g, i, j, k);
    });
}

// loop_init: p_0 = err, lap_p_0 = lap(p_0); sums of the first beta
template <class T>
__global__ void __launch_bounds__(kRedThreads, 4) k_gcr_init(geom g, dfield<T> err, dfield<T> p0, dfield<T> lp0, gcr_dev<T> *dv, double *part) {
  dd acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  for_interior(g, [&](int i, int j, int k) {
    const T e = err(i, j, k);
    const T l = lap<T>(fld<T>{err.o}, err, no_u{}, g, i, j, k);
    p0(i, j, k) = e;
    lp0(i, j, k) = l;
    acc[0] = dd_add(acc[0], dd{double(T(l * l)), 0.0});
    acc[1] = dd_add(acc[1], dd{double(T(e * l)), 0.0});
    });
  double mx = 0, mn = 0;
  if (grid_reduce<2, false>(acc, mx, mn, part, &dv->arrive) && threadIdx.x == 0 && threadIdx.y == 0) {
    dv->pend_den = T(ddv(acc[0]));
    dv->pend_num = T(ddv(acc[1]));
  }
}

template <class T>
struct dirs {
  dfield<T> p[kGcrMaxK], lp[kGcrMaxK];
};

// inner step v = NV - 1, first half (mpdata_rhs_vip_prs_gcrk.hpp:43-64)
template <class T, int NV>
__global__ void __launch_bounds__(kRedThreads, 4) k_gcr_update(geom g, T err_tol, dfield<T> err0, dfield<T> err1,
                                                               dfield<T> lap_err, dirs<T> D, gcr_dev<T> *dv, double *part) {
  constexpr int v = NV - 1;
  if (dv->done) return;
  const int cur = dv->cur;
  const dfield<T> ea = cur ? err1 : err0, eb = cur ? err0 : err1;
  const T den = dv->pend_den;
  const T b = den != T(0) ? -dv->pend_num / den : dv->beta;  // beta keeps its value when tmp_den is 0
  if (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) { dv->tmp_den[v] = den; dv->beta = b; }
  const dfield<T> lpv = D.lp[v];
  dfield<T> lps[NV];
#pragma unroll
  for (int l = 0; l < NV; ++l) lps[l] = D.lp[l];
  const fld_axpy<T> enew{ea.o, lpv.o, b};
  dd acc[NV];
#pragma unroll
  for (int l = 0; l < NV; ++l) acc[l] = dd{0.0, 0.0};
  double mx = -DBL_MAX, mn = DBL_MAX;
  for_interior(g, [&](int i, int j, int k) {
    const T e = enew(off3(ea, i, j, k));
    eb(i, j, k) = e;
    mx = fmax(mx, double(e));
    mn = fmin(mn, double(e));
    const T le = lap<T>(enew, ea, no_u{}, g, i, j, k);
    lap_err(i, j, k) = le;
#pragma unroll
    for (int l = 0; l < NV; ++l) acc[l] = dd_add(acc[l], dd{double(T(le * lps[l](i, j, k))), 0.0});
  });
  if (grid_reduce<NV, true>(acc, mx, mn, part, &dv->arrive) && threadIdx.x == 0 && threadIdx.y == 0) {
    const T amx = fabs(T(mx)), amn = fabs(T(mn));
    const T error = amx < amn ? amn : amx;  // std::max(|max|, |min|)
    dv->residual = double(error);
    if (error <= err_tol) dv->converged = 1;
#pragma unroll
    for (int l = 0; l < NV; ++l) {
      const T dl = l == v ? den : dv->tmp_den[l];
      if (dl != T(0)) dv->alpha[l] = -T(ddv(acc[l])) / dl;
    }
  }
}

// 3D form of k_gcr_update, in two phases within one launch (one reduction).
// Interior: the points whose whole stencil lies inside the grid (every coordinate
// in [2, n-3]).  A block owns a tile of kTJ x kTK (j, k) columns of the interior and
// marches along i over a chunk of planes; the updated error of plane i+2, on the
// tile plus a halo of 2, goes to a ring of 4 shared planes, so the Laplacian reads
// its j and k neighbours from the plane of i, its i+2 neighbour from the plane of
// i+2 and its i-2 neighbour from the thread's registers.  Shell: the remaining
// points (within 2 of a face), with the general lap, one point per thread.  The
// arithmetic of every point is k_gcr_update's (same operations in the same order).
constexpr int kTJ = 8, kTK = 32, kPJ = kTJ + 4, kPK = kTK + 4, kGcrChunk = 32, kSteps = 2;
static_assert(kTJ * kTK == kRedThreads, "one tile column per thread");
template <class T, int NV>
__global__ void __launch_bounds__(kRedThreads, NV == 1 ? 4 : 2) k_gcr_update3(geom g, T err_tol, dfield<T> err0,
                                                                dfield<T> err1, dfield<T> lap_err, dirs<T> D,
                                                                gcr_dev<T> *dv, double *part, int chunk) {
  constexpr int v = NV - 1;
  if (dv->done) return;
  const int cur = dv->cur;
  const dfield<T> ea = cur ? err1 : err0, eb = cur ? err0 : err1;
  const T den = dv->pend_den;
  const T b = den != T(0) ? -dv->pend_num / den : dv->beta;  // beta keeps its value when tmp_den is 0
  if (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) { dv->tmp_den[v] = den; dv->beta = b; }
  const dfield<T> lpv = D.lp[v];
  const fld_axpy<T> enew{ea.o, lpv.o, b};
  dd acc[NV];
#pragma unroll
  for (int l = 0; l < NV; ++l) acc[l] = dd{0.0, 0.0};
  double mx = -DBL_MAX, mn = DBL_MAX;
  // every pressure-type field has the same layout: one linear offset addresses a
  // point in all of them
  T *const ebo = eb.o, *const leo = lap_err.o;
  const T *const eao = ea.o, *const lpvo = lpv.o;
  const T *lpo[NV];
#pragma unroll
  for (int l = 0; l < NV; ++l) lpo[l] = D.lp[l].o;
  const long long s0 = ea.s0;
  // per-point outputs (mpdata_rhs_vip_prs_gcrk.hpp:43-64); Phi += beta p_v is
  // applied by k_gcr_direction, which reads p_v anyway
  auto finish = [&](long long o, T e, T le, const T *clp) {
    ebo[o] = e;
    mx = fmax(mx, double(e));
    mn = fmin(mn, double(e));
    leo[o] = le;
#pragma unroll
    for (int l = 0; l < NV; ++l) acc[l] = dd_add(acc[l], dd{double(T(le * clp[l])), 0.0});
  };

  const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
  // ---- interior: column march ----
  __shared__ T pl[8][kPJ][kPK];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTK + tx;
  const int m0 = n0 - 4, m1 = n1 - 4, m2 = n2 - 4;  // interior extents
  const int nkt = m2 > 0 ? (m2 + kTK - 1) / kTK : 0, njt = m1 > 0 ? (m1 + kTJ - 1) / kTJ : 0;
  const int nch = m0 > 0 ? (m0 + chunk - 1) / chunk : 0;
  const long long n_items = (long long)nkt * njt * nch;
  constexpr int NQ = (kPJ * kPK + kRedThreads - 1) / kRedThreads;  // tile points per thread
  auto slot = [](int i) { return i & 7; };  // i & 7 is i mod 8
  for (long long item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int kt = int(item % nkt);
    const long long rest = item / nkt;
    const int jt = int(rest % njt), ch = int(rest / njt);
    const int j = 2 + jt * kTJ + ty, k = 2 + kt * kTK + tx;
    const int i0 = 2 + ch * chunk, i1 = min(i0 + chunk, n0 - 2);
    const bool own = j < n1 - 2 && k < n2 - 2;
    // this thread's tile points (with halo) and their offsets within a plane
    long long qo[NQ];
    bool qin[NQ];
#pragma unroll
    for (int u = 0; u < NQ; ++u) {
      const int q = tid + u * kRedThreads, pj = q / kPK, pk = q - pj * kPK;
      const int jj = jt * kTJ + pj, kk = kt * kTK + pk;  // = origin - 2 + offset, origin at 2
      qin[u] = q < kPJ * kPK && jj < n1 && kk < n2;
      qo[u] = qin[u] ? off3(ea, 0, jj, kk) : 0;
    }
    // err and lap_p of the tile points of kSteps planes, loaded a pass before they are used
    T xa[kSteps][NQ], xb[kSteps][NQ];
    auto load = [&](int i, int q0) {
      const long long io = (long long)i * s0;
      const bool iok = i < n0;
#pragma unroll
      for (int u = 0; u < NQ; ++u) {
        const bool ok = qin[u] && iok;
        xa[q0][u] = ok ? eao[io + qo[u]] : T(0);
        xb[q0][u] = ok ? lpvo[io + qo[u]] : T(0);
      }
    };
    auto store = [&](int i, int q0) {  // enew = err + beta lap_p (fld_axpy)
      T *P = &pl[slot(i)][0][0];
#pragma unroll
      for (int u = 0; u < NQ; ++u) {
        const int q = tid + u * kRedThreads;
        if (q < kPJ * kPK) P[q] = xa[q0][u] + b * xb[q0][u];
      }
    };
    __syncthreads();  // the previous item's reads are done
    for (int i = i0 - 2; i <= i0 + 1; ++i) { load(i, 0); store(i, 0); }
#pragma unroll
    for (int q0 = 0; q0 < kSteps; ++q0) load(i0 + 2 + q0, q0);
    __syncthreads();
    T cm2 = pl[slot(i0 - 2)][ty + 2][tx + 2], cm1 = pl[slot(i0 - 1)][ty + 2][tx + 2];
    const long long colo = own ? off3(ea, 0, j, k) : 0;
    T flp[kSteps][NV];
    auto load_own = [&](int i, int q0) {  // the own point's lap_p of every direction, a pass ahead
      if (own && i < i1) {
        const long long o = colo + i * s0;
#pragma unroll
        for (int l = 0; l < NV; ++l) flp[q0][l] = lpo[l][o];
      }
    };
#pragma unroll
    for (int q0 = 0; q0 < kSteps; ++q0) load_own(i0 + q0, q0);
    // kSteps planes per barrier: the ring of 8 shared planes holds the 4 planes a pass
    // reads (i .. i+kSteps+1) and the kSteps planes the next pass writes
    for (int i = i0; i < i1; i += kSteps) {
#pragma unroll
      for (int q0 = 0; q0 < kSteps; ++q0) store(i + 2 + q0, q0);
#pragma unroll
      for (int q0 = 0; q0 < kSteps; ++q0) load(i + 2 + kSteps + q0, q0);
      T clp[kSteps][NV];
#pragma unroll
      for (int q0 = 0; q0 < kSteps; ++q0) {
#pragma unroll
        for (int l = 0; l < NV; ++l) clp[q0][l] = flp[q0][l];
      }
#pragma unroll
      for (int q0 = 0; q0 < kSteps; ++q0) load_own(i + kSteps + q0, q0);
      __syncthreads();
#pragma unroll
      for (int q0 = 0; q0 < kSteps; ++q0) {
        const int ip = i + q0;
        const T c0 = pl[slot(ip)][ty + 2][tx + 2];
        if (own && ip < i1) {
          const T(*P)[kPK] = pl[slot(ip)];
          const T nb[3][2] = {{pl[slot(ip + 2)][ty + 2][tx + 2], cm2},
                              {P[ty + 4][tx + 2], P[ty][tx + 2]},
                              {P[ty + 2][tx + 4], P[ty + 2][tx]}};
          T le = T(0);
#pragma unroll
          for (int d = 0; d < 3; ++d) {  // lap: grad(c+1) - grad(c-1), each a centred difference
            const T dx = g.dx<T>(d), rdx = g.rdx<T>(d);
            const T gp = mpdx::qdiv<T>(nb[d][0] - c0, dx, rdx) * T(0.5);
            const T gm = mpdx::qdiv<T>(c0 - nb[d][1], dx, rdx) * T(0.5);
            const T term = mpdx::qdiv<T>(gp - gm, dx, rdx) * T(0.5);
            le = d == 0 ? term : le + term;
          }
          finish(colo + ip * s0, c0, le, clp[q0]);
        }
        cm2 = cm1;
        cm1 = c0;
      }
    }
  }
  // ---- shell: points within 2 of a face ----
  // i-slabs {0, 1, n0-2, n0-1} x all (j, k); then j-slabs inside them; then k-slabs
  const int ci0 = n0 < 4 ? n0 : 4, ii = n0 - ci0;                // i layers in the shell, interior i count
  const int cj0 = n1 < 4 ? n1 : 4, jj = n1 - cj0, ck0 = n2 < 4 ? n2 : 4;
  const long long sa = (long long)ci0 * n1 * n2, sb = (long long)ii * cj0 * n2, sc = (long long)ii * jj * ck0;
  auto shell_coord = [](int q, int c, int n) { return q < c / 2 ? q : n - c + q; };  // q-th shell layer
  const long long nthr = (long long)gridDim.x * kRedThreads;
  for (long long q = (long long)blockIdx.x * kRedThreads + tid; q < sa + sb + sc; q += nthr) {
    int i, j, k;
    if (q < sa) {
      k = int(q % n2); const long long r = q / n2; j = int(r % n1); i = shell_coord(int(r / n1), ci0, n0);
    } else if (q < sa + sb) {
      const long long w = q - sa;
      k = int(w % n2); const long long r = w / n2; j = shell_coord(int(r % cj0), cj0, n1); i = 2 + int(r / cj0);
    } else {
      const long long w = q - sa - sb;
      k = shell_coord(int(w % ck0), ck0, n2); const long long r = w / ck0; j = 2 + int(r % jj); i = 2 + int(r / jj);
    }
    const long long o = off3(ea, i, j, k);
    const T e = enew(o);
    const T le = lap<T>(enew, ea, no_u{}, g, i, j, k);
    T clp[NV];
#pragma unroll
    for (int l = 0; l < NV; ++l) clp[l] = lpo[l][o];
    finish(o, e, le, clp);
  }
  if (grid_reduce<NV, true>(acc, mx, mn, part, &dv->arrive) && threadIdx.x == 0 && threadIdx.y == 0) {
    const T amx = fabs(T(mx)), amn = fabs(T(mn));
    const T error = amx < amn ? amn : amx;  // std::max(|max|, |min|)
    dv->residual = double(error);
    if (error <= err_tol) dv->converged = 1;
#pragma unroll
    for (int l = 0; l < NV; ++l) {
      const T dl = l == v ? den : dv->tmp_den[l];
      if (dl != T(0)) dv->alpha[l] = -T(ddv(acc[l])) / dl;
    }
  }
}

// inner step v = NV - 1, second half: next search direction (mpdata_rhs_vip_prs_gcrk.hpp:66-92)
template <class T, int NV>
__global__ void __launch_bounds__(kRedThreads, 3) k_gcr_direction(geom g, int kk, dfield<T> phi, dfield<T> err0,
                                                                  dfield<T> err1, dfield<T> lap_err, dirs<T> D,
                                                                  gcr_dev<T> *dv, double *part) {
  constexpr int v = NV - 1;
  if (dv->done) return;
  const int cur = dv->cur;
  const T b = dv->beta;  // this inner step's beta, set by k_gcr_update
  const dfield<T> e = cur ? err0 : err1;  // the error written by k_gcr_update
  T a[NV];
  dfield<T> ps[NV], lps[NV];
#pragma unroll
  for (int l = 0; l < NV; ++l) { a[l] = dv->alpha[l]; ps[l] = D.p[l]; lps[l] = D.lp[l]; }
  const bool restart = v == kk - 1;
  const dfield<T> pd = restart ? D.p[0] : D.p[NV < kGcrMaxK ? NV : 0], lpd = restart ? D.lp[0] : D.lp[NV < kGcrMaxK ? NV : 0];
  dd acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  // every pressure-type field has the same layout: one linear offset per point
  const T *const eo = e.o, *const leo = lap_err.o;
  T *const pdo = pd.o, *const lpdo = lpd.o, *const phio = phi.o;
  const T *po[NV], *lpo[NV];
#pragma unroll
  for (int l = 0; l < NV; ++l) { po[l] = ps[l].o; lpo[l] = lps[l].o; }
  // U points per thread and pass, all loads issued before the arithmetic (memory-level parallelism)
  constexpr int U = NV == 1 ? 4 : (NV <= 4 ? 2 : 1);
  for (int row = blockIdx.x * blockDim.y + threadIdx.y; row < g.nrows; row += gridDim.x * blockDim.y) {
    int i = row, j = 0;
    if (g.nd == 3) { i = row / g.n[1]; j = row - i * g.n[1]; }
    if constexpr (std::is_same<T, double>::value && NV == 1) {
      // one search direction in FP64 (cr, and the first inner step of gcrk): pairs of
      // points with 16-byte loads and stores (a row starts on a 128-byte boundary);
      // both branches of the reference compute p = err + alpha p, lap_p = lap_err + alpha lap_p
      const long long ob = g.nd == 3 ? off3(e, i, j, 0) : off3(e, i, 0, 0);
      const T a0 = a[0];
      for (int f0 = 2 * threadIdx.x; f0 < g.nf; f0 += 4 * blockDim.x) {
        double2 E[2], L[2], H[2], PV[2], LV[2];
        int nv[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int f = f0 + 2 * u * blockDim.x;
          nv[u] = f + 1 < g.nf ? 2 : (f < g.nf ? 1 : 0);
          const long long q = ob + f;
          if (nv[u] == 2) {
            E[u] = *reinterpret_cast<const double2 *>(eo + q);
            L[u] = *reinterpret_cast<const double2 *>(leo + q);
            H[u] = *reinterpret_cast<const double2 *>(phio + q);
            PV[u] = *reinterpret_cast<const double2 *>(po[0] + q);
            LV[u] = *reinterpret_cast<const double2 *>(lpo[0] + q);
          } else if (nv[u] == 1) {
            E[u] = make_double2(eo[q], 0.0); L[u] = make_double2(leo[q], 0.0); H[u] = make_double2(phio[q], 0.0);
            PV[u] = make_double2(po[0][q], 0.0); LV[u] = make_double2(lpo[0][q], 0.0);
          }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          if (nv[u] == 0) continue;
          const long long q = ob + f0 + 2 * u * blockDim.x;
          const double ph0 = H[u].x + b * PV[u].x, ph1 = H[u].y + b * PV[u].y;  // Phi += beta p_v
          const double pn0 = E[u].x + a0 * PV[u].x, pn1 = E[u].y + a0 * PV[u].y;
          const double ln0 = L[u].x + a0 * LV[u].x, ln1 = L[u].y + a0 * LV[u].y;
          acc[0] = dd_add(acc[0], dd{ln0 * ln0, 0.0});
          acc[1] = dd_add(acc[1], dd{E[u].x * ln0, 0.0});
          if (nv[u] == 2) {
            *reinterpret_cast<double2 *>(phio + q) = make_double2(ph0, ph1);
            *reinterpret_cast<double2 *>(pdo + q) = make_double2(pn0, pn1);
            *reinterpret_cast<double2 *>(lpdo + q) = make_double2(ln0, ln1);
            acc[0] = dd_add(acc[0], dd{ln1 * ln1, 0.0});
            acc[1] = dd_add(acc[1], dd{E[u].y * ln1, 0.0});
          } else {
            phio[q] = ph0; pdo[q] = pn0; lpdo[q] = ln0;
          }
        }
      }
    } else {
    for (int f0 = threadIdx.x; f0 < g.nf; f0 += U * blockDim.x) {
      long long o[U];
      bool ok[U];
      T ev[U], le[U], ph[U], pv[U][NV], lv[U][NV];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int f = f0 + u * blockDim.x;
        ok[u] = f < g.nf;
        o[u] = ok[u] ? (g.nd == 3 ? off3(e, i, j, f) : off3(e, i, f, 0)) : 0;
        ev[u] = ok[u] ? eo[o[u]] : T(0);
        le[u] = ok[u] ? leo[o[u]] : T(0);
        ph[u] = ok[u] ? phio[o[u]] : T(0);
#pragma unroll
        for (int l = 0; l < NV; ++l) {
          pv[u][l] = ok[u] ? po[l][o[u]] : T(0);
          lv[u][l] = ok[u] ? lpo[l][o[u]] : T(0);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (!ok[u]) continue;
        phio[o[u]] = ph[u] + b * pv[u][v];  // Phi += beta p_v (mpdata_rhs_vip_prs_gcrk.hpp:51)
        T pn, ln;
        if (!restart) {
          pn = ev[u];
          ln = le[u];
#pragma unroll
          for (int l = 0; l < NV; ++l) {
            pn = pn + a[l] * pv[u][l];
            ln = ln + a[l] * lv[u][l];
          }
        } else {
          pn = ev[u] + a[0] * pv[u][0];
          ln = le[u] + a[0] * lv[u][0];
#pragma unroll
          for (int l = 1; l < NV; ++l) {
            pn = pn + a[l] * pv[u][l];
            ln = ln + a[l] * lv[u][l];
          }
        }
        pdo[o[u]] = pn;
        lpdo[o[u]] = ln;
        acc[0] = dd_add(acc[0], dd{double(T(ln * ln)), 0.0});
        acc[1] = dd_add(acc[1], dd{double(T(ev[u] * ln)), 0.0});
      }
    }
    }
  }
  double mx = 0, mn = 0;
  if (grid_reduce<2, false>(acc, mx, mn, part, &dv->arrive) && threadIdx.x == 0 && threadIdx.y == 0) {
    dv->pend_den = T(ddv(acc[0]));
    dv->pend_num = T(ddv(acc[1]));
    dv->cur = 1 - cur;
    if (restart) {  // end of one loop body (mpdata_rhs_vip_prs_common.hpp:111-125)
      dv->iters += 1;
      if (dv->converged) dv->done = 1;
      if (dv->iters > 10000) { dv->stuck = 1; dv->done = 1; }
    }
  }
}

// one inner step of GCR(k), NV = v + 1 known at compile time
template <class T, int NV>
void launch_inner(unsigned G, dim3 blk, cudaStream_t s, const geom &g, int kk, T err_tol, dfield<T> phi, dfield<T> e0,
                  dfield<T> e1, dfield<T> le, const dirs<T> &D, gcr_dev<T> *dv, double *part) {
  if (g.nd == 3 && !g.norm) k_gcr_update3<T, NV><<<G, blk, 0, s>>>(g, err_tol, e0, e1, le, D, dv, part, kGcrChunk);
  else k_gcr_update<T, NV><<<G, blk, 0, s>>>(g, err_tol, e0, e1, le, D, dv, part);
  k_gcr_direction<T, NV><<<G, blk, 0, s>>>(g, kk, phi, e0, e1, le, D, dv, part);
}
template <class T>
void launch_inner(int v, unsigned G, dim3 blk, cudaStream_t s, const geom &g, int kk, T err_tol, dfield<T> phi,
                  dfield<T> e0, dfield<T> e1, dfield<T> le, const dirs<T> &D, gcr_dev<T> *dv, double *part) {
  switch (v + 1) {
    case 1: launch_inner<T, 1>(G, blk, s, g, kk, err_tol, phi, e0, e1, le, D, dv, part); break;
    case 2: launch_inner<T, 2>(G, blk, s, g, kk, err_tol, phi, e0, e1, le, D, dv, part); break;
    case 3: launch_inner<T, 3>(G, blk, s, g, kk, err_tol, phi, e0, e1, le, D, dv, part); break;
    case 4: launch_inner<T, 4>(G, blk, s, g, kk, err_tol, phi, e0, e1, le, D, dv, part); break;
    case 5: launch_inner<T, 5>(G, blk, s, g, kk, err_tol, phi, e0, e1, le, D, dv, part); break;
    case 6: launch_inner<T, 6>(G, blk, s, g, kk, err_tol, phi, e0, e1, le, D, dv, part); break;
    case 7: launch_inner<T, 7>(G, blk, s, g, kk, err_tol, phi, e0, e1, le, D, dv, part); break;
    default: launch_inner<T, 8>(G, blk, s, g, kk, err_tol, phi, e0, e1, le, D, dv, part); break;
  }
}

// ---------------------------------------------------------------------------
// Learned corrections before plain GCR: q = M(err) from the network, a step along
// q, and err updated with the exact lap of q, so the stopping test of the plain
// iterations that follow is the reference's.  The error is updated in place (no
// stencil reads it in the same kernel).

// q(n-1) = q(0) along every cyclic axis (in axis order, as a halo fill would):
// the network pads a cyclic axis with period n, while point n-1 of the
// reference's cyclic convention duplicates point 0; a correction without the
// duplicate would make Phi, and the projected velocity, differ across the seam
template <class T>
__global__ void k_seam_dup(geom g, dfield<T> q, int d) {
  for_interior(g, [&](int i, int j, int k) {
    const int c[3] = {i, j, k};
    if (c[d] != g.n[d] - 1) return;
    const long long o = off3(q, i, j, k);
    q.o[o] = q.o[o - (long long)(g.n[d] - 1) * stride(q, d)];
  });
}

// A learned correction: q = M(err) (written into p0 by the network), lap_q =
// lap(q), and the sums of the step length that minimises the error in the energy
// norm of the operator (the norm the network is trained in):
// beta = -<err, q> / <q, lap q>  (err = lap(Phi) - rhs = lap(Phi - Phi*))
template <class T>
__global__ void __launch_bounds__(kRedThreads, 4) k_gcr_init_pc(geom g, dfield<T> err, dfield<T> p0, dfield<T> lp0,
                                                                gcr_dev<T> *dv, double *part) {
  if (dv->done || dv->bad || dv->converged) return;
  dd acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  for_interior(g, [&](int i, int j, int k) {
    const T q = p0(i, j, k);
    const T l = lap<T>(fld<T>{p0.o}, p0, no_u{}, g, i, j, k);
    lp0(i, j, k) = l;
    acc[0] = dd_add(acc[0], dd{double(T(q * l)), 0.0});
    acc[1] = dd_add(acc[1], dd{double(T(err(i, j, k) * q)), 0.0});
  });
  double mx = 0, mn = 0;
  if (grid_reduce<2, false>(acc, mx, mn, part, &dv->arrive) && threadIdx.x == 0 && threadIdx.y == 0) {
    dv->pend_den = T(ddv(acc[0]));
    dv->pend_num = T(ddv(acc[1]));
  }
}

// step v = NV - 1: Phi += beta p_v, err += beta lap_p_v, convergence test
template <class T, int NV>
__global__ void __launch_bounds__(kRedThreads, 4) k_gcr_update_pc(geom g, T err_tol, dfield<T> phi, dfield<T> err,
                                                                  dirs<T> D, gcr_dev<T> *dv, double *part) {
  constexpr int v = NV - 1;
  if (dv->done || dv->bad || dv->converged) return;
  const T den = dv->pend_den;
  const T b = den != T(0) ? -dv->pend_num / den : dv->beta;
  // a direction from the network whose sums are not finite (an overflowing or NaN
  // output) must not touch Phi or err: every block sees the same sums and returns,
  // and the host continues with plain GCR from the iterate as it stands
  // (a correction along q needs <q, lap q> < 0: lap is negative on every direction
  // it does not annihilate)
  if (!isfinite(double(den)) || !isfinite(double(b)) || !(den < T(0))) {
    if (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) dv->bad = 1;
    return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) { dv->tmp_den[v] = den; dv->beta = b; }
  const dfield<T> pv = D.p[v], lpv = D.lp[v];
  dd acc[1] = {{0.0, 0.0}};
  double mx = -DBL_MAX, mn = DBL_MAX;
  for_interior(g, [&](int i, int j, int k) {
    phi(i, j, k) = phi(i, j, k) + b * pv(i, j, k);
    const T e = err(i, j, k) + b * lpv(i, j, k);
    err(i, j, k) = e;
    mx = fmax(mx, double(e));
    mn = fmin(mn, double(e));
  });
  if (grid_reduce<1, true>(acc, mx, mn, part, &dv->arrive) && threadIdx.x == 0 && threadIdx.y == 0) {
    const T amx = fabs(T(mx)), amn = fabs(T(mn));
    const T error = amx < amn ? amn : amx;
    dv->residual = double(error);
    if (error <= err_tol) dv->converged = 1;
  }
}

template <class T, int NV>
void launch_pc_update(unsigned G, dim3 blk, cudaStream_t s, const geom &g, T err_tol, dfield<T> phi, dfield<T> err,
                      const dirs<T> &D, gcr_dev<T> *dv, double *part) {
  k_gcr_update_pc<T, NV><<<G, blk, 0, s>>>(g, err_tol, phi, err, D, dv, part);
}
#define MPDX_NV_SWITCH(v, CALL)                     \
  switch ((v) + 1) {                                \
    case 1: CALL(1); break;                         \
    case 2: CALL(2); break;                         \
    case 3: CALL(3); break;                         \
    case 4: CALL(4); break;                         \
    case 5: CALL(5); break;                         \
    case 6: CALL(6); break;                         \
    case 7: CALL(7); break;                         \
    default: CALL(8); break;                        \
  }

// training pairs: a field's interior as a compact FP32 array, or the difference of two fields
template <class T>
__global__ void k_to_compact(geom g, dfield<T> a, dfield<T> b, float *out) {
  for_interior(g, [&](int i, int j, int k) {
    const long long v = ((long long)i * g.n[1] + j) * g.n[2] + k;
    out[v] = b.o ? float(a(i, j, k) - b(i, j, k)) : float(a(i, j, k));
  });
}
template <class T>
__global__ void k_copy_field(geom g, dfield<T> src, dfield<T> dst) {
  for_interior(g, [&](int i, int j, int k) { dst(i, j, k) = src(i, j, k); });
}
// e = c q - t of the training loss
__global__ void k_sub(const float *a, float ca, const float *b, long long n, float *o) {  // o = ca * a - b
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) o[q] = ca * a[q] - b[q];
}
__global__ void k_sumsq(const float *x, long long n, double *out) {
  double sq = 0.0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    sq += double(x[q]) * double(x[q]);
  for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, sq);
}
// r / rms(r), t / rms(r) with rms from the sum of squares in *ss
__global__ void k_scale_rms(const float *r, const float *t, long long n, const double *ss, float *ro, float *to) {
  const double rms = sqrt(*ss / double(n));
  const float inv = rms > 0.0 ? float(1.0 / rms) : 1.f;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    ro[q] = r[q] * inv;
    to[q] = t[q] * inv;
  }
}

// centred gradient of a compact FP32 array along axis d at point c (the pressure
// solve's lap_tmp: (x(c+1) - x(c-1)) / 2 dx, neighbours under the halo rule, zero
// on a rigid wall)
__device__ __forceinline__ float grad_c(const geom &g, const dfield<float> &lay, const float *x, int d, const int *c) {
  if (rigid_edge(g, d, c[d])) return 0.f;
  const long long o = off3(lay, c[0], c[1], c[2]), sd = stride(lay, d), base = o - c[d] * sd;
  const fld<float> A{x};
  return (aval<float>(A, g, d, base, sd, c[d] + 1) - aval<float>(A, g, d, base, sd, c[d] - 1)) * (0.5f * g.rdxf[d]);
}
// gd[d] = G_d x for each axis (where gd[d] is not null), *sum += sum_d |G_d x|^2
__global__ void __launch_bounds__(kRedThreads, 4) k_grad_sq(geom g, const float *x, float *g0, float *g1, float *g2,
                                                           double *sum) {
  const dfield<float> lay{const_cast<float *>(x), (long long)g.n[1] * g.n[2], g.n[2], g.nd == 3 ? 1 : 0};
  float *gd[3] = {g0, g1, g2};
  double sq = 0.0;
  for_interior(g, [&](int i, int j, int k) {
    const int c[3] = {i, j, k};
    const long long o = off3(lay, i, j, k);
    for (int d = 0; d < g.nd; ++d) {
      const float v = grad_c(g, lay, x, d, c);
      if (gd[d]) gd[d][o] = v;
      sq += double(v) * double(v);
    }
  });
  for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
  if (((threadIdx.y * blockDim.x + threadIdx.x) & 31) == 0) atomicAdd(sum, sq);
}
// out = f * sum_d G_d^T y_d, f = 2 c / (*den): the gradient of sum_d |G_d e|^2 / den
// with respect to q for e = c q - t.  G_d^T gathers the rows that read point m:
// cyclic (period n - 1): y(m-1) [m >= 1] + y(n-1) [m = 1] - y(m+1) [m <= n-2] - y(0) [m = n-2];
// rigid (rows 0 and n-1 zero): y(m-1) [1 <= m-1 <= n-2] - y(m+1) [1 <= m+1 <= n-2]
__global__ void __launch_bounds__(kRedThreads, 4) k_grad_adj(geom g, const float *y0, const float *y1, const float *y2,
                                                            const double *den, float c, float *out) {
  const dfield<float> lay{out, (long long)g.n[1] * g.n[2], g.n[2], g.nd == 3 ? 1 : 0};
  const float *yd[3] = {y0, y1, y2};
  const float f = *den > 0.0 ? float(2.0 * double(c) / *den) : 0.f;
  for_interior(g, [&](int i, int j, int k) {
    const int c3[3] = {i, j, k};
    const long long o = off3(lay, i, j, k);
    float acc = 0.f;
    for (int d = 0; d < g.nd; ++d) {
      const int m = c3[d], n = g.n[d];
      const long long sd = stride(lay, d), base = o - m * sd;
      const float *y = yd[d];
      float v = 0.f;
      if (g.bc[d][0] == MPDX_BC_CYCLIC) {
        if (m >= 1) v += y[base + (m - 1) * sd];
        if (m == 1) v += y[base + (n - 1) * sd];
        if (m <= n - 2) v -= y[base + (m + 1) * sd];
        if (m == n - 2) v -= y[base];
      } else {
        if (m - 1 >= 1 && m - 1 <= n - 2) v += y[base + (m - 1) * sd];
        if (m + 1 >= 1 && m + 1 <= n - 2) v -= y[base + (m + 1) * sd];
      }
      acc += v * (0.5f * g.rdxf[d]);
    }
    out[o] = f * acc;
  });
}


// ---------------------------------------------------------------------------
// pointwise stages

enum { APPLY_PROJECT = 0, APPLY_RHS = 1, APPLY_FINISH = 2 };

// grad Phi applied to the velocities: pressure_solver_apply + set_edges
// (PROJECT), vip_rhs -= grad Phi (RHS, hook_ante_loop), or pressure_solver_apply +
// normalize_vip (with g.norm) + set_edges + vip_rhs = (vip_rhs + u) / (dt / 2)
// (FINISH, vip_rhs_impl_fnlz)
template <class T, class P>
__global__ void __launch_bounds__(kRedThreads, 4) k_apply_grad(geom g, int mode, dfield<P> phi, vec_u<T> vel, vec_u<T> vr, T hdt) {
  for_interior(g, [&](int i, int j, int k) {
    const int c[3] = {i, j, k};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (d >= g.nd) break;
      const long long sd = stride(phi, d);
      const P gd = grad<P>(fld<P>{phi.o}, g, d, off3(phi, i, j, k) - c[d] * sd, sd, c[d]);
      if (mode == APPLY_RHS) {
        vr.u[d](i, j, k) = T(P(vr.u[d](i, j, k)) - gd);
        continue;
      }
      T v = T(P(vel.u[d](i, j, k)) - gd);
      if (mode == APPLY_FINISH && g.norm) v = v / T(g.dn<P>(d, off3(phi, i, j, k)));  // normalize_vip
      if (rigid_edge(g, d, c[d])) v = T(0);
      vel.u[d](i, j, k) = v;
      if (mode == APPLY_FINISH) {
        const T r = vr.u[d](i, j, k) + v;
        vr.u[d](i, j, k) = r / hdt;
      }
    }
    });
}

template <class T>
struct eqns {
  dfield<T> psi[4], rhs[4];
};

// extrp (mpdata_rhs_vip_common.hpp:120-153): stash = -beta stash + (1 + beta) u
template <class T>
__global__ void k_extrp(geom g, vec_u<T> stash, vec_u<T> vel, T b) {
  for_interior(g, [&](int i, int j, int k) {
    _Pragma("unroll") for (int d = 0; d < 3; ++d) if (d < g.nd) {
      T s = stash.u[d](i, j, k) * -b;
      s = s + (T(1) + b) * vel.u[d](i, j, k);
      stash.u[d](i, j, k) = s;
    }
    });
}

// intrp<d> (mpdata_rhs_vip.hpp:122-143): GC = dt / di * 0.5 * (u(i) + u(i+1)) over a box
template <class T>
__global__ void k_intrp(dfield<T> gc, dfield<T> src, int d, T c, int i0, int j0, int k0, int ni, int nj, int nk) {
  const long long tot = (long long)ni * nj * nk;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int k = k0 + int(q % nk);
    const long long r = q / nk;
    const int j = j0 + int(r % nj), i = i0 + int(r / nj);
    const T s1 = d == 0 ? src(i + 1, j, k) : (d == 1 ? src(i, j + 1, k) : src(i, j, k + 1));
    gc(i, j, k) = c * (src(i, j, k) + s1);
  }
}

// fields and constants of the forcings: theta environment, absorber, heat flux
// (boussinesq_common.hpp:20-60, boussinesq_impl.hpp), velocity absorber
// (mpdata_rhs_vip_common.hpp:182-256)
template <class T>
struct forcing {
  dfield<T> the, tabs, hflx, dthe, vabc;
  vec_u<T> relax;
  int impl, vab;  // impl_tht; vip_vab (MPDX_VAB_*)
  T grav, tref, dt;
};

// hook_ante_step: fill_stash, vip_rhs_expl_calc, apply_rhs(dt / 2), vip_rhs_apply
template <class T>
__global__ void k_ante_step(geom g, int ne, eqns<T> E, const int *vip, vec_u<T> stash, vec_u<T> vr, T dt2, T hdt,
                            forcing<T> F) {
  for_interior(g, [&](int i, int j, int k) {
    _Pragma("unroll") for (int d = 0; d < 3; ++d) if (d < g.nd) stash.u[d](i, j, k) = E.psi[vip[d]](i, j, k);
    if (F.vab == MPDX_VAB_EXPL)  // factor 2: vip_rhs_apply multiplies by dt / 2
      _Pragma("unroll") for (int d = 0; d < 3; ++d) if (d < g.nd)
        vr.u[d](i, j, k) += -2 * F.vabc(i, j, k) * (E.psi[vip[d]](i, j, k) - F.relax.u[d](i, j, k));
    _Pragma("unroll") for (int e = 0; e < 4; ++e) if (e < ne) E.psi[e](i, j, k) = E.psi[e](i, j, k) + dt2 * E.rhs[e](i, j, k);
    _Pragma("unroll") for (int d = 0; d < 3; ++d) if (d < g.nd) {
      E.psi[vip[d]](i, j, k) = E.psi[vip[d]](i, j, k) + hdt * vr.u[d](i, j, k);
      vr.u[d](i, j, k) = T(0);
    }
    });
}

// update_rhs (rhs = 0, then the buoyancy and theta forcings of boussinesq_expl.hpp:81-126
// or boussinesq_impl.hpp:82-113 at `at` = 0 / 1), then (post step) apply_rhs(dt / 2),
// vip_rhs = -u and add_relax, or (ante loop) vip_rhs_impl_init
template <class T>
__global__ void k_rhs(geom g, int ne, int post, eqns<T> E, const int *vip, int iw, int ith, forcing<T> F, T dt2,
                      vec_u<T> vr) {
  for_interior(g, [&](int i, int j, int k) {
    _Pragma("unroll") for (int e = 0; e < 4; ++e) if (e < ne) E.rhs[e](i, j, k) = T(0);
    const T th = E.psi[ith](i, j, k), te = F.the(i, j, k), ta = F.tabs(i, j, k), hf = F.hflx(i, j, k);
    const T hdt = T(0.5) * F.dt;
    if (!F.impl) {
      if (!post) {
        E.rhs[ith](i, j, k) = T(0) + (hf - ta * (th - te));
        E.rhs[iw](i, j, k) = T(0) + F.grav * (th - te) / F.tref;
      } else {
        const T x = (th + hdt * hf + hdt * ta * te) / (1 + hdt * ta);
        E.rhs[ith](i, j, k) = T(0) + (hf - ta * (x - te));
        E.rhs[iw](i, j, k) = T(0) + F.grav * (x - te) / F.tref;
      }
    } else if (!post) {
      E.rhs[ith](i, j, k) = T(0) + (-E.psi[iw](i, j, k) * F.dthe(i, j, k) + hf - ta * th);
      E.rhs[iw](i, j, k) = T(0) + F.grav * th / F.tref;
    } else {
      const T rt = T(0) + hf;
      E.rhs[ith](i, j, k) = rt;
      E.rhs[iw](i, j, k) = T(0) + F.grav * (th + hdt * rt) / (F.tref * (1 + hdt * ta));
    }
    if (post) {
      _Pragma("unroll") for (int e = 0; e < 4; ++e) if (e < ne) E.psi[e](i, j, k) = E.psi[e](i, j, k) + dt2 * E.rhs[e](i, j, k);
      _Pragma("unroll") for (int d = 0; d < 3; ++d) if (d < g.nd) {
        vr.u[d](i, j, k) = -E.psi[vip[d]](i, j, k);
        if (F.vab == MPDX_VAB_IMPL)  // add_relax (mpdata_rhs_vip_common.hpp:247-254)
          E.psi[vip[d]](i, j, k) += T(0.5) * F.dt * F.vabc(i, j, k) * F.relax.u[d](i, j, k);
      }
    } else {
      _Pragma("unroll") for (int d = 0; d < 3; ++d) if (d < g.nd) {
        if (F.vab == MPDX_VAB_IMPL) vr.u[d](i, j, k) = -F.vabc(i, j, k) * (E.psi[vip[d]](i, j, k) - F.relax.u[d](i, j, k));
        else vr.u[d](i, j, k) = T(0);
      }
    }
    });
}

// impl_tht end of step (boussinesq_impl.hpp:115-125): theta with the implicit
// w dtht_e / dz term, and its tendency
template <class T>
__global__ void k_impl_fnlz(geom g, eqns<T> E, int iw, int ith, forcing<T> F) {
  for_interior(g, [&](int i, int j, int k) {
    const T w = E.psi[iw](i, j, k), dte = F.dthe(i, j, k), ta = F.tabs(i, j, k);
    const T th = (E.psi[ith](i, j, k) - T(0.5) * F.dt * w * dte) / (1 + T(0.5) * F.dt * ta);
    E.psi[ith](i, j, k) = th;
    E.rhs[ith](i, j, k) += -w * dte - ta * th;
    });
}

// dtht_e = d(tht_e)/dz after the scalar halo fill of tht_e (boussinesq_impl.hpp:38-50):
// along the vertical axis v, cyclic neighbours wrap with period n-1, rigid ones
// mirror (rigid_3d.hpp fill_halos_sclr: a(-1) = a(1), a(n) = a(n-2))
template <class T>
__global__ void k_dtht_e(geom g, dfield<T> te, dfield<T> out) {
  const int v = g.nd - 1;
  for_interior(g, [&](int i, int j, int k) {
    const int c[3] = {i, j, k};
    const int n = g.n[v];
    auto at = [&](int q) {
      if (q < 0) q = g.bc[v][0] == MPDX_BC_CYCLIC ? q + n - 1 : -q;
      else if (q > n - 1) q = g.bc[v][1] == MPDX_BC_CYCLIC ? q - (n - 1) : 2 * (n - 1) - q;
      int a[3] = {c[0], c[1], c[2]};
      a[v] = q;
      return te(a[0], a[1], a[2]);
    };
    out(i, j, k) = mpdx::qdiv<T>(at(c[v] + 1) - at(c[v] - 1), g.dx<T>(v), g.rdx<T>(v)) * T(0.5);
    });
}

// denominators of normalize_vip (mpdata_rhs_vip_common.hpp:235-245, boussinesq_impl.hpp:61-80),
// evaluated in real_t and kept in the pressure type
template <class T, class P>
__global__ void k_norm_den(geom g, forcing<T> F, dfield<P> d0, dfield<P> d1, dfield<P> d2) {
  for_interior(g, [&](int i, int j, int k) {
    const T hdt = T(0.5) * F.dt;
    const T vh = F.vab == MPDX_VAB_IMPL ? 1 + hdt * F.vabc(i, j, k) : T(1);
    T vv = vh;
    if (F.impl) {
      const T b = T(0.25) * F.dt * F.dt * F.grav / F.tref * F.dthe(i, j, k) / (1 + hdt * F.tabs(i, j, k));
      vv = F.vab == MPDX_VAB_IMPL ? 1 + hdt * F.vabc(i, j, k) + b : 1 + b;
    }
    dfield<P> D[3] = {d0, d1, d2};
    _Pragma("unroll") for (int d = 0; d < 3; ++d) if (d < g.nd) D[d](i, j, k) = P(d == g.nd - 1 ? vv : vh);
    });
}

// ini_pressure, first part: Phi = -sum_d 0.5 u_d^2 and its mean
template <class T, class P>
__global__ void k_phi_ini(geom g, dfield<P> phi, vec_u<T> vel, gcr_dev<P> *dv, double *part, double npoints) {
  dd acc[1] = {{0.0, 0.0}};
  for_interior(g, [&](int i, int j, int k) {
    P p = P(0);
    _Pragma("unroll") for (int d = 0; d < 3; ++d) if (d < g.nd) {
      const P v = P(vel.u[d](i, j, k));
      p = p - P(0.5) * (v * v);
    }
    phi(i, j, k) = p;
    acc[0] = dd_add(acc[0], dd{double(p), 0.0});
    });
  double mx = 0, mn = 0;
  if (grid_reduce<1, false>(acc, mx, mn, part, &dv->arrive) && threadIdx.x == 0 && threadIdx.y == 0) dv->mean = P(ddv(acc[0])) / P(npoints);
}
template <class P>
__global__ void k_phi_sub_mean(geom g, dfield<P> phi, const gcr_dev<P> *dv) {
  const P m = dv->mean;
  for_interior(g, [&](int i, int j, int k) {
    phi(i, j, k) = phi(i, j, k) - m;
    });
}

}  // namespace bq

// ---------------------------------------------------------------------------
// host sequencer

namespace {
template <class T>
bq::geom make_geom(const mpdata_state<T> &st, const double *dijk) {
  bq::geom g;
  g.nd = st.nd;
  for (int d = 0; d < 3; ++d) {
    g.n[d] = st.n[d];
    g.bc[d][0] = st.bcs[d][0];
    g.bc[d][1] = st.bcs[d][1];
    g.dxd[d] = dijk[d];
    g.rdxd[d] = 1.0 / dijk[d];                  // RN(1/dx) in FP64
    g.dxf[d] = float(dijk[d]);
    g.rdxf[d] = 1.0f / float(dijk[d]);          // RN(1/dx) in FP32
  }
  g.cells = st.cells();
  g.nf = st.n[st.nd - 1];
  g.nrows = int(g.cells / g.nf);
  return g;
}
const dim3 kBlk(32, kRedThreads / 32);  // 32 points along the contiguous axis x 8 rows
unsigned red_grid(const bq::geom &g) {
  const long long b = (g.nrows + kBlk.y - 1) / kBlk.y;
  return unsigned(std::max(1LL, std::min<long long>(b, kRedBlocks)));
}
}  // namespace

template <class T, class P>
boussinesq<T, P>::boussinesq(const mpdx_config &c, cudaStream_t s) {
  if (c.n_dims < 2) throw error(MPDX_E_UNSUPPORTED, "the Boussinesq solver needs 2 or 3 dimensions");
  if (c.n_eqns != c.n_dims + 1) throw error(MPDX_E_ARG, "the Boussinesq solver advects n_dims + 1 equations (velocities and theta)");
  if (c.precond != MPDX_PRECOND_IDENTITY && c.precond != MPDX_PRECOND_LEARNED) throw error(MPDX_E_ARG, "unknown preconditioner");
  if (c.dt <= 0) throw error(MPDX_E_ARG, "dt must be positive");
  if (c.tht_ref == 0) throw error(MPDX_E_ARG, "Tht_ref must be non-zero");
  for (int q = 0; q < 2 * c.n_dims; ++q)
    if (c.bcs[q] != MPDX_BC_CYCLIC && c.bcs[q] != MPDX_BC_RIGID && c.bcs[q] != MPDX_BC_GNDSKY)
      throw error(MPDX_E_UNSUPPORTED, "the Boussinesq solver supports cyclic and rigid boundaries");
  k_iters = c.prs_scheme == MPDX_PRS_CR ? 1 : c.prs_k_iters;  // cr is gcrk<1> (mpdata_rhs_vip_prs.hpp:55-64)
  if (k_iters < 1 || k_iters > kGcrMaxK) throw error(MPDX_E_ARG, "prs_k_iters must be in 1..8");
  st.stream = s;
  st.setup(c.n_dims, c.grid, c.n_eqns, unsigned(c.opts), c.n_iters, c.bcs);
  for (int d = 0; d < st.nd; ++d)
    if (st.n[d] < 2 * st.H + 1) throw error(MPDX_E_GRID, "libmpdata++: bogus grid size");
  st.max_abs_div_eps = c.max_abs_div_eps < 0 ? std::numeric_limits<T>::epsilon() : T(c.max_abs_div_eps);
  st.upwind_filter_freq = c.upwind_filter_freq;
  dt = c.dt;
  dtT = T(c.dt);
  // grid spacings as real_t values (what the reference's rt_params hold), kept in double
  dijk[0] = double(T(c.di)); dijk[1] = double(T(c.dj)); dijk[2] = double(T(c.dk));
  g = T(c.g); tht_ref = T(c.tht_ref);
  err_tol = P(T(c.prs_tol)) / P(dtT);  // mpdata_rhs_vip_prs_common.hpp:205
  const int ixs[3] = {c.ix_u, c.n_dims == 3 ? c.ix_v : c.ix_w, c.ix_w};
  bool seen[4] = {false, false, false, false};
  for (int d = 0; d < st.nd; ++d) {
    vip[d] = ixs[d];
    if (vip[d] < 0 || vip[d] >= st.n_eqns || seen[vip[d]]) throw error(MPDX_E_ARG, "invalid velocity equation indices");
    seen[vip[d]] = true;
  }
  ix_w = c.ix_w; ix_tht = c.ix_tht;
  if (ix_tht < 0 || ix_tht >= st.n_eqns || seen[ix_tht]) throw error(MPDX_E_ARG, "invalid theta equation index");
  impl_tht = c.impl_tht ? 1 : 0;
  vab = c.vip_vab;
  if (vab != MPDX_VAB_NONE && vab != MPDX_VAB_EXPL && vab != MPDX_VAB_IMPL) throw error(MPDX_E_ARG, "unknown velocity absorber");
  for (int d = 0; d < st.nd; ++d) { st.alloc_sclr(stash[d]); st.alloc_sclr(vip_rhs[d]); st.alloc_sclr(vab_relax[d]); }
  st.alloc_sclr(tht_abs); st.alloc_sclr(hflux_frc); st.alloc_sclr(vab_coeff); st.alloc_sclr(dtht_e);
  // hflux_frc = 0, tht_abs = 0 (boussinesq_common.hpp:51-52), whatever the allocation holds
  MPDX_CUDA(cudaMemsetAsync(tht_abs.base, 0, tht_abs.bytes, s));
  MPDX_CUDA(cudaMemsetAsync(hflux_frc.base, 0, hflux_frc.bytes, s));
  if (normalizes())
    for (int d = 0; d < st.nd; ++d) st.alloc_sclr(den[d]);
  for (int e = 0; e < st.n_eqns; ++e) st.alloc_sclr(rhs[e]);
  st.alloc_sclr(tht_e); st.alloc_sclr(Phi); st.alloc_sclr(err[0]); st.alloc_sclr(err[1]); st.alloc_sclr(lap_err);
  p_err.resize(k_iters); lap_p_err.resize(k_iters);
  for (int v = 0; v < k_iters; ++v) { st.alloc_sclr(p_err[v]); st.alloc_sclr(lap_p_err[v]); }
  MPDX_CUDA(cudaMalloc(&dev, sizeof(gcr_dev<P>)));
  MPDX_CUDA(cudaMallocHost(&hdev, sizeof(gcr_dev<P>)));
  gcr_dev<P> init;
  std::memset(&init, 0, sizeof(init));
  init.beta = P(.25);  // mpdata_rhs_vip_prs_gcrk.hpp:110-112
  for (int v = 0; v < kGcrMaxK; ++v) { init.alpha[v] = P(1); init.tmp_den[v] = P(1); }
  MPDX_CUDA(cudaMemcpy(dev, &init, sizeof(init), cudaMemcpyHostToDevice));
  MPDX_CUDA(cudaMalloc(&part, sizeof(double) * kRedBlocks * kRedSlots * 2));
  MPDX_CUDA(cudaMalloc(&scratch, 64));
  MPDX_CUDA(cudaMalloc(&vip_dev, 3 * sizeof(int)));
  MPDX_CUDA(cudaMemcpy(vip_dev, vip, 3 * sizeof(int), cudaMemcpyHostToDevice));
}

template <class T, class P>
boussinesq<T, P>::~boussinesq() {
  if (dev) cudaFree(dev);
  if (hdev) cudaFreeHost(hdev);
  if (part) cudaFree(part);
  if (scratch) cudaFree(scratch);
  if (vip_dev) cudaFree(vip_dev);
  for (float *p : {pairs, tr_r, tr_t, tr_q, tr_z, tr_dq, tr_a, tr_b}) if (p) cudaFree(p);
  if (tr_loss) cudaFree(tr_loss);
  for (cudaEvent_t e : ev_solve) if (e) cudaEventDestroy(e);
}

// pressure_solver_update (mpdata_rhs_vip_prs_common.hpp:99-123) without the final
// gradient, which the callers fuse into their own kernels
template <class T, class P>
void boussinesq<T, P>::pressure_solve(bool simple) {
  const trace_range tr(use_net && net ? "gcr_solve_learned" : "gcr_solve");
  const auto gm = simple ? make_geom(st, dijk) : norm_geom(make_geom(st, dijk));
  const unsigned G = red_grid(gm);
  cudaStream_t s = st.stream;
  bq::vec_u<T> u;
  for (int d = 0; d < 3; ++d) u.u[d] = d < st.nd ? vips(d).v : vips(0).v;
  bq::dirs<P> D;
  for (int v = 0; v < kGcrMaxK; ++v) {
    D.p[v] = p_err[std::min(v, k_iters - 1)].v;
    D.lp[v] = lap_p_err[std::min(v, k_iters - 1)].v;
  }
  if (!ev_solve[0]) { MPDX_CUDA(cudaEventCreate(&ev_solve[0])); MPDX_CUDA(cudaEventCreate(&ev_solve[1])); }
  MPDX_CUDA(cudaEventRecord(ev_solve[0], s));
  // recording: the pair (residual, Phi_end - Phi) at the start and at up to
  // kSnaps later iterations of this plain solve
  const bool rec = pairs && n_pairs < max_pairs && !(use_net && net);
  long long rec_slots[1 + kSnaps];
  int n_rec = 0;
  if (rec) {
    rec_slots[n_rec++] = n_pairs++;
    bq::k_copy_field<P><<<G, kBlk, 0, s>>>(gm, Phi.v, snap[0].v);
  }
  bq::k_gcr_reset<P><<<1, 1, 0, s>>>(dev);
  bq::k_err_init<P, T><<<G, kBlk, 0, s>>>(gm, Phi.v, u, err[0].v);
  if (rec) bq::k_to_compact<P><<<G, kBlk, 0, s>>>(gm, err[0].v, dfield<P>{}, pairs + size_t(rec_slots[0]) * 2 * gm.cells);
  const bool learned = use_net && net;
  const int nl_idx = learned && nl_fixed < 0 ? pick_nl() : -1;
  const long long nl = !learned ? 0 : (nl_fixed >= 0 ? nl_fixed : nl_cand[nl_idx]);
  bool pcnd = learned && nl > 0;
  fell_back = false;
  restarted = false;
  long long discarded = 0;  // iterations of a learned attempt that was given up
  if (learned) bq::k_copy_field<P><<<G, kBlk, 0, s>>>(gm, Phi.v, phi_start.v);
  long long learned_steps = 0;
  if (pcnd) {
    // the learned corrections: nl steps Phi += beta q, err += beta lap(q) along
    // q = M(err), each with the energy-optimal beta, before plain GCR starts
    if constexpr (std::is_same<P, double>::value) {
      for (long long l = 0; l < nl; ++l) {
        const auto &e = err[0].v;
        net->forward_field(e.o, e.s0, e.s1, e.s2, nullptr, p_err[0].v.o, &dev->converged);
        for (int d = 0; d < st.nd; ++d)
          if (gm.bc[d][0] == MPDX_BC_CYCLIC) bq::k_seam_dup<P><<<G, kBlk, 0, s>>>(gm, p_err[0].v, d);
        bq::k_gcr_init_pc<P><<<G, kBlk, 0, s>>>(gm, err[0].v, p_err[0].v, lap_p_err[0].v, dev, part);
        bq::launch_pc_update<P, 1>(G, kBlk, s, gm, err_tol, Phi.v, err[0].v, D, dev, part);
      }
    }
    MPDX_LAUNCH_CHECK();
    learned_steps = nl;
    fell_back = true;  // the solve continues with plain directions
    pcnd = false;
    MPDX_CUDA(cudaMemcpyAsync(hdev, dev, sizeof(gcr_dev<P>), cudaMemcpyDeviceToHost, s));
    MPDX_CUDA(cudaStreamSynchronize(s));
    // a correction with non-finite sums changed nothing; the residual test of the
    // reference runs in the plain iterations that follow
    bq::k_gcr_clear_bad<P><<<1, 1, 0, s>>>(dev);
    bq::k_gcr_reset_conv<P><<<1, 1, 0, s>>>(dev);
  }
  bq::k_gcr_init<P><<<G, kBlk, 0, s>>>(gm, err[0].v, p_err[0].v, lap_p_err[0].v, dev, part);
  MPDX_LAUNCH_CHECK();
  long long launched = 0;
  for (;;) {
    long long batch = launched == 0 ? std::max(1LL, predicted) : std::max(4LL, predicted / 4);
    if (rec) batch = std::min(batch, 16LL);  // snapshots are taken between batches
    for (long long b = 0; b < batch; ++b)
      for (int v = 0; v < k_iters; ++v)
        bq::launch_inner<P>(v, G, kBlk, s, gm, k_iters, err_tol, Phi.v, err[0].v, err[1].v, lap_err.v, D, dev, part);
    MPDX_LAUNCH_CHECK();
    launched += batch;
    MPDX_CUDA(cudaEventRecord(ev_solve[1], s));
    MPDX_CUDA(cudaMemcpyAsync(hdev, dev, sizeof(gcr_dev<P>), cudaMemcpyDeviceToHost, s));
    MPDX_CUDA(cudaStreamSynchronize(s));
    // a learned solve that, after handing over, still runs far past a plain solve's
    // iteration count is redone from its start with plain GCR alone, so the learned
    // form never gives a worse result than the method without it
    if (learned && !restarted && (hdev->stuck || (!pcnd && hdev->iters > 4 * last_plain_iters + 200))) {
      discarded = hdev->iters;
      bq::k_copy_field<P><<<G, kBlk, 0, s>>>(gm, phi_start.v, Phi.v);
      bq::k_gcr_reset<P><<<1, 1, 0, s>>>(dev);
      bq::k_err_init<P, T><<<G, kBlk, 0, s>>>(gm, Phi.v, u, err[0].v);
      bq::k_gcr_init<P><<<G, kBlk, 0, s>>>(gm, err[0].v, p_err[0].v, lap_p_err[0].v, dev, part);
      MPDX_LAUNCH_CHECK();
      pcnd = false;
      fell_back = true;
      restarted = true;
      launched = 0;
      continue;
    }
    if (hdev->stuck) throw error(MPDX_E_PRS_STUCK, "libmpdata++: stuck in pressure solver");
    if (hdev->done) break;
    if (rec && n_rec < 1 + kSnaps && n_pairs < max_pairs && hdev->iters >= 16LL << (n_rec - 1)) {
      const auto &e = err[hdev->cur].v;  // the current error after the last inner step
      rec_slots[n_rec] = n_pairs++;
      bq::k_to_compact<P><<<G, kBlk, 0, s>>>(gm, e, dfield<P>{}, pairs + size_t(rec_slots[n_rec]) * 2 * gm.cells);
      bq::k_copy_field<P><<<G, kBlk, 0, s>>>(gm, Phi.v, snap[n_rec].v);
      MPDX_LAUNCH_CHECK();
      ++n_rec;
    }
  }
  {
    float ms = 0;
    MPDX_CUDA(cudaEventElapsedTime(&ms, ev_solve[0], ev_solve[1]));
    last_solve_ms = ms;
  }
  iters = hdev->iters + learned_steps + discarded;
  iters_total += iters;
  if (learned) {
    if (nl_idx >= 0) {
      nl_ms[nl_idx] = nl_tries[nl_idx] == 0 ? last_solve_ms : 0.5 * (nl_ms[nl_idx] + last_solve_ms);
      ++nl_tries[nl_idx];
    }
    nl_used = nl;
    ++n_learned;
  }
  if (!(use_net && net)) { last_plain_iters = iters; last_plain_ms = last_solve_ms; }
  last_residual = hdev->residual;
  predicted = std::max(1LL, iters);
  for (int q = 0; q < n_rec; ++q)  // corrections Phi_end - Phi_snapshot
    bq::k_to_compact<P><<<G, kBlk, 0, s>>>(gm, Phi.v, snap[q].v, pairs + (size_t(rec_slots[q]) * 2 + 1) * gm.cells);
  MPDX_LAUNCH_CHECK();
}
template <class T, class P>
void boussinesq<T, P>::ensure_net() {
  if (net) return;
  if constexpr (!std::is_same<P, double>::value) {
    throw error(MPDX_E_UNSUPPORTED, "the learned preconditioner needs the FP64 pressure solve (dtype 8, or prs_fp64)");
  } else {
    int grid[3], wrap[3];
    for (int d = 0; d < 3; ++d) {
      grid[d] = d < st.nd ? st.n[d] : 1;
      wrap[d] = d < st.nd ? (st.bcs[d][0] == MPDX_BC_CYCLIC ? 1 : 0) : 1;
    }
    net.reset(new pc::net(st.nd, grid, wrap, pc_channels, 12345, st.stream));
    st.alloc_sclr(phi_start);
  }
}

template <class T, class P>
void boussinesq<T, P>::precond_record(long long n) {
  if constexpr (!std::is_same<P, double>::value) {
    (void)n;
    throw error(MPDX_E_UNSUPPORTED, "the learned preconditioner needs the FP64 pressure solve (dtype 8, or prs_fp64)");
  } else {
    if (n < 0) throw error(MPDX_E_ARG, "negative pair count");
    if (pairs) { cudaFree(pairs); pairs = nullptr; }
    max_pairs = n;
    n_pairs = 0;
    if (n == 0) return;
    const size_t vox = size_t(st.cells());
    MPDX_CUDA(cudaMalloc(&pairs, size_t(n) * 2 * vox * sizeof(float)));
    for (auto &f : snap)
      if (!f.base) st.alloc_sclr(f);
  }
}


template <class T, class P>
void boussinesq<T, P>::ensure_training() {
  const long long vox = st.cells();
  if (!tr_r) {
    for (float **b : {&tr_r, &tr_t, &tr_q, &tr_z, &tr_dq, &tr_a, &tr_b}) MPDX_CUDA(cudaMalloc(b, vox * sizeof(float)));
    MPDX_CUDA(cudaMalloc(&tr_loss, 4 * sizeof(double)));
  }

}

// Energy-norm loss of one pair (r, t) held in tr_r / tr_t: q = net(r), e = c q - t,
// E = e^T (-A) e / (t^T (-A) t) (1 for a zero output); with grad, the parameter
// gradient goes to net->grad.  Returns E (read back from the device).
template <class T, class P>
double boussinesq<T, P>::pair_energy(float c, bool grad) {
  const auto gm = make_geom(st, dijk);
  const unsigned G = red_grid(gm);
  cudaStream_t s = st.stream;
  const long long vox = st.cells();
  net->forward_compact(tr_r, tr_q);
  bq::k_sub<<<1184, 256, 0, s>>>(tr_q, c, tr_t, vox, tr_z);                 // e = c q - t
  MPDX_CUDA(cudaMemsetAsync(tr_loss, 0, 2 * sizeof(double), s));
  // |grad e|^2 and |grad t|^2 (the gradients of e kept for the adjoint)
  bq::k_grad_sq<<<G, kBlk, 0, s>>>(gm, tr_z, tr_dq, st.nd > 1 ? tr_a : nullptr, st.nd > 2 ? tr_b : nullptr, tr_loss);
  bq::k_grad_sq<<<G, kBlk, 0, s>>>(gm, tr_t, nullptr, nullptr, nullptr, tr_loss + 1);
  if (grad) {
    bq::k_grad_adj<<<G, kBlk, 0, s>>>(gm, tr_dq, tr_a, tr_b, tr_loss + 1, c, tr_q);  // dL/dq
    MPDX_LAUNCH_CHECK();
    net->backward(tr_r, tr_q, net->grad);
  }
  MPDX_LAUNCH_CHECK();
  double h[2];
  MPDX_CUDA(cudaMemcpyAsync(h, tr_loss, sizeof(h), cudaMemcpyDeviceToHost, s));
  MPDX_CUDA(cudaStreamSynchronize(s));
  return h[1] > 0.0 ? h[0] / h[1] : 1.0;  // |grad e|^2 / |grad t|^2
}

// pair k of the recorded ones, divided by rms(r), into tr_r / tr_t (the loss does not
// depend on the common scale of a pair: the network is linear)
template <class T, class P>
void boussinesq<T, P>::load_pair(long long k) {
  cudaStream_t s = st.stream;
  const long long vox = st.cells();
  const float *r = pairs + size_t(k) * 2 * vox, *d = r + vox;
  MPDX_CUDA(cudaMemsetAsync(tr_loss + 3, 0, sizeof(double), s));
  bq::k_sumsq<<<296, 256, 0, s>>>(r, vox, tr_loss + 3);
  bq::k_scale_rms<<<1184, 256, 0, s>>>(r, d, vox, tr_loss + 3, tr_r, tr_t);
  MPDX_LAUNCH_CHECK();
}

template <class T, class P>
double boussinesq<T, P>::precond_train(long long steps, double lr, unsigned long long seed) {
  if constexpr (!std::is_same<P, double>::value) {
    (void)steps; (void)lr; (void)seed;
    throw error(MPDX_E_UNSUPPORTED, "the learned preconditioner needs the FP64 pressure solve (dtype 8, or prs_fp64)");
  } else {
    if (n_pairs < 1) throw error(MPDX_E_ARG, "no recorded pressure solves to train on (call precond_record first)");
    ensure_net();
    ensure_training();
    const long long vox = st.cells();
    cudaStream_t s = st.stream;
    // output scale: A^-1 amplifies the residual by orders of magnitude, so the
    // network learns q with c * q ~ correction, c = rms(correction) / rms(residual)
    // over the recorded pairs (GCR itself is indifferent to the scale of q)
    if (out_scale <= 0) {
      double rr = 0, dd = 0;
      for (long long k = 0; k < n_pairs; ++k) {
        const float *r = pairs + size_t(k) * 2 * vox, *d = r + vox;
        MPDX_CUDA(cudaMemsetAsync(tr_loss, 0, 2 * sizeof(double), s));
        bq::k_sumsq<<<296, 256, 0, s>>>(r, vox, tr_loss);
        bq::k_sumsq<<<296, 256, 0, s>>>(d, vox, tr_loss + 1);
        double h[2];
        MPDX_CUDA(cudaMemcpyAsync(h, tr_loss, sizeof(h), cudaMemcpyDeviceToHost, s));
        MPDX_CUDA(cudaStreamSynchronize(s));
        rr += h[0]; dd += h[1];
      }
      out_scale = rr > 0 ? std::sqrt(dd / rr) : 1.0;
    }
    const float c = float(out_scale);
    // the last fifth of the pairs (at least one) is held out: the validation loss
    // chooses the weights returned; training draws from the rest (all of them when
    // only one pair was recorded)
    const long long n_val = std::min(8LL, std::max(1LL, n_pairs / 5)), n_tr = n_pairs > 1 ? n_pairs - n_val : 1;
    auto validate = [&]() {
      double sum = 0;
      for (long long k = n_pairs - n_val; k < n_pairs; ++k) { load_pair(k); sum += pair_energy(c, false); }
      return sum / double(n_val);
    };
    std::vector<float> best(size_t(net->n_params));
    net->get_params(best.data());  // the starting weights (the zero-output layer at first)
    double best_val = validate();
    const long long every = std::max(1LL, steps / 20), warm = std::max(1LL, steps / 20);
    unsigned long long x = seed * 6364136223846793005ull + 1442695040888963407ull;
    for (long long it = 0; it < steps; ++it) {
      x = x * 6364136223846793005ull + 1442695040888963407ull;
      load_pair((long long)((x >> 33) % (unsigned long long)n_tr));
      pair_energy(c, true);
      // linear warm-up, then cosine decay to 1 % of lr
      const double ph = it < warm ? double(it + 1) / double(warm)
                                  : 0.01 + 0.99 * 0.5 * (1.0 + std::cos(3.14159265358979 * double(it - warm) / double(std::max(1LL, steps - warm))));
      net->adam_step(float(lr * ph));
      if ((it + 1) % every == 0 || it + 1 == steps) {
        const double v = validate();
        if (v < best_val) { best_val = v; net->get_params(best.data()); }
      }
    }
    net->set_params(best.data());
    last_train_loss = best_val;
    return best_val;
  }
}

template <class T, class P>
double boussinesq<T, P>::precond_loss_grad(const double *r, const double *t, double c, float *grad_host) {
  if constexpr (!std::is_same<P, double>::value) {
    (void)r; (void)t; (void)c; (void)grad_host;
    throw error(MPDX_E_UNSUPPORTED, "the learned preconditioner needs the FP64 pressure solve (dtype 8, or prs_fp64)");
  } else {
    ensure_net();
    ensure_training();
    const long long vox = st.cells();
    std::vector<float> hr(vox), ht(vox);
    for (long long q = 0; q < vox; ++q) { hr[q] = float(r[q]); ht[q] = float(t[q]); }
    MPDX_CUDA(cudaMemcpyAsync(tr_r, hr.data(), vox * sizeof(float), cudaMemcpyHostToDevice, st.stream));
    MPDX_CUDA(cudaMemcpyAsync(tr_t, ht.data(), vox * sizeof(float), cudaMemcpyHostToDevice, st.stream));
    const double E = pair_energy(float(c), grad_host != nullptr);
    if (grad_host) {
      MPDX_CUDA(cudaMemcpyAsync(grad_host, net->grad, net->n_params * sizeof(float), cudaMemcpyDeviceToHost, st.stream));
      MPDX_CUDA(cudaStreamSynchronize(st.stream));
    }
    return E;
  }
}

// the number of learned directions at the start of the next learned solve: every
// candidate is tried twice (in order), then the one with the shortest mean solve
// time is taken, and every 64th learned solve re-measures one candidate in turn
template <class T, class P>
int boussinesq<T, P>::pick_nl() {
  for (int c = 0; c < kNlCand; ++c)
    if (nl_tries[c] < 2) return c;
  if (n_learned % 64 == 63) return int((n_learned / 64) % kNlCand);
  int best = 0;
  for (int c = 1; c < kNlCand; ++c)
    if (nl_ms[c] < nl_ms[best]) best = c;
  return best;
}

template <class T, class P>
void boussinesq<T, P>::precond_enable(bool on) {
  if (on) ensure_net();
  use_net = on;
}


template <class T, class P>
void boussinesq<T, P>::ante_loop() {
  const auto gm = make_geom(st, dijk);
  const unsigned G = red_grid(gm);
  cudaStream_t s = st.stream;
  bq::vec_u<T> u, vr;
  for (int d = 0; d < 3; ++d) {
    const int dd = d < st.nd ? d : 0;
    u.u[d] = vips(dd).v; vr.u[d] = vip_rhs[dd].v;
  }
  if (impl_tht) {  // calc_dtht_e (boussinesq_impl.hpp:57-61) comes first
    bq::k_dtht_e<T><<<G, kBlk, 0, s>>>(gm, tht_e.v, dtht_e.v);
    MPDX_LAUNCH_CHECK();
  }
  // initial projection (mpdata_rhs_vip_prs_common.hpp:130-146), with the simple
  // Laplacian (no normalize_vip); save_edges is a no-op here
  MPDX_CUDA(cudaMemsetAsync(Phi.base, 0, Phi.bytes, s));
  pressure_solve(true);
  bq::k_apply_grad<T, P><<<G, kBlk, 0, s>>>(gm, bq::APPLY_PROJECT, Phi.v, u, vr, T(0));
  MPDX_LAUNCH_CHECK();
  // mpdata_rhs_vip_common.hpp:283-302: GC = 0, stash = 0, parent hooks, vip_rhs = 0
  for (int d = 0; d < st.nd; ++d) {
    MPDX_CUDA(cudaMemsetAsync(st.GC[d].base, 0, st.GC[d].bytes, s));
    MPDX_CUDA(cudaMemsetAsync(stash[d].base, 0, stash[d].bytes, s));
    MPDX_CUDA(cudaMemsetAsync(vip_rhs[d].base, 0, vip_rhs[d].bytes, s));
  }
  gen.ante_loop(scratch);
  bq::eqns<T> E;
  for (int e = 0; e < 4; ++e) {
    const int ee = e < st.n_eqns ? e : 0;
    E.psi[e] = st.psi[ee][st.tl[ee]].v;
    E.rhs[e] = rhs[ee].v;
  }
  // update_rhs(dt / 2, at = 0) and vip_rhs_impl_init; update_rhs's halo exchange of
  // every equation is left out: the next read of any halo is preceded by its own exchange
  bq::k_rhs<T><<<G, kBlk, 0, s>>>(gm, st.n_eqns, 0, E, vip_dev, ix_w, ix_tht, forcing(), dtT / 2, vr);
  // ini_pressure (mpdata_rhs_vip_prs_common.hpp:86-97), then vip_rhs -= grad Phi
  double npoints = 1;
  for (int d = 0; d < st.nd; ++d) npoints *= st.n[d];
  bq::k_phi_ini<T, P><<<G, kBlk, 0, s>>>(gm, Phi.v, u, dev, part, npoints);
  bq::k_phi_sub_mean<P><<<G, kBlk, 0, s>>>(gm, Phi.v, dev);
  bq::k_apply_grad<T, P><<<G, kBlk, 0, s>>>(gm, bq::APPLY_RHS, Phi.v, u, vr, T(0));
  MPDX_LAUNCH_CHECK();
}

template <class T, class P>
void boussinesq<T, P>::step() {
  const auto gm = make_geom(st, dijk);
  const unsigned G = red_grid(gm);
  cudaStream_t s = st.stream;
  bq::vec_u<T> u, vr, sh;
  for (int d = 0; d < 3; ++d) {
    const int dd = d < st.nd ? d : 0;
    u.u[d] = vips(dd).v; vr.u[d] = vip_rhs[dd].v; sh.u[d] = stash[dd].v;
  }
  // calc_gc: extrapolate_in_time + interpolate_in_space
  const T b = dt_stash0 > T(0) ? dtT / (2 * dt_stash0) : T(0);
  bq::k_extrp<T><<<G, kBlk, 0, s>>>(gm, sh, u, b);
  MPDX_LAUNCH_CHECK();
  const int ex = st.H - 1;
  for (int d = 0; d < st.nd; ++d) gen.xchng_pres(stash[d], ex);
  for (int d = 0; d < st.nd; ++d) {
    rng r[3];
    for (int q = 0; q < 3; ++q) r[q] = q < st.nd ? ext(st.ir[q], ex) : rng{0, 0};
    r[d] = ext(st.im[d], ex);
    const T c = dtT / T(dijk[d]) * T(.5);
    const long long tot = (long long)r[0].n() * r[1].n() * r[2].n();
    bq::k_intrp<T><<<std::max(1u, std::min(ceil_div(tot, 256), 65535u * 8)), 256, 0, s>>>(
        st.GC[d].v, stash[d].v, d, c, r[0].f, r[1].f, r[2].f, r[0].n(), r[1].n(), r[2].n());
  }
  MPDX_LAUNCH_CHECK();
  gen.xchng_vctr_alng(st.GC, false, true);
  gen.xchng_vctr_nrml(st.GC, ex);
  // hook_ante_step
  bq::eqns<T> E;
  for (int e = 0; e < 4; ++e) {
    const int ee = e < st.n_eqns ? e : 0;
    E.psi[e] = st.psi[ee][st.tl[ee]].v;
    E.rhs[e] = rhs[ee].v;
  }
  bq::k_ante_step<T><<<G, kBlk, 0, s>>>(gm, st.n_eqns, E, vip_dev, sh, vr, dtT / 2, T(0.5) * dtT, forcing());
  MPDX_LAUNCH_CHECK();
  // advection of every equation
  gen.step();
  ++st.timestep;
  dt_stash0 = dtT;
  // hook_post_step
  for (int d = 0; d < 3; ++d) u.u[d] = vips(d < st.nd ? d : 0).v;
  for (int e = 0; e < 4; ++e) E.psi[e] = st.psi[e < st.n_eqns ? e : 0][st.tl[e < st.n_eqns ? e : 0]].v;
  bq::k_rhs<T><<<G, kBlk, 0, s>>>(gm, st.n_eqns, 1, E, vip_dev, ix_w, ix_tht, forcing(), dtT / 2, vr);
  MPDX_LAUNCH_CHECK();
  pressure_solve(false);
  bq::k_apply_grad<T, P><<<G, kBlk, 0, s>>>(norm_geom(gm), bq::APPLY_FINISH, Phi.v, u, vr, T(0.5) * dtT);
  if (impl_tht) bq::k_impl_fnlz<T><<<G, kBlk, 0, s>>>(gm, E, ix_w, ix_tht, forcing());
  MPDX_LAUNCH_CHECK();
}

template <class T, class P>
bq::forcing<T> boussinesq<T, P>::forcing() {
  bq::forcing<T> F;
  F.the = tht_e.v; F.tabs = tht_abs.v; F.hflx = hflux_frc.v; F.dthe = dtht_e.v; F.vabc = vab_coeff.v;
  for (int d = 0; d < 3; ++d) F.relax.u[d] = vab_relax[d < st.nd ? d : 0].v;
  F.impl = impl_tht; F.vab = vab;
  F.grav = g; F.tref = tht_ref; F.dt = dtT;
  return F;
}

// the geometry with normalize_vip inside lap() and after the pressure gradient,
// where the configuration normalises (velocity absorber impl, or impl_tht)
template <class T, class P>
bq::geom boussinesq<T, P>::norm_geom(bq::geom gm) const {
  if (!normalizes()) return gm;
  gm.norm = 1;
  for (int d = 0; d < 3; ++d) gm.den[d] = den[d < st.nd ? d : 0].v.o;
  return gm;
}

template <class T, class P>
void boussinesq<T, P>::advance(long long nt) {
  if (nt <= 0) return;
  if (st.timestep == 0) ante_loop();
  if (normalizes()) {  // from the absorber / theta fields as they are now
    const auto gm = make_geom(st, dijk);
    bq::k_norm_den<T, P><<<red_grid(gm), kBlk, 0, st.stream>>>(gm, forcing(), den[0].v, den[1].v, den[2].v);
    MPDX_LAUNCH_CHECK();
  }
  for (long long t = 0; t < nt; ++t) step();
}

template struct boussinesq<float, float>;
template struct boussinesq<float, double>;
template struct boussinesq<double, double>;

}  // namespace mpdx
