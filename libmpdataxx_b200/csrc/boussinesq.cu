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
//   k_gcr_update: Phi += beta p_v, err' = err + beta lap_p_v, lap_err = lap(err'),
//                 max|err'| and the alpha sums;
//   k_gcr_direction: new search direction and its lap, and the sums of the
//                 next beta.
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

namespace mpdx {
namespace bq {

struct geom {
  int nd, n[3], bc[3][2];
  double dx[3];  // converted to the arithmetic type where used
  long long cells;
};

__device__ __forceinline__ void ijk_of(const geom &g, long long q, int &i, int &j, int &k) {
  k = int(q % g.n[2]);
  const long long r = q / g.n[2];
  j = int(r % g.n[1]);
  i = int(r / g.n[1]);
}

// plain field and err + beta * lap_p (the updated error, evaluated where it is read)
template <class T>
struct fld {
  dfield<T> a;
  __device__ __forceinline__ T operator()(int i, int j, int k) const { return a(i, j, k); }
};
template <class T>
struct fld_axpy {
  dfield<T> x, y;
  T b;
  __device__ __forceinline__ T operator()(int i, int j, int k) const { return x(i, j, k) + b * y(i, j, k); }
};

// value at the point whose coordinate d is replaced by q (q inside [0, n))
template <class T, class F>
__device__ __forceinline__ T at(const F &A, int d, int i, int j, int k, int q) {
  return d == 0 ? A(q, j, k) : (d == 1 ? A(i, q, k) : A(i, j, q));
}

// A at coordinate q in [-2, n+1] along d with the pressure halo rule
// (cyclic_2d.hpp:35-38 -> fill_halos_sclr; rigid_2d.hpp:26-35, 134-143)
template <class T, class F>
__device__ __forceinline__ T aval(const F &A, const geom &g, int d, int i, int j, int k, int q) {
  const int n = g.n[d];
  if (q >= 0 && q < n) return at<T>(A, d, i, j, k, q);
  const int side = q < 0 ? 0 : 1;
  if (g.bc[d][side] == MPDX_BC_CYCLIC) return at<T>(A, d, i, j, k, q < 0 ? q + n - 1 : q - (n - 1));
  const int e = side == 0 ? 0 : n - 1, m = side == 0 ? -q : q - (n - 1);
  return T(2) * at<T>(A, d, i, j, k, e) - at<T>(A, d, i, j, k, side == 0 ? m : n - 1 - m);
}

__device__ __forceinline__ bool rigid_edge(const geom &g, int d, int q) {
  return (q == 0 && g.bc[d][0] == MPDX_BC_RIGID) || (q == g.n[d] - 1 && g.bc[d][1] == MPDX_BC_RIGID);
}

// grad_d A at interior coordinate q (nabla_formulae.hpp:18-41)
template <class T, class F>
__device__ __forceinline__ T grad(const F &A, const geom &g, int d, int i, int j, int k, int q) {
  return (aval<T>(A, g, d, i, j, k, q + 1) - aval<T>(A, g, d, i, j, k, q - 1)) / T(g.dx[d]) / T(2);
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
__device__ __forceinline__ T lt(const F &A, const U &u, const geom &g, int d, int i, int j, int k, int q) {
  if (rigid_edge(g, d, q)) return T(0);
  T v = grad<T>(A, g, d, i, j, k, q);
  if constexpr (is_vec<U>::value) {
    const auto &ud = u.u[d];
    v -= T(d == 0 ? ud(q, j, k) : (d == 1 ? ud(i, q, k) : ud(i, j, q)));
  }
  return v;
}
// lap_tmp[d] at coordinate q in [-1, n] (its own pressure halo fill)
template <class T, class F, class U>
__device__ __forceinline__ T LT(const F &A, const U &u, const geom &g, int d, int i, int j, int k, int q) {
  const int n = g.n[d];
  if (q >= 0 && q < n) return lt<T>(A, u, g, d, i, j, k, q);
  const int side = q < 0 ? 0 : 1;
  if (g.bc[d][side] == MPDX_BC_CYCLIC) return lt<T>(A, u, g, d, i, j, k, q < 0 ? q + n - 1 : q - (n - 1));
  const int e = side == 0 ? 0 : n - 1, m = side == 0 ? -q : q - (n - 1);
  return T(2) * lt<T>(A, u, g, d, i, j, k, e) - lt<T>(A, u, g, d, i, j, k, side == 0 ? m : n - 1 - m);
}
// lap(A) at interior point (i, j, k): div(grad A [- u]) (mpdata_rhs_vip_prs_common.hpp:49-84,
// nabla_formulae.hpp:184-215)
template <class T, class F, class U>
__device__ __forceinline__ T lap(const F &A, const U &u, const geom &g, int i, int j, int k) {
  T r = (LT<T>(A, u, g, 0, i, j, k, i + 1) - LT<T>(A, u, g, 0, i, j, k, i - 1)) / T(g.dx[0]) / T(2)
      + (LT<T>(A, u, g, 1, i, j, k, j + 1) - LT<T>(A, u, g, 1, i, j, k, j - 1)) / T(g.dx[1]) / T(2);
  if (g.nd == 3) r = r + (LT<T>(A, u, g, 2, i, j, k, k + 1) - LT<T>(A, u, g, 2, i, j, k, k - 1)) / T(g.dx[2]) / T(2);
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
__device__ bool grid_reduce(dd *acc, int ns, bool mm, double &mx, double &mn, double *part, unsigned *arrive) {
  __shared__ dd wsum[kRedThreads / 32];
  __shared__ double wmx[kRedThreads / 32], wmn[kRedThreads / 32];
  __shared__ bool last;
  __shared__ dd bsum[kRedSlots];
  __shared__ double bmx, bmn;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double *mine = part + size_t(blockIdx.x) * kRedSlots * 2;
  for (int s = 0; s < ns; ++s) {
    const dd v = warp_sum(acc[s]);
    if (lane == 0) wsum[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      dd t = wsum[0];
      for (int q = 1; q < nw; ++q) t = dd_add(t, wsum[q]);
      mine[2 * s] = t.s;
      mine[2 * s + 1] = t.c;
    }
    __syncthreads();
  }
  if (mm) {
    warp_mm(mx, mn);
    if (lane == 0) { wmx[w] = mx; wmn[w] = mn; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = wmx[0], b = wmn[0];
      for (int q = 1; q < nw; ++q) { a = fmax(a, wmx[q]); b = fmin(b, wmn[q]); }
      mine[2 * (kRedSlots - 1)] = a;
      mine[2 * (kRedSlots - 1) + 1] = b;
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(arrive, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return false;
  __threadfence();
  for (int s = 0; s < ns; ++s) {
    dd v{0.0, 0.0};
    for (int b = threadIdx.x; b < int(gridDim.x); b += blockDim.x) {
      const double *p = part + size_t(b) * kRedSlots * 2 + 2 * s;
      v = dd_add(v, dd{__ldcg(p), __ldcg(p + 1)});
    }
    v = warp_sum(v);
    if (lane == 0) wsum[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      dd t = wsum[0];
      for (int q = 1; q < nw; ++q) t = dd_add(t, wsum[q]);
      bsum[s] = t;
    }
    __syncthreads();
  }
  if (mm) {
    double a = -DBL_MAX, b = DBL_MAX;
    for (int q = threadIdx.x; q < int(gridDim.x); q += blockDim.x) {
      const double *p = part + size_t(q) * kRedSlots * 2 + 2 * (kRedSlots - 1);
      a = fmax(a, __ldcg(p));
      b = fmin(b, __ldcg(p + 1));
    }
    warp_mm(a, b);
    if (lane == 0) { wmx[w] = a; wmn[w] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double x = wmx[0], y = wmn[0];
      for (int q = 1; q < nw; ++q) { x = fmax(x, wmx[q]); y = fmin(y, wmn[q]); }
      bmx = x; bmn = y;
    }
    __syncthreads();
    mx = bmx; mn = bmn;
  }
  for (int s = 0; s < ns; ++s) acc[s] = bsum[s];
  if (threadIdx.x == 0) *arrive = 0u;
  return true;
}

__device__ __forceinline__ double ddv(dd a) { return a.s + a.c; }

// ---------------------------------------------------------------------------
// GCR kernels

template <class T>
__global__ void k_gcr_reset(gcr_dev<T> *dv) {
  dv->converged = 0; dv->done = 0; dv->stuck = 0; dv->cur = 0; dv->iters = 0; dv->arrive = 0u;
}

// err = lap(Phi) with err_init (u = the velocity being projected)
template <class P, class T>
__global__ void k_err_init(geom g, dfield<P> phi, vec_u<T> u, dfield<P> err) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.cells; q += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    ijk_of(g, q, i, j, k);
    err(i, j, k) = lap<P>(fld<P>{phi}, u, g, i, j, k);
  }
}

// loop_init: p_0 = err, lap_p_0 = lap(p_0); sums of the first beta
template <class T>
__global__ void k_gcr_init(geom g, dfield<T> err, dfield<T> p0, dfield<T> lp0, gcr_dev<T> *dv, double *part) {
  dd acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.cells; q += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    ijk_of(g, q, i, j, k);
    const T e = err(i, j, k);
    const T l = lap<T>(fld<T>{err}, no_u{}, g, i, j, k);
    p0(i, j, k) = e;
    lp0(i, j, k) = l;
    acc[0] = dd_add(acc[0], dd{double(T(l * l)), 0.0});
    acc[1] = dd_add(acc[1], dd{double(T(e * l)), 0.0});
  }
  double mx = 0, mn = 0;
  if (grid_reduce(acc, 2, false, mx, mn, part, &dv->arrive) && threadIdx.x == 0) {
    dv->pend_den = T(ddv(acc[0]));
    dv->pend_num = T(ddv(acc[1]));
  }
}

template <class T>
struct dirs {
  dfield<T> p[kGcrMaxK], lp[kGcrMaxK];
};

// inner step v, first half (mpdata_rhs_vip_prs_gcrk.hpp:43-64)
template <class T>
__global__ void k_gcr_update(geom g, int v, T err_tol, dfield<T> phi, dfield<T> err0, dfield<T> err1, dfield<T> lap_err,
                             dirs<T> D, gcr_dev<T> *dv, double *part) {
  if (dv->done) return;
  const int cur = dv->cur;
  const dfield<T> ea = cur ? err1 : err0, eb = cur ? err0 : err1;
  const T den = dv->pend_den;
  const T b = den != T(0) ? -dv->pend_num / den : dv->beta;  // beta keeps its value when tmp_den is 0
  if (blockIdx.x == 0 && threadIdx.x == 0) { dv->tmp_den[v] = den; dv->beta = b; }
  const dfield<T> pv = D.p[v], lpv = D.lp[v];
  const fld_axpy<T> enew{ea, lpv, b};
  dd acc[kGcrMaxK];
  for (int l = 0; l <= v; ++l) acc[l] = dd{0.0, 0.0};
  double mx = -DBL_MAX, mn = DBL_MAX;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.cells; q += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    ijk_of(g, q, i, j, k);
    phi(i, j, k) = phi(i, j, k) + b * pv(i, j, k);
    const T e = enew(i, j, k);
    eb(i, j, k) = e;
    mx = fmax(mx, double(e));
    mn = fmin(mn, double(e));
    const T le = lap<T>(enew, no_u{}, g, i, j, k);
    lap_err(i, j, k) = le;
    for (int l = 0; l <= v; ++l) acc[l] = dd_add(acc[l], dd{double(T(le * D.lp[l](i, j, k))), 0.0});
  }
  if (grid_reduce(acc, v + 1, true, mx, mn, part, &dv->arrive) && threadIdx.x == 0) {
    const T amx = fabs(T(mx)), amn = fabs(T(mn));
    const T error = amx < amn ? amn : amx;  // std::max(|max|, |min|)
    dv->residual = double(error);
    if (error <= err_tol) dv->converged = 1;
    for (int l = 0; l <= v; ++l) {
      const T dl = l == v ? den : dv->tmp_den[l];
      if (dl != T(0)) dv->alpha[l] = -T(ddv(acc[l])) / dl;
    }
  }
}

// inner step v, second half: next search direction (mpdata_rhs_vip_prs_gcrk.hpp:66-92)
template <class T>
__global__ void k_gcr_direction(geom g, int v, int kk, dfield<T> err0, dfield<T> err1, dfield<T> lap_err, dirs<T> D,
                                gcr_dev<T> *dv, double *part) {
  if (dv->done) return;
  const int cur = dv->cur;
  const dfield<T> e = cur ? err0 : err1;  // the error written by k_gcr_update
  T a[kGcrMaxK];
  for (int l = 0; l <= v; ++l) a[l] = dv->alpha[l];
  const int dst = v < kk - 1 ? v + 1 : 0;
  const dfield<T> pd = D.p[dst], lpd = D.lp[dst];
  dd acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.cells; q += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    ijk_of(g, q, i, j, k);
    const T ev = e(i, j, k);
    T pn, ln;
    if (v < kk - 1) {
      pn = ev;
      ln = lap_err(i, j, k);
      for (int l = 0; l <= v; ++l) {
        pn = pn + a[l] * D.p[l](i, j, k);
        ln = ln + a[l] * D.lp[l](i, j, k);
      }
    } else {
      pn = ev + a[0] * D.p[0](i, j, k);
      ln = lap_err(i, j, k) + a[0] * D.lp[0](i, j, k);
      for (int l = 1; l <= v; ++l) {
        pn = pn + a[l] * D.p[l](i, j, k);
        ln = ln + a[l] * D.lp[l](i, j, k);
      }
    }
    pd(i, j, k) = pn;
    lpd(i, j, k) = ln;
    acc[0] = dd_add(acc[0], dd{double(T(ln * ln)), 0.0});
    acc[1] = dd_add(acc[1], dd{double(T(ev * ln)), 0.0});
  }
  double mx = 0, mn = 0;
  if (grid_reduce(acc, 2, false, mx, mn, part, &dv->arrive) && threadIdx.x == 0) {
    dv->pend_den = T(ddv(acc[0]));
    dv->pend_num = T(ddv(acc[1]));
    dv->cur = 1 - cur;
    if (v == kk - 1) {  // end of one loop body (mpdata_rhs_vip_prs_common.hpp:111-125)
      dv->iters += 1;
      if (dv->converged) dv->done = 1;
      if (dv->iters > 10000) { dv->stuck = 1; dv->done = 1; }
    }
  }
}

// ---------------------------------------------------------------------------
// pointwise stages

enum { APPLY_PROJECT = 0, APPLY_RHS = 1, APPLY_FINISH = 2 };

// grad Phi applied to the velocities: pressure_solver_apply + set_edges
// (PROJECT), vip_rhs -= grad Phi (RHS, hook_ante_loop), or pressure_solver_apply +
// set_edges + vip_rhs = (vip_rhs + u) / (dt / 2) (FINISH, vip_rhs_impl_fnlz)
template <class T, class P>
__global__ void k_apply_grad(geom g, int mode, dfield<P> phi, vec_u<T> vel, vec_u<T> vr, T hdt) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.cells; q += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    ijk_of(g, q, i, j, k);
    const int c[3] = {i, j, k};
    for (int d = 0; d < g.nd; ++d) {
      const P gd = grad<P>(fld<P>{phi}, g, d, i, j, k, c[d]);
      if (mode == APPLY_RHS) {
        vr.u[d](i, j, k) = T(P(vr.u[d](i, j, k)) - gd);
        continue;
      }
      T v = T(P(vel.u[d](i, j, k)) - gd);
      if (rigid_edge(g, d, c[d])) v = T(0);
      vel.u[d](i, j, k) = v;
      if (mode == APPLY_FINISH) {
        const T r = vr.u[d](i, j, k) + v;
        vr.u[d](i, j, k) = r / hdt;
      }
    }
  }
}

template <class T>
struct eqns {
  dfield<T> psi[4], rhs[4];
};

// extrp (mpdata_rhs_vip_common.hpp:120-153): stash = -beta stash + (1 + beta) u
template <class T>
__global__ void k_extrp(geom g, vec_u<T> stash, vec_u<T> vel, T b) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.cells; q += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    ijk_of(g, q, i, j, k);
    for (int d = 0; d < g.nd; ++d) {
      T s = stash.u[d](i, j, k) * -b;
      s = s + (T(1) + b) * vel.u[d](i, j, k);
      stash.u[d](i, j, k) = s;
    }
  }
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

// hook_ante_step: fill_stash, apply_rhs(dt / 2), vip_rhs_apply
template <class T>
__global__ void k_ante_step(geom g, int ne, eqns<T> E, const int *vip, vec_u<T> stash, vec_u<T> vr, T dt2, T hdt) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.cells; q += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    ijk_of(g, q, i, j, k);
    for (int d = 0; d < g.nd; ++d) stash.u[d](i, j, k) = E.psi[vip[d]](i, j, k);
    for (int e = 0; e < ne; ++e) E.psi[e](i, j, k) = E.psi[e](i, j, k) + dt2 * E.rhs[e](i, j, k);
    for (int d = 0; d < g.nd; ++d) {
      E.psi[vip[d]](i, j, k) = E.psi[vip[d]](i, j, k) + hdt * vr.u[d](i, j, k);
      vr.u[d](i, j, k) = T(0);
    }
  }
}

// update_rhs (rhs = 0; rhs[w] += g (tht - tht_e) / Tht_ref), then (post step)
// apply_rhs(dt / 2) and vip_rhs = -u, or (ante loop) vip_rhs = 0
template <class T>
__global__ void k_rhs(geom g, int ne, int post, eqns<T> E, const int *vip, int iw, int ith, dfield<T> the, T grav,
                      T tref, T dt2, vec_u<T> vr) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.cells; q += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    ijk_of(g, q, i, j, k);
    for (int e = 0; e < ne; ++e) E.rhs[e](i, j, k) = T(0);
    E.rhs[iw](i, j, k) = T(0) + grav * (E.psi[ith](i, j, k) - the(i, j, k)) / tref;
    if (post) {
      for (int e = 0; e < ne; ++e) E.psi[e](i, j, k) = E.psi[e](i, j, k) + dt2 * E.rhs[e](i, j, k);
      for (int d = 0; d < g.nd; ++d) vr.u[d](i, j, k) = -E.psi[vip[d]](i, j, k);
    } else {
      for (int d = 0; d < g.nd; ++d) vr.u[d](i, j, k) = T(0);
    }
  }
}

// ini_pressure, first part: Phi = -sum_d 0.5 u_d^2 and its mean
template <class T, class P>
__global__ void k_phi_ini(geom g, dfield<P> phi, vec_u<T> vel, gcr_dev<P> *dv, double *part, double npoints) {
  dd acc[1] = {{0.0, 0.0}};
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.cells; q += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    ijk_of(g, q, i, j, k);
    P p = P(0);
    for (int d = 0; d < g.nd; ++d) {
      const P v = P(vel.u[d](i, j, k));
      p = p - P(0.5) * (v * v);
    }
    phi(i, j, k) = p;
    acc[0] = dd_add(acc[0], dd{double(p), 0.0});
  }
  double mx = 0, mn = 0;
  if (grid_reduce(acc, 1, false, mx, mn, part, &dv->arrive) && threadIdx.x == 0) dv->mean = P(ddv(acc[0])) / P(npoints);
}
template <class P>
__global__ void k_phi_sub_mean(geom g, dfield<P> phi, const gcr_dev<P> *dv) {
  const P m = dv->mean;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < g.cells; q += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    ijk_of(g, q, i, j, k);
    phi(i, j, k) = phi(i, j, k) - m;
  }
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
    g.dx[d] = dijk[d];
  }
  g.cells = st.cells();
  return g;
}
unsigned red_grid(long long cells) {
  long long b = (cells + kRedThreads - 1) / kRedThreads;
  return unsigned(std::max(1LL, std::min<long long>(b, kRedBlocks)));
}
}  // namespace

template <class T, class P>
boussinesq<T, P>::boussinesq(const mpdx_config &c, cudaStream_t s) {
  if (c.n_dims < 2) throw error(MPDX_E_UNSUPPORTED, "the Boussinesq solver needs 2 or 3 dimensions");
  if (c.n_eqns != c.n_dims + 1) throw error(MPDX_E_ARG, "the Boussinesq solver advects n_dims + 1 equations (velocities and theta)");
  if (c.precond != MPDX_PRECOND_IDENTITY) throw error(MPDX_E_UNSUPPORTED, "preconditioner not built");
  if (c.dt <= 0) throw error(MPDX_E_ARG, "dt must be positive");
  if (c.tht_ref == 0) throw error(MPDX_E_ARG, "Tht_ref must be non-zero");
  for (int q = 0; q < 2 * c.n_dims; ++q)
    if (c.bcs[q] != MPDX_BC_CYCLIC && c.bcs[q] != MPDX_BC_RIGID)
      throw error(MPDX_E_UNSUPPORTED, "the Boussinesq solver supports cyclic and rigid boundaries");
  k_iters = c.prs_scheme == MPDX_PRS_CR ? 1 : c.prs_k_iters;  // cr is gcrk<1> (mpdata_rhs_vip_prs.hpp:55-64)
  if (k_iters < 1 || k_iters > kGcrMaxK) throw error(MPDX_E_ARG, "prs_k_iters must be in 1..8");
  st.stream = s;
  st.setup(c.n_dims, c.grid, c.n_eqns, unsigned(c.opts), c.n_iters, c.bcs);
  for (int d = 0; d < st.nd; ++d)
    if (st.n[d] < 2 * st.H + 1) throw error(MPDX_E_GRID, "libmpdata++: bogus grid size");
  st.max_abs_div_eps = c.max_abs_div_eps < 0 ? std::numeric_limits<T>::epsilon() : T(c.max_abs_div_eps);
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
  for (int d = 0; d < st.nd; ++d) { st.alloc_sclr(stash[d]); st.alloc_sclr(vip_rhs[d]); }
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
}

// pressure_solver_update (mpdata_rhs_vip_prs_common.hpp:99-123) without the final
// gradient, which the callers fuse into their own kernels
template <class T, class P>
void boussinesq<T, P>::pressure_solve() {
  const auto gm = make_geom(st, dijk);
  const unsigned G = red_grid(gm.cells);
  cudaStream_t s = st.stream;
  bq::vec_u<T> u;
  for (int d = 0; d < 3; ++d) u.u[d] = d < st.nd ? vips(d).v : vips(0).v;
  bq::dirs<P> D;
  for (int v = 0; v < kGcrMaxK; ++v) {
    D.p[v] = p_err[std::min(v, k_iters - 1)].v;
    D.lp[v] = lap_p_err[std::min(v, k_iters - 1)].v;
  }
  bq::k_gcr_reset<P><<<1, 1, 0, s>>>(dev);
  bq::k_err_init<P, T><<<G, kRedThreads, 0, s>>>(gm, Phi.v, u, err[0].v);
  bq::k_gcr_init<P><<<G, kRedThreads, 0, s>>>(gm, err[0].v, p_err[0].v, lap_p_err[0].v, dev, part);
  MPDX_LAUNCH_CHECK();
  long long launched = 0;
  for (;;) {
    const long long batch = launched == 0 ? std::max(1LL, predicted) : std::max(4LL, predicted / 4);
    for (long long b = 0; b < batch; ++b)
      for (int v = 0; v < k_iters; ++v) {
        bq::k_gcr_update<P><<<G, kRedThreads, 0, s>>>(gm, v, err_tol, Phi.v, err[0].v, err[1].v, lap_err.v, D, dev, part);
        bq::k_gcr_direction<P><<<G, kRedThreads, 0, s>>>(gm, v, k_iters, err[0].v, err[1].v, lap_err.v, D, dev, part);
      }
    MPDX_LAUNCH_CHECK();
    launched += batch;
    MPDX_CUDA(cudaMemcpyAsync(hdev, dev, sizeof(gcr_dev<P>), cudaMemcpyDeviceToHost, s));
    MPDX_CUDA(cudaStreamSynchronize(s));
    if (hdev->stuck) throw error(MPDX_E_PRS_STUCK, "libmpdata++: stuck in pressure solver");
    if (hdev->done) break;
  }
  iters = hdev->iters;
  iters_total += iters;
  last_residual = hdev->residual;
  predicted = std::max(1LL, iters);
}

template <class T, class P>
void boussinesq<T, P>::ante_loop() {
  const auto gm = make_geom(st, dijk);
  const unsigned G = red_grid(gm.cells);
  cudaStream_t s = st.stream;
  bq::vec_u<T> u, vr;
  for (int d = 0; d < 3; ++d) {
    const int dd = d < st.nd ? d : 0;
    u.u[d] = vips(dd).v; vr.u[d] = vip_rhs[dd].v;
  }
  // initial projection (mpdata_rhs_vip_prs_common.hpp:130-146); save_edges is a no-op here
  MPDX_CUDA(cudaMemsetAsync(Phi.base, 0, Phi.bytes, s));
  pressure_solve();
  bq::k_apply_grad<T, P><<<G, kRedThreads, 0, s>>>(gm, bq::APPLY_PROJECT, Phi.v, u, vr, T(0));
  MPDX_LAUNCH_CHECK();
  // mpdata_rhs_vip_common.hpp:283-302: GC = 0, stash = 0, parent hooks, vip_rhs = 0
  for (int d = 0; d < st.nd; ++d) {
    MPDX_CUDA(cudaMemsetAsync(st.GC[d].base, 0, st.GC[d].bytes, s));
    MPDX_CUDA(cudaMemsetAsync(stash[d].base, 0, stash[d].bytes, s));
  }
  gen.ante_loop(scratch);
  bq::eqns<T> E;
  for (int e = 0; e < 4; ++e) {
    const int ee = e < st.n_eqns ? e : 0;
    E.psi[e] = st.psi[ee][st.tl[ee]].v;
    E.rhs[e] = rhs[ee].v;
  }
  // update_rhs(dt / 2, at = 0); update_rhs's halo exchange of every equation is
  // left out: the next read of any halo is preceded by its own exchange
  bq::k_rhs<T><<<G, kRedThreads, 0, s>>>(gm, st.n_eqns, 0, E, vip_dev, ix_w, ix_tht, tht_e.v, g, tht_ref, dtT / 2, vr);
  // ini_pressure (mpdata_rhs_vip_prs_common.hpp:86-97), then vip_rhs -= grad Phi
  double npoints = 1;
  for (int d = 0; d < st.nd; ++d) npoints *= st.n[d];
  bq::k_phi_ini<T, P><<<G, kRedThreads, 0, s>>>(gm, Phi.v, u, dev, part, npoints);
  bq::k_phi_sub_mean<P><<<G, kRedThreads, 0, s>>>(gm, Phi.v, dev);
  bq::k_apply_grad<T, P><<<G, kRedThreads, 0, s>>>(gm, bq::APPLY_RHS, Phi.v, u, vr, T(0));
  MPDX_LAUNCH_CHECK();
}

template <class T, class P>
void boussinesq<T, P>::step() {
  const auto gm = make_geom(st, dijk);
  const unsigned G = red_grid(gm.cells);
  cudaStream_t s = st.stream;
  bq::vec_u<T> u, vr, sh;
  for (int d = 0; d < 3; ++d) {
    const int dd = d < st.nd ? d : 0;
    u.u[d] = vips(dd).v; vr.u[d] = vip_rhs[dd].v; sh.u[d] = stash[dd].v;
  }
  // calc_gc: extrapolate_in_time + interpolate_in_space
  const T b = dt_stash0 > T(0) ? dtT / (2 * dt_stash0) : T(0);
  bq::k_extrp<T><<<G, kRedThreads, 0, s>>>(gm, sh, u, b);
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
  bq::k_ante_step<T><<<G, kRedThreads, 0, s>>>(gm, st.n_eqns, E, vip_dev, sh, vr, dtT / 2, T(0.5) * dtT);
  MPDX_LAUNCH_CHECK();
  // advection of every equation
  gen.step();
  ++st.timestep;
  dt_stash0 = dtT;
  // hook_post_step
  for (int d = 0; d < 3; ++d) u.u[d] = vips(d < st.nd ? d : 0).v;
  for (int e = 0; e < 4; ++e) E.psi[e] = st.psi[e < st.n_eqns ? e : 0][st.tl[e < st.n_eqns ? e : 0]].v;
  bq::k_rhs<T><<<G, kRedThreads, 0, s>>>(gm, st.n_eqns, 1, E, vip_dev, ix_w, ix_tht, tht_e.v, g, tht_ref, dtT / 2, vr);
  MPDX_LAUNCH_CHECK();
  pressure_solve();
  bq::k_apply_grad<T, P><<<G, kRedThreads, 0, s>>>(gm, bq::APPLY_FINISH, Phi.v, u, vr, T(0.5) * dtT);
  MPDX_LAUNCH_CHECK();
}

template <class T, class P>
void boussinesq<T, P>::advance(long long nt) {
  if (nt <= 0) return;
  if (st.timestep == 0) ante_loop();
  for (long long t = 0; t < nt; ++t) step();
}

template struct boussinesq<float, float>;
template struct boussinesq<float, double>;
template struct boussinesq<double, double>;

}  // namespace mpdx
