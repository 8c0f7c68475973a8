// Fused 2D MPDATA step (n_iters 2 or 3; options {0, fct, iga, iga|fct} for
// n_iters = 2 and {0, fct} for n_iters = 3; all boundaries cyclic).
//
// Decomposition (1.5D blocking): a CTA owns a strip of TJ = W - 2H columns
// (j, contiguous in memory) and marches along x (i) over LX rows.  Every stage
// works on full-width rows of W = NT columns, one column per thread; the H
// outermost columns on each side are computed from wrapped neighbours and
// lose validity by at most one column per stage, which H covers.  Per step t:
//   loads   psi^n row t+2, GC_x faces t+1, GC_y row t+1          [cp.async, one step ahead]
//   psi1    row t        upwind pass                            (mpdata_osc_2d.hpp:137-160)
//   min/max row t-1      of psi^n                               (mpdata_fct_2d.hpp:31-46)
//   C~1     x-face t-1/2... y-faces of row t-1                  (formulae_mpdata_2d.hpp:242-278)
//   betas1  row t-2                                             (formulae_mpdata_fct_2d.hpp:21-120)
//   flux1   x-face t-3+1/2, y-faces row t-3 (limited)           (formulae_mpdata_fct_2d.hpp:122-214)
//   psi2    row t-3      corrective donor-cell pass
// and for n_iters = 3 a second corrective iteration whose antidiffusive
// velocity is computed from psi2 and the unlimited C~1 (GC_unco of the
// reference, mpdata_common.hpp:40-47), ending with psi3 at row t-6.
#pragma once

#include <cfloat>

#include "fused3d.cuh"

namespace mpdx {
namespace f2 {

using f3::flux;
using f3::frac;
using f3::lims;
using f3::mn;
using f3::mx;
using f3::neg;
using f3::pos;
using f3::wrap;

template <class T>
struct prob {  // one 2D problem
  dfield<T> in, out, g0, g1;
  int P0, P1;  // periods
  int n0, n1;  // points per axis
};

template <int NI, bool FCT>
struct rows {
  // ring sizes (rows) and offsets, in units of W
  static constexpr int NP0 = 5, NG0 = 4, NG1 = 3, NP1 = 4;
  static constexpr int NMM = NI == 3 ? 5 : 2;
  static constexpr int NC1X = NI == 3 ? 5 : 3, NC1Y = NI == 3 ? 4 : 3;
  static constexpr int o_p0 = 0, o_g0 = o_p0 + NP0, o_g1 = o_g0 + NG0, o_p1 = o_g1 + NG1;
  static constexpr int o_mn = o_p1 + NP1, o_mx = o_mn + NMM;
  static constexpr int o_c1x = o_mx + NMM, o_c1y = o_c1x + NC1X;
  static constexpr int o_bu1 = o_c1y + NC1Y, o_bd1 = o_bu1 + 2, o_fx1 = o_bd1 + 2, o_fy1 = o_fx1 + 2;
  static constexpr int o_p2 = o_fy1 + 1;
  static constexpr int NP2 = NI == 3 ? 4 : 0;
  static constexpr int o_c2x = o_p2 + NP2, o_c2y = o_c2x + (NI == 3 ? 3 : 0);
  static constexpr int o_bu2 = o_c2y + (NI == 3 ? 3 : 0), o_bd2 = o_bu2 + (NI == 3 ? 2 : 0);
  static constexpr int o_fx2 = o_bd2 + (NI == 3 ? 2 : 0), o_fy2 = o_fx2 + (NI == 3 ? 2 : 0);
  static constexpr int total = o_fy2 + (NI == 3 ? 1 : 0);
};

__device__ __forceinline__ int rslot(int x, int n) { return ((x % n) + n) % n; }
__device__ __forceinline__ int pmod(int x, int P) { const int r = x % P; return r < 0 ? r + P : r; }

// One strip of one problem: columns [j0, j0 + W - 2H), rows [x0, x1).
template <class T, int NI, bool IGA, bool FCT, int NT, int H>
__device__ void strip(const prob<T> &A, int j0, int x0, int x1, T *sm) {
  constexpr int W = NT;
  using R = rows<NI, FCT>;
  const int c = threadIdx.x;            // column within the row buffers
  const int jg = pmod(j0 + c - H, A.P1);
  const bool inner = c > 0 && c < W - 1;  // has both neighbours in the buffer
  auto row = [&](int off, int n, int x) { return sm + (off + rslot(x, n)) * W; };
  auto P0 = [&](int x) { return row(R::o_p0, R::NP0, x); };
  auto G0 = [&](int x) { return row(R::o_g0, R::NG0, x); };
  auto G1 = [&](int x) { return row(R::o_g1, R::NG1, x); };
  auto P1 = [&](int x) { return row(R::o_p1, R::NP1, x); };
  auto MN = [&](int x) { return row(R::o_mn, R::NMM, x); };
  auto MX = [&](int x) { return row(R::o_mx, R::NMM, x); };
  auto C1X = [&](int x) { return row(R::o_c1x, R::NC1X, x); };
  auto C1Y = [&](int x) { return row(R::o_c1y, R::NC1Y, x); };
  auto BU1 = [&](int x) { return row(R::o_bu1, 2, x); };
  auto BD1 = [&](int x) { return row(R::o_bd1, 2, x); };
  auto FX1 = [&](int x) { return row(R::o_fx1, 2, x); };
  T *FY1 = sm + R::o_fy1 * W;
  auto P2 = [&](int x) { return row(R::o_p2, R::NP2 > 0 ? R::NP2 : 1, x); };
  auto C2X = [&](int x) { return row(R::o_c2x, 3, x); };
  auto C2Y = [&](int x) { return row(R::o_c2y, 3, x); };
  auto BU2 = [&](int x) { return row(R::o_bu2, 2, x); };
  auto BD2 = [&](int x) { return row(R::o_bd2, 2, x); };
  auto FX2 = [&](int x) { return row(R::o_fx2, 2, x); };
  T *FY2 = sm + R::o_fy2 * W;

  for (int q = c; q < R::total * W; q += NT) sm[q] = T(0);
  __syncthreads();

  auto load = [&](T *dst, const dfield<T> &f, int x) {
    const int xi = pmod(x, A.P0);
    f3::cp_async(dst + c, f.o + (long long)xi * f.s0 + jg);
  };
  auto nd2 = [](T a, T b, T cc, T d) -> T {  // ndy_psi (formulae_mpdata_psi_2d.hpp:188-240)
    if (IGA) return (a + b - cc - d) / T(4);
    return frac(a + b - cc - d, a + b + cc + d);
  };
  auto ndx = [](T p1, T p0) -> T {  // ndx_psi 2D (formulae_mpdata_psi_2d.hpp:127-185)
    if (IGA) return T(2) * (p1 - p0) / T(2);
    return T(2) * frac(p1 - p0, p1 + p0);
  };
  // antidiff 2D (formulae_mpdata_2d.hpp:256-277): C, GC1_bar_xy, ndx, ndy
  auto adiff = [&](T C, T gc1, T nx, T ny) -> T {
    return fabs(C) / T(2) * (T(1) - fabs(C) / T(1)) * nx - C * gc1 / T(2) * ny;
  };
  auto lim = [](T C, T bd_l, T bu_r, T bu_l, T bd_r) -> T {
    return C > T(0) ? mn(T(1), mn(bd_l, bu_r)) : mn(T(1), mn(bu_l, bd_r));
  };

  const int lag = NI == 3 ? 6 : 3;
  const int ts = x0 - (NI == 3 ? 5 : 3);
  const int te = x1 - 1 + lag;
  // prologue: psi^n rows ts-2..ts+1, GC_x faces ts-2..ts, GC_y rows ts-1..ts
  for (int x = ts - 2; x <= ts + 1; ++x) load(P0(x), A.in, x);
  for (int x = ts - 2; x <= ts; ++x) load(G0(x), A.g0, x);
  for (int x = ts - 1; x <= ts; ++x) load(G1(x), A.g1, x);
  f3::cp_commit();

  for (int t = ts; t <= te; ++t) {
    f3::cp_wait_all();
    __syncthreads();
    load(P0(t + 2), A.in, t + 2);
    load(G0(t + 1), A.g0, t + 1);
    load(G1(t + 1), A.g1, t + 1);
    f3::cp_commit();

    // psi1 row t, psi_min/max row t-1
    {
      const T *pm = P0(t - 1), *pc = P0(t), *pp = P0(t + 1), *gxm = G0(t - 1), *gxp = G0(t), *gy = G1(t);
      T v = T(0);
      if (inner) {
        const T cc = pc[c];
        const T fxp = flux(cc, pp[c], gxp[c]), fxm = flux(pm[c], cc, gxm[c]);
        const T fyp = flux(cc, pc[c + 1], gy[c]), fym = flux(pc[c - 1], cc, gy[c - 1]);
        v = cc + ((-fxp + fxm) + (-fyp + fym)) / T(1);
      }
      P1(t)[c] = v;
      if (FCT) {
        const T *qm = P0(t - 2), *qc = P0(t - 1), *qp = P0(t);
        T lo = T(0), hi = T(0);
        if (inner) {
          const T cc = qc[c];
          lo = mn(mn(mn(mn(qc[c + 1], qm[c]), cc), qp[c]), qc[c - 1]);
          hi = mx(mx(mx(mx(qc[c + 1], qm[c]), cc), qp[c]), qc[c - 1]);
        }
        MN(t - 1)[c] = lo;
        MX(t - 1)[c] = hi;
      }
    }
    __syncthreads();

    // C~1: x-face (t-1)+1/2 and y-faces of row t-1 (GC is the advector)
    {
      const int x = t - 1;
      const T *pm = P1(x - 1), *pc = P1(x), *pp = P1(x + 1);
      const T *g0m = G0(x - 1), *g0c = G0(x), *g1c = G1(x), *g1p = G1(x + 1);
      T vx = T(0), vy = T(0);
      if (inner) {
        // dim 0: frame a = x, b = y
        const T gc1x = (g1p[c] + g1c[c] + g1p[c - 1] + g1c[c - 1]) / T(4);
        vx = adiff(g0c[c], gc1x, ndx(pp[c], pc[c]), nd2(pp[c + 1], pc[c + 1], pp[c - 1], pc[c - 1]));
        // dim 1: frame a = y (face c+1/2), b = x
        const T gc1y = (g0c[c + 1] + g0c[c] + g0m[c + 1] + g0m[c]) / T(4);
        vy = adiff(g1c[c], gc1y, ndx(pc[c + 1], pc[c]), nd2(pp[c + 1], pp[c], pm[c + 1], pm[c]));
      }
      C1X(x)[c] = vx;
      C1Y(x)[c] = vy;
    }
    __syncthreads();

    // betas1 row t-2
    if (FCT) {
      const int x = t - 2;
      const T *pm = P1(x - 1), *pc = P1(x), *pp = P1(x + 1);
      const T *cxm = C1X(x - 1), *cxc = C1X(x), *cy = C1Y(x);
      T bu = T(0), bd = T(0);
      if (inner) {
        const T cc = pc[c];
        T fxm = cxm[c], fxp = cxc[c], fym = cy[c - 1], fyp = cy[c];
        if (!IGA) {
          fxm = flux(pm[c], cc, fxm); fxp = flux(cc, pp[c], fxp);
          fym = flux(pc[c - 1], cc, fym); fyp = flux(cc, pc[c + 1], fyp);
        }
        const T hi = mx(MX(x)[c], mx(pc[c + 1], mx(pm[c], mx(cc, mx(pp[c], pc[c - 1])))));
        const T lo = mn(MN(x)[c], mn(pc[c + 1], mn(pm[c], mn(cc, mn(pp[c], pc[c - 1])))));
        const T du = (pos(fxm) - neg(fxp)) + (pos(fym) - neg(fyp));
        const T dd = (pos(fxp) - neg(fxm)) + (pos(fyp) - neg(fym));
        bu = (hi - cc) * T(1) / (du + lims<T>::eps());
        bd = (cc - lo) * T(1) / (dd + lims<T>::eps());
      }
      BU1(x)[c] = bu;
      BD1(x)[c] = bd;
      __syncthreads();
    }

    // limited fluxes of iteration 1: x-face (t-3)+1/2, y-faces of row t-3
    {
      const int x = t - 3;
      const T *pc = P1(x), *pp = P1(x + 1);
      T fx = T(0), fy = T(0);
      if (inner) {
        T C = C1X(x)[c];
        if (FCT) C = C * lim(C, BD1(x)[c], BU1(x + 1)[c], BU1(x)[c], BD1(x + 1)[c]);
        fx = IGA ? C : flux(pc[c], pp[c], C);
        T D = C1Y(x)[c];
        if (FCT) D = D * lim(D, BD1(x)[c], BU1(x)[c + 1], BU1(x)[c], BD1(x)[c + 1]);
        fy = IGA ? D : flux(pc[c], pc[c + 1], D);
      }
      FX1(x)[c] = fx;
      FY1[c] = fy;
    }
    __syncthreads();

    // psi2 row t-3
    {
      const int x = t - 3;
      T v = T(0);
      if (inner) v = P1(x)[c] + ((-FX1(x)[c] + FX1(x - 1)[c]) + (-FY1[c] + FY1[c - 1])) / T(1);
      if (NI == 2) {
        if (x >= x0 && x < x1 && c >= H && c < W - H && j0 + c - H < A.P1) {
          const int j = j0 + c - H;
          A.out(x, j, 0) = v;
          if (x == 0) A.out(A.n0 - 1, j, 0) = v;
          if (j == 0) A.out(x, A.n1 - 1, 0) = v;
          if (x == 0 && j == 0) A.out(A.n0 - 1, A.n1 - 1, 0) = v;
        }
        continue;
      }
      P2(x)[c] = v;
    }
    if (NI == 3) {
      __syncthreads();
      // C~2 from psi2 and the unlimited C~1: x-face (t-4)+1/2, y-faces of row t-4
      {
        const int x = t - 4;
        const T *pm = P2(x - 1), *pc = P2(x), *pp = P2(x + 1);
        const T *g0m = C1X(x - 1), *g0c = C1X(x), *g1c = C1Y(x), *g1p = C1Y(x + 1);
        T vx = T(0), vy = T(0);
        if (inner) {
          const T gc1x = (g1p[c] + g1c[c] + g1p[c - 1] + g1c[c - 1]) / T(4);
          vx = adiff(g0c[c], gc1x, ndx(pp[c], pc[c]), nd2(pp[c + 1], pc[c + 1], pp[c - 1], pc[c - 1]));
          const T gc1y = (g0c[c + 1] + g0c[c] + g0m[c + 1] + g0m[c]) / T(4);
          vy = adiff(g1c[c], gc1y, ndx(pc[c + 1], pc[c]), nd2(pp[c + 1], pp[c], pm[c + 1], pm[c]));
        }
        C2X(x)[c] = vx;
        C2Y(x)[c] = vy;
      }
      __syncthreads();
      // betas2 row t-5 (psi_min/max still from psi^n, mpdata_fct_2d.hpp:31-46)
      if (FCT) {
        const int x = t - 5;
        const T *pm = P2(x - 1), *pc = P2(x), *pp = P2(x + 1);
        const T *cxm = C2X(x - 1), *cxc = C2X(x), *cy = C2Y(x);
        T bu = T(0), bd = T(0);
        if (inner) {
          const T cc = pc[c];
          T fxm = cxm[c], fxp = cxc[c], fym = cy[c - 1], fyp = cy[c];
          fxm = flux(pm[c], cc, fxm); fxp = flux(cc, pp[c], fxp);
          fym = flux(pc[c - 1], cc, fym); fyp = flux(cc, pc[c + 1], fyp);
          const T hi = mx(MX(x)[c], mx(pc[c + 1], mx(pm[c], mx(cc, mx(pp[c], pc[c - 1])))));
          const T lo = mn(MN(x)[c], mn(pc[c + 1], mn(pm[c], mn(cc, mn(pp[c], pc[c - 1])))));
          const T du = (pos(fxm) - neg(fxp)) + (pos(fym) - neg(fyp));
          const T dd = (pos(fxp) - neg(fxm)) + (pos(fyp) - neg(fym));
          bu = (hi - cc) * T(1) / (du + lims<T>::eps());
          bd = (cc - lo) * T(1) / (dd + lims<T>::eps());
        }
        BU2(x)[c] = bu;
        BD2(x)[c] = bd;
        __syncthreads();
      }
      // limited fluxes of iteration 2: x-face (t-6)+1/2, y-faces of row t-6
      {
        const int x = t - 6;
        const T *pc = P2(x), *pp = P2(x + 1);
        T fx = T(0), fy = T(0);
        if (inner) {
          T C = C2X(x)[c];
          if (FCT) C = C * lim(C, BD2(x)[c], BU2(x + 1)[c], BU2(x)[c], BD2(x + 1)[c]);
          fx = flux(pc[c], pp[c], C);
          T D = C2Y(x)[c];
          if (FCT) D = D * lim(D, BD2(x)[c], BU2(x)[c + 1], BU2(x)[c], BD2(x)[c + 1]);
          fy = flux(pc[c], pc[c + 1], D);
        }
        FX2(x)[c] = fx;
        FY2[c] = fy;
      }
      __syncthreads();
      {
        const int x = t - 6;
        if (inner && x >= x0 && x < x1 && c >= H && c < W - H && j0 + c - H < A.P1) {
          const T v = P2(x)[c] + ((-FX2(x)[c] + FX2(x - 1)[c]) + (-FY2[c] + FY2[c - 1])) / T(1);
          const int j = j0 + c - H;
          A.out(x, j, 0) = v;
          if (x == 0) A.out(A.n0 - 1, j, 0) = v;
          if (j == 0) A.out(x, A.n1 - 1, 0) = v;
          if (x == 0 && j == 0) A.out(A.n0 - 1, A.n1 - 1, 0) = v;
        }
      }
    }
  }
  f3::cp_wait_all();
  __syncthreads();
}

template <class T, int NI, bool IGA, bool FCT, int NT, int H>
__global__ void __launch_bounds__(NT) k_fused2d(const prob<T> A, int LX) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  const int j0 = blockIdx.x * (NT - 2 * H);
  const int x0 = blockIdx.y * LX;
  strip<T, NI, IGA, FCT, NT, H>(A, j0, x0, min(x0 + LX, A.P0), sm);
}

// work item of the batched launch: problem, strip origin and row range
struct item {
  int prob, j0, x0, x1;
};

// Persistent batched launch: a fixed grid of resident CTAs takes work items
// from a shared counter until the list is exhausted (no CTA waits on another).
template <class T, int NI, bool IGA, bool FCT, int NT, int H>
__global__ void __launch_bounds__(NT) k_fused2d_batched(const prob<T> *probs, const item *items, int n_items,
                                                        int *counter) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  __shared__ int next;
  for (;;) {
    if (threadIdx.x == 0) next = atomicAdd(counter, 1);
    __syncthreads();
    const int w = next;
    __syncthreads();
    if (w >= n_items) break;
    const item it = items[w];
    const prob<T> A = probs[it.prob];
    strip<T, NI, IGA, FCT, NT, H>(A, it.j0, it.x0, it.x1, sm);
  }
}

}  // namespace f2
}  // namespace mpdx
