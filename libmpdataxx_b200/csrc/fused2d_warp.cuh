// Fused 2D MPDATA step, one warp per strip (n_iters 2 or 3; options {0, fct,
// iga, iga|fct} for n_iters = 2 and {0, fct} for n_iters = 3; all boundaries
// cyclic).
//
// Decomposition.  A warp owns a strip of 128 columns (j, contiguous in memory)
// of one problem -- lane l holds the quad of columns j0 - 4 HQ + 4 l .. +3 --
// and marches along x (i) over a chunk of rows.  Everything stays in
// registers: x-neighbours are the lane's own values of earlier rows, j-neighbours
// come from the neighbouring lanes by shuffles.  There is no shared memory and
// no block barrier; warps are independent.  Every stage loses at most one
// column of validity at each strip edge, so the HQ outermost quads on each
// side (4 columns per corrective iteration) are halo and are not written.
//
// Per step t (psi^n row t+1, GC_x face t+1/2 and GC_y row t arrive):
//   psi1(t)            donor-cell pass                         (mpdata_osc_2d.hpp:137-160)
//   C~x(t-1/2), C~y(t-1) antidiffusive velocities of psi1      (formulae_mpdata_2d.hpp:242-278)
//   betas(t-1)         with psi_min/max of psi^n at t-1         (formulae_mpdata_fct_2d.hpp:21-120,
//                                                               mpdata_fct_2d.hpp:31-46)
//   C_mono x(t-3/2), y(t-2), psi2(t-2)                         (formulae_mpdata_fct_2d.hpp:122-214)
// and for n_iters = 3 the same chain once more on psi2 with the unlimited
// C~ of the first iteration as advector (GC_unco, mpdata_common.hpp:40-47),
// ending with psi3(t-4).  Expressions follow the reference's operand order
// (as the one-thread-per-column kernel in fused2d.cuh does); the FP64
// instantiation is compiled without FMA contraction.
#pragma once

#include "fused2d.cuh"

namespace mpdx {
namespace f2w {

using f3::lims;
using f3::pmod;
using f3::qflux;
using qd::q4;

// halo quads per strip side and the valid columns of a strip
template <int NI> struct shape {
  static constexpr int HQ = NI == 3 ? 2 : 1;
  static constexpr int WV = 128 - 8 * HQ;   // columns written per strip
  static constexpr int LAG = NI == 3 ? 4 : 2;  // rows between psi^n arriving and psi^{n+1} leaving
};

// row x (already reduced modulo the period) of field f, columns jb..jb+3;
// jc holds the columns modulo the period for quads that straddle the seam
template <class T>
__device__ __forceinline__ q4<T> ldq(const dfield<T> &f, int x, int jb, bool contig, const int *jc) {
  const T *row = f.o + (long long)x * f.s0;
  if (contig) {
    if constexpr (sizeof(T) == 4) {
      const float4 v = __ldg(reinterpret_cast<const float4 *>(row + jb));
      return qd::mk(v.x, v.y, v.z, v.w);
    } else {
      const double2 a = __ldg(reinterpret_cast<const double2 *>(row + jb));
      const double2 b = __ldg(reinterpret_cast<const double2 *>(row + jb) + 1);
      return qd::mkd(a.x, a.y, b.x, b.y);
    }
  }
  if constexpr (sizeof(T) == 4) return qd::mk(__ldg(row + jc[0]), __ldg(row + jc[1]), __ldg(row + jc[2]), __ldg(row + jc[3]));
  else return qd::mkd(__ldg(row + jc[0]), __ldg(row + jc[1]), __ldg(row + jc[2]), __ldg(row + jc[3]));
}

template <class T>
__device__ __forceinline__ T el(const q4<T> &v, int e) {
  if constexpr (sizeof(T) == 4) return e == 0 ? v.a.x : e == 1 ? v.a.y : e == 2 ? v.b.x : v.b.y;
  else return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w;
}

// the quotients of the antidiffusive velocities: in FP32 the approximate-reciprocal
// quotient (__fdividef: within 2 ulp for the denominators here, sums of psi plus
// FLT_MIN, below 2^126; the FP32 FCT betas keep the correctly rounded quotient, on
// which the exact bound properties rest); in FP64 mpdx::rdivd for these and the betas.
__device__ __forceinline__ q4<float> adq(const q4<float> &a, const q4<float> &b) {
  return qd::mk(__fdividef(a.a.x, b.a.x), __fdividef(a.a.y, b.a.y), __fdividef(a.b.x, b.b.x), __fdividef(a.b.y, b.b.y));
}
// FP64: the quotient without the division's slow path (mpdx::rdivd, within one ulp)
__device__ __forceinline__ q4<double> adq(const q4<double> &a, const q4<double> &b) {
  return qd::mkd(rdivd(a.x, b.x), rdivd(a.y, b.y), rdivd(a.z, b.z), rdivd(a.w, b.w));
}
// ndx_psi 2D (formulae_mpdata_psi_2d.hpp:127-185): iga 2 (p1 - p0) / 2 = p1 - p0
template <class T, bool IGA>
__device__ __forceinline__ q4<T> ndx(const q4<T> &p1, const q4<T> &p0) {
  if (IGA) return p1 - p0;
  return qd::bc<T>(T(2)) * adq(p1 - p0, (p1 + p0) + qd::bc<T>(lims<T>::tiny()));
}
// ndy_psi 2D (formulae_mpdata_psi_2d.hpp:188-240)
template <class T, bool IGA>
__device__ __forceinline__ q4<T> ndy(const q4<T> &a, const q4<T> &b, const q4<T> &c, const q4<T> &d) {
  if (IGA) return (((a + b) - c) - d) * qd::bc<T>(T(0.25));
  return adq(((a + b) - c) - d, (((a + b) + c) + d) + qd::bc<T>(lims<T>::tiny()));
}
// antidiff 2D (formulae_mpdata_2d.hpp:256-277) with G = 1:
// |C|/2 (1 - |C|) ndx - (C gc1)/2 ndy
template <class T>
__device__ __forceinline__ q4<T> adiff(const q4<T> &C, const q4<T> &gc1, const q4<T> &nx, const q4<T> &ny) {
  const q4<T> h = qd::bc<T>(T(0.5));
  const q4<T> a = qd::qabs(C);
  return ((a * h) * (qd::bc<T>(T(1)) - a)) * nx - ((C * gc1) * h) * ny;
}

// betas (formulae_mpdata_fct_2d.hpp:21-120): c = psi at the point, xm/xp/ym/yp its
// neighbours, mnq/mxq psi_min/max of psi^n, f* the (antidiffusive) fluxes through
// its four faces
template <class T>
__device__ __forceinline__ void betas(const q4<T> &c, const q4<T> &xm, const q4<T> &xp, const q4<T> &ym, const q4<T> &yp,
                                      const q4<T> &mnq, const q4<T> &mxq, const q4<T> &fxm, const q4<T> &fxp,
                                      const q4<T> &fym, const q4<T> &fyp, q4<T> &bu, q4<T> &bd) {
  // max(psi_max, psi(i,j+1), psi(i-1,j), psi(i,j), psi(i+1,j), psi(i,j-1)) as a right fold
  const q4<T> hi = qd::qmax(mxq, qd::qmax(yp, qd::qmax(xm, qd::qmax(c, qd::qmax(xp, ym)))));
  const q4<T> lo = qd::qmin(mnq, qd::qmin(yp, qd::qmin(xm, qd::qmin(c, qd::qmin(xp, ym)))));
  const q4<T> du = (qd::pos(fxm) - qd::neg(fxp)) + (qd::pos(fym) - qd::neg(fyp));
  const q4<T> dd = (qd::pos(fxp) - qd::neg(fxm)) + (qd::pos(fyp) - qd::neg(fym));
  const q4<T> e = qd::bc<T>(lims<T>::eps());
  if constexpr (sizeof(T) == 8) {  // FP64: mpdx::rdivd, as the antidiffusive velocities
    bu = adq(hi - c, du + e);
    bd = adq(c - lo, dd + e);
  } else {
    bu = (hi - c) / (du + e);
    bd = (c - lo) / (dd + e);
  }
}

// psi_min / psi_max of psi^n over the 5-point stencil (mpdata_fct_2d.hpp:31-46):
// min(psi(i,j+1), psi(i-1,j), psi(i,j), psi(i+1,j), psi(i,j-1)) as a left fold
template <class T>
__device__ __forceinline__ void minmax(const q4<T> &xm, const q4<T> &c, const q4<T> &xp, q4<T> &mnq, q4<T> &mxq) {
  const q4<T> yp = qd::kp1(c), ym = qd::km1(c);
  mnq = qd::qmin(qd::qmin(qd::qmin(qd::qmin(yp, xm), c), xp), ym);
  mxq = qd::qmax(qd::qmax(qd::qmax(qd::qmax(yp, xm), c), xp), ym);
}

// one strip of one problem: columns [j0, j0 + WV), rows [x0, x1)
template <class T, int NI, bool IGA, bool FCT>
__device__ __forceinline__ void march(const f2::prob<T> &A, int j0, int x0, int x1) {
  static_assert(NI == 2 || (NI == 3 && !IGA), "n_iters 3 is built without iga");
  using Q = q4<T>;
  using S = shape<NI>;
  const int lane = threadIdx.x & 31;
  const int jb = j0 - 4 * S::HQ + 4 * lane;
  const bool contig = jb >= 0 && jb + 3 < A.P1;
  int jc[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) jc[e] = pmod(jb + e, A.P1);
  auto L = [&](const dfield<T> &f, int x) { return ldq(f, pmod(x, A.P0), jb, contig, jc); };

  const int ts = x0 - S::LAG, te = x1 - 1 + S::LAG;
  const Q zero = qd::bc<T>(T(0));

  // psi^n rows t-2..t, GC_x faces t-2, t-1 (index i = face i+1/2), GC_y row t-1
  Q pn2 = L(A.in, ts - 2), pn1 = L(A.in, ts - 1), pn0 = L(A.in, ts);
  Q gx2 = L(A.g0, ts - 2), gx1 = L(A.g0, ts - 1), gy1 = L(A.g1, ts - 1);
  // next row's inputs, loaded one step ahead
  Q n_pn = L(A.in, ts + 1), n_gx = L(A.g0, ts), n_gy = L(A.g1, ts);
  Q p1_2 = zero, p1_1 = zero;          // psi1 rows t-2, t-1
  Q cx2 = zero, cy2 = zero;            // C~x face index t-2, C~y row t-2
  Q bu2 = zero, bd2 = zero;            // betas row t-2
  Q fx3 = zero;                        // limited x flux, face index t-3
  // second iteration (n_iters = 3)
  Q cx4 = zero, cx3 = zero, cy3 = zero;  // unlimited C~1: x faces t-4, t-3; y row t-3
  Q mn2 = zero, mx2 = zero, mn3 = zero, mx3 = zero;  // psi_min/max rows t-2, t-3
  Q p2_4 = zero, p2_3 = zero;          // psi2 rows t-4, t-3
  Q dx4 = zero, dy4 = zero;            // C~2: x face t-4, y row t-4
  Q eu4 = zero, ed4 = zero;            // betas2 row t-4
  Q gx5 = zero;                        // limited x flux of iteration 2, face t-5

  Q fx_up = qflux(pn1, pn0, gx1);     // upwind x flux through face ts-1/2
  // rows loaded one step ahead (psi^n t+2, Courant components t+1), reduced modulo
  // the period by a compare per step
  int xin = pmod(ts + 2, A.P0), xg = pmod(ts + 1, A.P0);
  for (int t = ts; t <= te; ++t) {
    const Q pnp = n_pn, gx0 = n_gx, gy0 = n_gy;  // psi^n row t+1, GC_x face t, GC_y row t
    if (t < te) {
      n_pn = ldq(A.in, xin, jb, contig, jc);
      n_gx = ldq(A.g0, xg, jb, contig, jc);
      n_gy = ldq(A.g1, xg, jb, contig, jc);
    }
    if (++xin == A.P0) xin = 0;
    if (++xg == A.P0) xg = 0;

    // ---- psi1(t) (donor-cell, donorcell_formulae.hpp:104-130) ----
    // every face flux is evaluated once: the flux through face t-1/2 is the one
    // computed for face t+1/2 of the previous row, the flux through j-1/2 of a
    // column the j+1/2 flux of its left neighbour (the same operands, the same value)
    const Q fxp = qflux(pn0, pnp, gx0), fxm = fx_up;
    const Q fyp = qflux(pn0, qd::kp1(pn0), gy0), fym = qd::km1(fyp);
    fx_up = fxp;
    const Q p1_0 = pn0 + (((-fxp) + fxm) + ((-fyp) + fym));

    // ---- C~x face t-1 (between rows t-1 and t), C~y row t-1 ----
    const Q cx1 = adiff(gx1, f3::avg4(gy0, gy1, qd::km1(gy0), qd::km1(gy1)), ndx<T, IGA>(p1_0, p1_1),
                        ndy<T, IGA>(qd::kp1(p1_0), qd::kp1(p1_1), qd::km1(p1_0), qd::km1(p1_1)));
    const Q cy1 = adiff(gy1, f3::avg4(qd::kp1(gx1), gx1, qd::kp1(gx2), gx2), ndx<T, IGA>(qd::kp1(p1_1), p1_1),
                        ndy<T, IGA>(qd::kp1(p1_0), p1_0, qd::kp1(p1_2), p1_2));

    // ---- betas row t-1 ----
    Q bu1 = zero, bd1 = zero, mn1 = zero, mx1 = zero;
    if (FCT) {
      minmax(pn2, pn1, pn0, mn1, mx1);
      Q fm = cx2, fp = cx1, gm = qd::km1(cy1), gp = cy1;
      const Q ym = qd::km1(p1_1), yp = qd::kp1(p1_1);
      if (!IGA) {
        fm = qflux(p1_2, p1_1, fm); fp = qflux(p1_1, p1_0, fp);
        gm = qflux(ym, p1_1, gm); gp = qflux(p1_1, yp, gp);
      }
      betas(p1_1, p1_2, p1_0, ym, yp, mn1, mx1, fm, fp, gm, gp, bu1, bd1);
    }

    // ---- limited fluxes: x face t-2, y row t-2; psi2(t-2) ----
    Q fx = cx2, fy = cy2;
    if (FCT) {
      fx = fx * qd::qlim(fx, bd2, bu1, bu2, bd1);
      fy = fy * qd::qlim(fy, bd2, qd::kp1(bu2), bu2, qd::kp1(bd2));
    }
    if (!IGA) {
      fx = qflux(p1_2, p1_1, fx);
      fy = qflux(p1_2, qd::kp1(p1_2), fy);
    }
    const Q p2_2 = p1_2 + (((-fx) + fx3) + ((-fy) + qd::km1(fy)));

    Q out = p2_2;
    int xo = t - 2;
    if (NI == 3) {
      // ---- C~2 from psi2 and the unlimited C~1: x face t-3, y row t-3 ----
      const Q dx3 = adiff(cx3, f3::avg4(cy2, cy3, qd::km1(cy2), qd::km1(cy3)), ndx<T, false>(p2_2, p2_3),
                          ndy<T, false>(qd::kp1(p2_2), qd::kp1(p2_3), qd::km1(p2_2), qd::km1(p2_3)));
      const Q dy3 = adiff(cy3, f3::avg4(qd::kp1(cx3), cx3, qd::kp1(cx4), cx4), ndx<T, false>(qd::kp1(p2_3), p2_3),
                          ndy<T, false>(qd::kp1(p2_2), p2_2, qd::kp1(p2_4), p2_4));
      // ---- betas2 row t-3 (bounds still from psi^n, mpdata_fct_2d.hpp:31-46) ----
      Q eu3 = zero, ed3 = zero;
      if (FCT) {
        const Q ym = qd::km1(p2_3), yp = qd::kp1(p2_3);
        betas(p2_3, p2_4, p2_2, ym, yp, mn3, mx3, qflux(p2_4, p2_3, dx4), qflux(p2_3, p2_2, dx3),
              qflux(ym, p2_3, qd::km1(dy3)), qflux(p2_3, yp, dy3), eu3, ed3);
      }
      // ---- limited fluxes of iteration 2: x face t-4, y row t-4; psi3(t-4) ----
      Q hx = dx4, hy = dy4;
      if (FCT) {
        hx = hx * qd::qlim(hx, ed4, eu3, eu4, ed3);
        hy = hy * qd::qlim(hy, ed4, qd::kp1(eu4), eu4, qd::kp1(ed4));
      }
      hx = qflux(p2_4, p2_3, hx);
      hy = qflux(p2_4, qd::kp1(p2_4), hy);
      out = p2_4 + (((-hx) + gx5) + ((-hy) + qd::km1(hy)));
      xo = t - 4;
      // shift the second iteration's history
      gx5 = hx; dx4 = dx3; dy4 = dy3; eu4 = eu3; ed4 = ed3;
      p2_4 = p2_3; p2_3 = p2_2;
      cx4 = cx3; cx3 = cx2; cy3 = cy2;
      mn3 = mn2; mx3 = mx2; mn2 = mn1; mx2 = mx1;
    }

    // ---- store row xo ----
    if (xo >= x0 && xo < x1 && lane >= S::HQ && lane < 32 - S::HQ) {
      T *o = A.out.o + (long long)xo * A.out.s0;
      if (contig) {
        qd::sts(o + jb, out);
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (jb + e < A.P1) o[jb + e] = el(out, e);
      }
      // cyclic duplicates at index n-1 (bcond/cyclic_2d.hpp convention)
      if (xo == 0 || jb == 0) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int j = jb + e;
          if (j >= A.P1) continue;
          const T v = el(out, e);
          if (xo == 0) A.out(A.n0 - 1, j, 0) = v;
          if (j == 0) A.out(xo, A.n1 - 1, 0) = v;
          if (xo == 0 && j == 0) A.out(A.n0 - 1, A.n1 - 1, 0) = v;
        }
      }
    }

    // ---- shift the first iteration's history ----
    pn2 = pn1; pn1 = pn0; pn0 = pnp;
    gx2 = gx1; gx1 = gx0; gy1 = gy0;
    p1_2 = p1_1; p1_1 = p1_0;
    cx2 = cx1; cy2 = cy1;
    bu2 = bu1; bd2 = bd1;
    fx3 = fx;
  }
}

// resident CTAs of 4 warps per SM that the register budget is sized for
// (FP64 quads take twice the registers of FP32 ones)
template <class T, int NI>
constexpr int kMinBlocks2 = sizeof(T) == 4 ? (NI == 3 ? 2 : 4) : (NI == 3 ? 1 : 2);

// The one 2D kernel, for the single-problem and the batched advance alike:
// persistent warps take work items (problem, strip, rows) from counter[0] until
// the list of n_items is exhausted (no warp waits on another).  One kernel with
// one call site of march keeps the FP32 arithmetic of both advances the same
// compiled code, so their results agree bit for bit (FMA contraction is decided
// once).  The last warp to finish re-arms the counter (counter[1] counts the
// finished warps), so consecutive launches on one stream need no reset.
template <class T, int NI, bool IGA, bool FCT>
__global__ void __launch_bounds__(128, kMinBlocks2<T, NI>) k_fused2d_w(const f2::prob<T> *probs, const f2::item *items,
                                                                   int n_items, int *counter) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    int q = 0;
    if (lane == 0) q = atomicAdd(counter, 1);
    q = __shfl_sync(0xffffffffu, q, 0);
    if (q >= n_items) break;
    const f2::item it = items[q];
    const f2::prob<T> A = probs[it.prob];  // the descriptor in registers
    march<T, NI, IGA, FCT>(A, it.j0, it.x0, it.x1);
  }
  if (lane == 0) {
    __threadfence();  // this warp's last take from counter[0] precedes its count
    const int n_warps = int(gridDim.x) * int(blockDim.x >> 5);
    if (atomicAdd(counter + 1, 1) == n_warps - 1) {
      counter[0] = 0;
      counter[1] = 0;
    }
  }
}

}  // namespace f2w
}  // namespace mpdx
