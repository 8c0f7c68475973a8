// Fused 3D MPDATA step (n_iters = 2, options {0, fct, iga, iga|fct}, all
// boundaries cyclic): one kernel computes the upwind pass, the antidiffusive
// pseudo-velocities, the FCT limiter and the corrective pass with every
// intermediate on chip; DRAM sees psi^n and the advector in, psi^{n+1} out.
//
// Decomposition (2.5D blocking).  A CTA owns a canvas of CR x 64 points of the
// (j, k) plane -- output rows [3, CR-3) and output columns [4, 60) plus the
// halo the stencils need -- and marches along x over a chunk of planes.  Each
// thread owns one quad (4 consecutive k) of one canvas row for the whole march:
//   * x-neighbours: the thread's own values of neighbouring planes (registers,
//     or its own slot of a shared plane);
//   * k-neighbours: warp shuffles (16 lanes span one 64-column row);
//   * j-neighbours: shared-memory planes, only for the quantities a
//     neighbouring row needs.
// Per step t the CTA computes
//   psi1      = donor-cell(psi^n, GC)           plane t+1   (mpdata_osc_3d.hpp:181-197)
//   min/max of psi^n (7-point stencil)          plane t     (mpdata_fct_3d.hpp:31-55)
//   C~        = antidiff(psi1, GC)              x-face t+1/2, y/z faces of plane t (formulae_mpdata_3d.hpp:254-295)
//   beta_up / beta_dn                           plane t     (formulae_mpdata_fct_3d.hpp:48-143)
//   C_mono    = GC_mono(C~, betas)              x-face t-1/2, y/z faces of plane t-1 (formulae_mpdata_fct_3d.hpp:148-250)
//   psi^{n+1} = donor-cell(psi1, C_mono)        plane t-1
// Canvas points outside the valid part are computed from wrapped neighbours and
// never written; each stage loses at most one point of validity per side,
// which the 3-row / 4-column halo covers.
//
// Periodicity follows libmpdata++'s cyclic convention (bcond/cyclic_3d.hpp):
// with n points per axis the period is n-1 and point n-1 duplicates point 0.
// Expressions follow the reference's operand order; the FP64 instantiation is
// compiled without FMA contraction and reproduces the reference's rounding.
#pragma once

#include <cfloat>

#include "quad.cuh"
#include "state.cuh"

namespace mpdx {
namespace f3 {

using qd::q4;

template <class T> struct lims;
template <> struct lims<float> {
  __device__ static float tiny() { return FLT_MIN; }
  __device__ static float eps() { return FLT_EPSILON; }
};
template <> struct lims<double> {
  __device__ static double tiny() { return DBL_MIN; }
  __device__ static double eps() { return DBL_EPSILON; }
};

// scalar helpers (also used by the 2D kernel)
template <class T> __device__ __forceinline__ T pos(T x) { return fmax(T(0), x); }   // std::max(0, x)
template <class T> __device__ __forceinline__ T neg(T x) { return fmin(T(0), x); }   // std::min(0, x)
template <class T> __device__ __forceinline__ T mx(T a, T b) { return fmax(a, b); }
template <class T> __device__ __forceinline__ T mn(T a, T b) { return fmin(a, b); }
template <class T> __device__ __forceinline__ T flux(T pl, T pr, T c) { return pos(c) * pl + neg(c) * pr; }
template <class T> __device__ __forceinline__ T frac(T nom, T den) { return nom / (den + lims<T>::tiny()); }
__device__ __forceinline__ int wrap(int x, int P) { return x < 0 ? x + P : (x >= P ? x - P : x); }
__device__ __forceinline__ int pmod(int x, int P) { const int r = x % P; return r < 0 ? r + P : r; }

template <class T>
__device__ __forceinline__ void cp_async(T *smem, const T *gmem) {
  const unsigned s = unsigned(__cvta_generic_to_shared(smem));
  if (sizeof(T) == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// quad formulae --------------------------------------------------------------
template <class T>
__device__ __forceinline__ q4<T> qflux(const q4<T> &pl, const q4<T> &pr, const q4<T> &c) {
  return qd::fma(qd::pos(c), pl, qd::neg(c) * pr);
}
template <class T, bool IGA>
__device__ __forceinline__ q4<T> qndx(const q4<T> &p1, const q4<T> &p0) {  // formulae_mpdata_psi_3d.hpp:262-318
  if (IGA) return p1 - p0;
  return qd::bc<T>(T(2)) * ((p1 - p0) / ((p1 + p0) + qd::bc<T>(lims<T>::tiny())));
}
template <class T, bool IGA>
__device__ __forceinline__ q4<T> qnd4(const q4<T> &a, const q4<T> &b, const q4<T> &c, const q4<T> &d) {
  if (IGA) return (((a + b) - c) - d) * qd::bc<T>(T(0.25));
  return (((a + b) - c) - d) / ((((a + b) + c) + d) + qd::bc<T>(lims<T>::tiny()));
}
// |C|/2 (1 - |C|) ndx - C/2 (gc1 ndy + gc2 ndz)   (G = 1)
template <class T>
__device__ __forceinline__ q4<T> qadiff(const q4<T> &C, const q4<T> &gc1, const q4<T> &gc2, const q4<T> &nx,
                                        const q4<T> &ny, const q4<T> &nz) {
  const q4<T> h = qd::bc<T>(T(0.5));
  const q4<T> a = qd::qabs(C);
  return ((a * h) * (qd::bc<T>(T(1)) - a)) * nx - (C * h) * (gc1 * ny + gc2 * nz);
}
template <class T>
__device__ __forceinline__ q4<T> avg4(const q4<T> &a, const q4<T> &b, const q4<T> &c, const q4<T> &d) {
  return (((a + b) + c) + d) * qd::bc<T>(T(0.25));
}

template <class T>
struct args {
  dfield<T> in, out, g0, g1, g2;
  int P0, P1, P2;   // periods (n - 1)
  int n0, n1, n2;   // points per axis (duplicate at n - 1)
  int LX;           // planes per CTA
  int tiles_z;      // tiles along k
};

template <int CR>
struct canvas {
  static constexpr int CC = 64, N = CR * CC, TY = CR - 6, TZ = 56, NT = CR * 16;
  // shared planes, in units of N elements; rings hold every plane a step reads
  // plus the one being prefetched (cp.async, one step ahead)
  static constexpr int NS0 = 5, NG0 = 4, NG1 = 3;
  static constexpr int S0 = 0, G0 = S0 + NS0, G1 = G0 + NG0, G2 = G1 + NG1, S1 = G2 + NG1, CY = S1 + 3,
                       BU = CY + 1, BD = BU + 2, FY = BD + 2, total = FY + 1;
};

// asynchronous copy of one quad of field f (plane x, canvas row offset `ro`,
// columns kb..kb+3) into shared memory at dst
template <class T>
__device__ __forceinline__ void gcopy(T *dst, const dfield<T> &f, int x, long long ro, int kb, bool contig, const int *kc) {
  const T *p = f.o + (long long)x * f.s0 + ro;
  if (contig) {
#pragma unroll
    for (int h = 0; h < int(sizeof(T) * 4 / 16); ++h) {
      const unsigned sa = unsigned(__cvta_generic_to_shared(dst + h * (16 / sizeof(T))));
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(p + kb + h * (16 / sizeof(T))));
    }
  } else {
#pragma unroll
    for (int e = 0; e < 4; ++e) cp_async(dst + e, p + kc[e]);
  }
}

template <class T>
__device__ __forceinline__ T elem(const q4<T> &v, int e) {
  if constexpr (sizeof(T) == 4) return e == 0 ? v.a.x : e == 1 ? v.a.y : e == 2 ? v.b.x : v.b.y;
  else return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w;
}

template <class T, bool IGA, bool FCT, int CR>
__global__ void __launch_bounds__(CR * 16, 1) k_fused3d(const args<T> A) {
  using C = canvas<CR>;
  using Q = q4<T>;
  constexpr int N = C::N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);

  const int tid = threadIdx.x, lane = tid & 31;
  const int r = 2 * (tid >> 5) + (lane >> 4);   // canvas row
  const int q = lane & 15;                      // quad within the row
  const int me = r * C::CC + 4 * q;             // canvas offset of the own quad
  // rows r+1 / r-1; the outermost rows reuse their own (they are halo)
  const int upc = r < CR - 1 ? me + C::CC : me, dnc = r > 0 ? me - C::CC : me;

  const int tile = blockIdx.x;
  const int j0 = (tile / A.tiles_z) * C::TY, k0 = (tile % A.tiles_z) * C::TZ;
  const int x0 = blockIdx.y * A.LX, x1 = min(x0 + A.LX, A.P0);

  // fixed global offsets of the own quad
  const int jg = pmod(j0 - 3 + r, A.P1);
  const int kb = k0 - 4 + 4 * q;
  const bool contig = kb >= 0 && kb + 3 < A.P2;
  int kc[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) kc[e] = pmod(kb + e, A.P2);
  const long long ro_in = (long long)jg * A.in.s1, ro_g0 = (long long)jg * A.g0.s1;
  const long long ro_g1 = (long long)jg * A.g1.s1, ro_g2 = (long long)jg * A.g2.s1;

  auto plane = [&](int base, int nslots, int x) { return sm + (base + ((x % nslots) + nslots) % nslots) * N; };
  auto cp_in = [&](int x) { gcopy(plane(C::S0, C::NS0, x) + me, A.in, pmod(x, A.P0), ro_in, kb, contig, kc); };
  auto cp_g0 = [&](int x) { gcopy(plane(C::G0, C::NG0, x) + me, A.g0, pmod(x, A.P0), ro_g0, kb, contig, kc); };
  auto cp_g1 = [&](int x) { gcopy(plane(C::G1, C::NG1, x) + me, A.g1, pmod(x, A.P0), ro_g1, kb, contig, kc); };
  auto cp_g2 = [&](int x) { gcopy(plane(C::G2, C::NG1, x) + me, A.g2, pmod(x, A.P0), ro_g2, kb, contig, kc); };

  for (int p = tid; p < C::total * N; p += C::NT) sm[p] = T(0);
  __syncthreads();

  const int ts = x0 - 3;
  // prologue: everything step ts reads (psi^n planes ts-1..ts+2, GC_x faces
  // ts-1..ts+1, GC_y/GC_z planes ts..ts+1); each step then prefetches one plane ahead
  for (int x = ts - 1; x <= ts + 2; ++x) cp_in(x);
  for (int x = ts - 1; x <= ts + 1; ++x) cp_g0(x);
  for (int x = ts; x <= ts + 1; ++x) { cp_g1(x); cp_g2(x); }
  cp_commit();

  const Q zero = qd::bc<T>(T(0));
  Q p_m = zero, p_c = zero;  // own psi1 at planes t-1, t
  Q cx_m = zero, cy_m = zero, cz_m = zero, bu_m = zero, bd_m = zero, fx_prev = zero;

  for (int t = ts; t <= x1; ++t) {
    cp_wait_all();
    __syncthreads();
    cp_in(t + 3);
    cp_g0(t + 2);
    cp_g1(t + 2);
    cp_g2(t + 2);
    cp_commit();
    T *S0m = plane(C::S0, C::NS0, t - 1), *S0c = plane(C::S0, C::NS0, t), *S0p = plane(C::S0, C::NS0, t + 1);
    T *S0pp = plane(C::S0, C::NS0, t + 2);
    T *G0m = plane(C::G0, C::NG0, t - 1), *G0c = plane(C::G0, C::NG0, t), *G0p = plane(C::G0, C::NG0, t + 1);
    T *G1c = plane(C::G1, C::NG1, t), *G1p = plane(C::G1, C::NG1, t + 1);
    T *G2c = plane(C::G2, C::NG1, t), *G2p = plane(C::G2, C::NG1, t + 1);
    T *S1m = plane(C::S1, 3, t - 1), *S1c = plane(C::S1, 3, t), *S1p = plane(C::S1, 3, t + 1);
    T *CY = sm + C::CY * N, *FY = sm + C::FY * N;
    T *BUc = plane(C::BU, 2, t), *BDc = plane(C::BD, 2, t), *BUm = plane(C::BU, 2, t - 1), *BDm = plane(C::BD, 2, t - 1);

    // ---- A: psi1 at plane t+1 ----
    Q p_p;
    {
      const Q c = qd::lds(S0p + me), s0c = qd::lds(S0c + me), s0pp = qd::lds(S0pp + me);
      const Q g0c = qd::lds(G0c + me), g0p = qd::lds(G0p + me), g1p = qd::lds(G1p + me), g2p = qd::lds(G2p + me);
      const Q fxp = qflux(c, s0pp, g0p), fxm = qflux(s0c, c, g0c);
      const Q fyp = qflux(c, qd::lds(S0p + upc), g1p), fym = qflux(qd::lds(S0p + dnc), c, qd::lds(G1p + dnc));
      const Q fzp = qflux(c, qd::kp1(c), g2p), fzm = qflux(qd::km1(c), c, qd::km1(g2p));
      p_p = c + ((((-fxp) + fxm) + ((-fyp) + fym)) + ((-fzp) + fzm));
      qd::sts(S1p + me, p_p);
    }
    __syncthreads();

    // ---- B: C~ on x-face t+1/2, y- and z-faces of plane t ----
    Q cx_c, cy_c, cz_c;
    {
      const Q pc_up = qd::lds(S1c + upc), pc_dn = qd::lds(S1c + dnc), pm_up = qd::lds(S1m + upc);
      const Q pp_up = qd::lds(S1p + upc), pp_dn = qd::lds(S1p + dnc);
      const Q g0c = qd::lds(G0c + me), g0m = qd::lds(G0m + me);
      const Q g1c = qd::lds(G1c + me), g1p = qd::lds(G1p + me), g2c = qd::lds(G2c + me), g2p = qd::lds(G2p + me);
      const Q g1c_dn = qd::lds(G1c + dnc);
      // x-face (frame a = x, b = y, c = z)
      {
        const Q ny = qnd4<T, IGA>(pp_up, pc_up, pp_dn, pc_dn);
        const Q nz = qnd4<T, IGA>(qd::kp1(p_p), qd::kp1(p_c), qd::km1(p_p), qd::km1(p_c));
        const Q gc1 = avg4(g1p, g1c, qd::lds(G1p + dnc), g1c_dn);
        const Q gc2 = avg4(g2p, g2c, qd::km1(g2p), qd::km1(g2c));
        cx_c = qadiff(g0c, gc1, gc2, qndx<T, IGA>(p_p, p_c), ny, nz);
      }
      // y-face j+1/2 (frame a = y, b = z, c = x)
      {
        const Q ny = qnd4<T, IGA>(qd::kp1(pc_up), qd::kp1(p_c), qd::km1(pc_up), qd::km1(p_c));
        const Q nz = qnd4<T, IGA>(pp_up, p_p, pm_up, p_m);
        const Q g2c_up = qd::lds(G2c + upc);
        const Q gc1 = avg4(g2c_up, g2c, qd::km1(g2c_up), qd::km1(g2c));
        const Q gc2 = avg4(qd::lds(G0c + upc), g0c, qd::lds(G0m + upc), g0m);
        cy_c = qadiff(g1c, gc1, gc2, qndx<T, IGA>(pc_up, p_c), ny, nz);
        qd::sts(CY + me, cy_c);
      }
      // z-face k+1/2 (frame a = z, b = x, c = y)
      {
        const Q ny = qnd4<T, IGA>(qd::kp1(p_p), p_p, qd::kp1(p_m), p_m);
        const Q nz = qnd4<T, IGA>(qd::kp1(pc_up), pc_up, qd::kp1(pc_dn), pc_dn);
        const Q gc1 = avg4(qd::kp1(g0c), g0c, qd::kp1(g0m), g0m);
        const Q gc2 = avg4(qd::kp1(g1c), g1c, qd::kp1(g1c_dn), g1c_dn);
        cz_c = qadiff(g2c, gc1, gc2, qndx<T, IGA>(qd::kp1(p_c), p_c), ny, nz);
      }
    }
    __syncthreads();

    // ---- C: betas at plane t ----
    Q bu_c = zero, bd_c = zero;
    if (FCT) {
      // psi_min / psi_max of psi^n over the 7-point stencil at plane t (mpdata_fct_3d.hpp:31-55)
      Q mnq, mxq;
      {
        const Q s0c = qd::lds(S0c + me), s0p = qd::lds(S0p + me), s0m = qd::lds(S0m + me);
        const Q yp = qd::lds(S0c + upc), ym = qd::lds(S0c + dnc), zp = qd::kp1(s0c), zm = qd::km1(s0c);
        mnq = qd::qmin(qd::qmin(qd::qmin(qd::qmin(qd::qmin(qd::qmin(s0c, s0p), s0m), yp), ym), zp), zm);
        mxq = qd::qmax(qd::qmax(qd::qmax(qd::qmax(qd::qmax(qd::qmax(s0c, s0p), s0m), yp), ym), zp), zm);
      }
      const Q c = p_c;
      const Q xp = p_p, xm = p_m, yp = qd::lds(S1c + upc), ym = qd::lds(S1c + dnc), zp = qd::kp1(c), zm = qd::km1(c);
      Q fxm = cx_m, fxp = cx_c, fym = qd::lds(CY + dnc), fyp = cy_c, fzm = qd::km1(cz_c), fzp = cz_c;
      if (!IGA) {
        fxm = qflux(xm, c, fxm); fxp = qflux(c, xp, fxp);
        fym = qflux(ym, c, fym); fyp = qflux(c, yp, fyp);
        fzm = qflux(zm, c, fzm); fzp = qflux(c, zp, fzp);
      }
      const Q hi = qd::qmax(mxq, qd::qmax(c, qd::qmax(xp, qd::qmax(xm, qd::qmax(yp, qd::qmax(ym, qd::qmax(zp, zm)))))));
      const Q lo = qd::qmin(mnq, qd::qmin(yp, qd::qmin(xm, qd::qmin(c, qd::qmin(xp, qd::qmin(zp, qd::qmin(zm, ym)))))));
      const Q du = ((qd::pos(fxm) - qd::neg(fxp)) + (qd::pos(fym) - qd::neg(fyp))) + (qd::pos(fzm) - qd::neg(fzp));
      const Q dd = ((qd::pos(fxp) - qd::neg(fxm)) + (qd::pos(fyp) - qd::neg(fym))) + (qd::pos(fzp) - qd::neg(fzm));
      const Q e = qd::bc<T>(lims<T>::eps());
      bu_c = (hi - c) / (du + e);
      bd_c = (c - lo) / (dd + e);
      qd::sts(BUc + me, bu_c);
      qd::sts(BDc + me, bd_c);
    }
    __syncthreads();

    // ---- D: limited pseudo-velocities and fluxes at plane t-1 ----
    Q fxx, fzz;
    {
      Q Cx = cx_m, Cy = cy_m, Cz = cz_m;
      if (FCT) {
        Cx = Cx * qd::qlim(Cx, bd_m, bu_c, bu_m, bd_c);
        Cy = Cy * qd::qlim(Cy, bd_m, qd::lds(BUm + upc), bu_m, qd::lds(BDm + upc));
        Cz = Cz * qd::qlim(Cz, bd_m, qd::kp1(bu_m), bu_m, qd::kp1(bd_m));
      }
      if (IGA) {
        fxx = Cx; fzz = Cz;
        qd::sts(FY + me, Cy);
      } else {
        fxx = qflux(p_m, p_c, Cx);
        fzz = qflux(p_m, qd::kp1(p_m), Cz);
        qd::sts(FY + me, qflux(p_m, qd::lds(S1m + upc), Cy));
      }
    }
    __syncthreads();

    // ---- E: psi^{n+1} at plane t-1 ----
    {
      const int x = t - 1;
      const Q fy = qd::lds(FY + me), fyd = qd::lds(FY + dnc);
      const Q v = p_m + ((((-fxx) + fx_prev) + ((-fy) + fyd)) + ((-fzz) + qd::km1(fzz)));
      fx_prev = fxx;
      const int jrow = j0 - 3 + r;
      if (x >= x0 && x < x1 && r >= 3 && r < CR - 3 && jrow < A.P1 && q >= 1 && q < 15) {
        T *o = A.out.o + (long long)x * A.out.s0 + (long long)jrow * A.out.s1;
        if (contig) {
          qd::sts(o + kb, v);
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if (kb + e < A.P2) o[kb + e] = elem(v, e);
        }
        // cyclic duplicates at index n-1 (bcond/cyclic_3d.hpp convention)
        if (x == 0 || jrow == 0 || kb == 0) {
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int k = kb + e;
            if (k >= A.P2) continue;
            const T val = elem(v, e);
            const int xs[2] = {x, x == 0 ? A.n0 - 1 : -1};
            const int js[2] = {jrow, jrow == 0 ? A.n1 - 1 : -1};
            const int ks[2] = {k, k == 0 ? A.n2 - 1 : -1};
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
              for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int c = 0; c < 2; ++c)
                  if ((a | b | c) && xs[a] >= 0 && js[b] >= 0 && ks[c] >= 0) A.out(xs[a], js[b], ks[c]) = val;
          }
        }
      }
    }

    // shift the x-history
    p_m = p_c; p_c = p_p;
    cx_m = cx_c; cy_m = cy_c; cz_m = cz_c;
    bu_m = bu_c; bd_m = bd_c;
  }
  cp_wait_all();
}

}  // namespace f3
}  // namespace mpdx
