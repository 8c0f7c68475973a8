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
// donor-cell flux pos(C) psi_l + neg(C) psi_r (donorcell_formulae.hpp:25-34),
// evaluated as C * (C > 0 ? psi_l : psi_r): one of the two products is an
// exact zero, so both forms give the same value for finite operands
template <class T>
__device__ __forceinline__ q4<T> qflux(const q4<T> &pl, const q4<T> &pr, const q4<T> &c) {
  return c * qd::sel_pos(c, pl, pr);
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

// slot bookkeeping of a ring of NS planes: base = slot of the oldest plane in use
template <int NS>
struct ring {
  int base;
  __device__ __forceinline__ int at(int i) const { const int v = base + i; return v >= NS ? v - NS : v; }
  __device__ __forceinline__ void next() { base = base + 1 == NS ? 0 : base + 1; }
};

template <int CR>
struct canvas {
  static constexpr int CC = 64, N = CR * CC, TY = CR - 6, TZ = 56, NT = CR * 16;
  // shared planes, in units of N elements; rings hold every plane a step reads
  // plus the one being prefetched (cp.async, one step ahead)
  static constexpr int NS0 = 5, NG0 = 4, NG1 = 3;
  static constexpr int S0 = 0, G0 = S0 + NS0, G1 = G0 + NG0, G2 = G1 + NG1, S1 = G2 + NG1, CY = S1 + 3,
                       BU = CY + 2, BD = BU + 2, total = BD + 2;
};

// asynchronous copy of one quad of field f (plane x, canvas row offset `ro`,
// columns kb..kb+3) into shared memory at dst
template <class T>
__device__ __forceinline__ void gcopy_row(T *dst, const T *p, int kb, bool contig, const int *kc) {
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
// the same for plane x of field f (x already reduced modulo the period)
template <class T>
__device__ __forceinline__ void gcopy(T *dst, const dfield<T> &f, int x, long long ro, int kb, bool contig, const int *kc) {
  gcopy_row(dst, f.o + (long long)x * f.s0 + ro, kb, contig, kc);
}

// pointer to one row of successive planes of a periodic field, advanced a plane
// at a time with the wrap done by a compare (no integer division in the loop)
template <class T>
struct plane_walker {
  const T *p;
  long long step, wrap;
  int x, P;
  __device__ void init(const dfield<T> &f, int x0, int P_, long long ro) {
    P = P_;
    x = pmod(x0, P);
    step = f.s0;
    wrap = (long long)P * f.s0;
    p = f.o + (long long)x * f.s0 + ro;
  }
  __device__ __forceinline__ void next() {
    p += step;
    if (++x == P) { x = 0; p -= wrap; }
  }
};

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
  // canvas offset of row r+d (the outermost rows stand in for missing ones: they are halo)
  auto R = [&](int d) { const int rr = r + d; return rr >= 0 && rr < CR ? me + d * C::CC : me; };
  const int up = R(1), dn = R(-1);

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
  auto cp_in = [&](T *dst, int x) { gcopy(dst + me, A.in, pmod(x, A.P0), ro_in, kb, contig, kc); };
  auto cp_g0 = [&](T *dst, int x) { gcopy(dst + me, A.g0, pmod(x, A.P0), ro_g0, kb, contig, kc); };
  auto cp_g1 = [&](T *dst, int x) { gcopy(dst + me, A.g1, pmod(x, A.P0), ro_g1, kb, contig, kc); };
  auto cp_g2 = [&](T *dst, int x) { gcopy(dst + me, A.g2, pmod(x, A.P0), ro_g2, kb, contig, kc); };

  for (int p = tid; p < C::total * N; p += C::NT) sm[p] = T(0);
  __syncthreads();

  const int ts = x0 - 3;
  // prologue: everything step ts reads (psi^n planes ts-1..ts+2, GC_x faces
  // ts-1..ts+1, GC_y/GC_z planes ts..ts+1); each step then prefetches one plane ahead
  for (int x = ts - 1; x <= ts + 2; ++x) cp_in(plane(C::S0, C::NS0, x), x);
  for (int x = ts - 1; x <= ts + 1; ++x) cp_g0(plane(C::G0, C::NG0, x), x);
  for (int x = ts; x <= ts + 1; ++x) { cp_g1(plane(C::G1, C::NG1, x), x); cp_g2(plane(C::G2, C::NG1, x), x); }
  cp_commit();

  const Q zero = qd::bc<T>(T(0));
  Q p_m = zero, p_c = zero;  // own psi1 at planes t-1, t
  Q cx_m = zero, cy_m = zero, cz_m = zero, bu_m = zero, bd_m = zero, fx_prev = zero;
  // ring slots of the oldest plane each step reads: psi^n and GC_x from t-1,
  // GC_y / GC_z from t, psi1 / C~_y / betas from t-1
  auto slot0 = [](int x, int n) { return ((x % n) + n) % n; };
  ring<C::NS0> r_s0{slot0(ts - 1, C::NS0)};
  ring<C::NG0> r_g0{slot0(ts - 1, C::NG0)};
  ring<C::NG1> r_g1{slot0(ts, C::NG1)};
  ring<3> r_s1{slot0(ts - 1, 3)};
  ring<2> r_2{slot0(ts - 1, 2)};

  // Barriers per step: one before the step reads the planes of the previous
  // step, one after psi1(t+1) is stored, and (FCT) one after the y-face
  // pseudo-velocities are stored, so that each row reads the face below it.
  // rows of the planes the steps prefetch: psi^n t+3, the Courant components t+2
  plane_walker<T> w_in, w_g0, w_g1, w_g2;
  w_in.init(A.in, ts + 3, A.P0, ro_in);
  w_g0.init(A.g0, ts + 2, A.P0, ro_g0);
  w_g1.init(A.g1, ts + 2, A.P0, ro_g1);
  w_g2.init(A.g2, ts + 2, A.P0, ro_g2);
  for (int t = ts; t <= x1; ++t) {
    cp_wait_all();
    __syncthreads();
    T *const s0b = sm + C::S0 * N, *const g0b = sm + C::G0 * N, *const g1b = sm + C::G1 * N, *const g2b = sm + C::G2 * N;
    gcopy_row(s0b + r_s0.at(4) * N + me, w_in.p, kb, contig, kc);
    gcopy_row(g0b + r_g0.at(3) * N + me, w_g0.p, kb, contig, kc);
    gcopy_row(g1b + r_g1.at(2) * N + me, w_g1.p, kb, contig, kc);
    gcopy_row(g2b + r_g1.at(2) * N + me, w_g2.p, kb, contig, kc);
    cp_commit();
    w_in.next(); w_g0.next(); w_g1.next(); w_g2.next();
    const T *S0m = s0b + r_s0.at(0) * N, *S0c = s0b + r_s0.at(1) * N, *S0p = s0b + r_s0.at(2) * N;
    const T *S0pp = s0b + r_s0.at(3) * N;
    const T *G0m = g0b + r_g0.at(0) * N, *G0c = g0b + r_g0.at(1) * N, *G0p = g0b + r_g0.at(2) * N;
    const T *G1c = g1b + r_g1.at(0) * N, *G1p = g1b + r_g1.at(1) * N;
    const T *G2c = g2b + r_g1.at(0) * N, *G2p = g2b + r_g1.at(1) * N;
    T *const s1b = sm + C::S1 * N;
    const T *S1m = s1b + r_s1.at(0) * N, *S1c = s1b + r_s1.at(1) * N;
    T *S1p = s1b + r_s1.at(2) * N;
    const int sc = r_2.at(1) * N, sm1 = r_2.at(0) * N;
    T *CYc = sm + C::CY * N + sc, *BUc = sm + C::BU * N + sc, *BDc = sm + C::BD * N + sc;
    const T *CYm = sm + C::CY * N + sm1, *BUm = sm + C::BU * N + sm1, *BDm = sm + C::BD * N + sm1;
    r_s0.next(); r_g0.next(); r_g1.next(); r_s1.next(); r_2.next();

    // ---- A: psi1 at plane t+1 (mpdata_osc_3d.hpp:181-197) ----
    auto psi1_row = [&](int o, int om, int op) {  // canvas offsets of the row and its neighbours
      const Q c = qd::lds(S0p + o);
      const Q fxp = qflux(c, qd::lds(S0pp + o), qd::lds(G0p + o));
      const Q fxm = qflux(qd::lds(S0c + o), c, qd::lds(G0c + o));
      const Q fyp = qflux(c, qd::lds(S0p + op), qd::lds(G1p + o));
      const Q fym = qflux(qd::lds(S0p + om), c, qd::lds(G1p + om));
      const Q g2p = qd::lds(G2p + o);
      const Q fzp = qflux(c, qd::kp1(c), g2p), fzm = qflux(qd::km1(c), c, qd::km1(g2p));
      return c + ((((-fxp) + fxm) + ((-fyp) + fym)) + ((-fzp) + fzm));
    };
    const Q p_p = psi1_row(me, dn, up);
    qd::sts(S1p + me, p_p);
    __syncthreads();
    const Q pp_up = qd::lds(S1p + up), pp_dn = qd::lds(S1p + dn);

    // ---- B: C~ on the own x-face t+1/2, y-face j+1/2 and z-faces of plane t ----
    const Q pc_up = qd::lds(S1c + up), pc_dn = qd::lds(S1c + dn);
    Q cx_c, cy_c, cz_c;
    {
      const Q pm_up = qd::lds(S1m + up);
      const Q g0c = qd::lds(G0c + me), g0m = qd::lds(G0m + me);
      const Q g1c = qd::lds(G1c + me), g1c_dn = qd::lds(G1c + dn), g2c = qd::lds(G2c + me);
      // x-face (frame a = x, b = y, c = z)
      {
        const Q g2p = qd::lds(G2p + me);
        const Q ny = qnd4<T, IGA>(pp_up, pc_up, pp_dn, pc_dn);
        const Q nz = qnd4<T, IGA>(qd::kp1(p_p), qd::kp1(p_c), qd::km1(p_p), qd::km1(p_c));
        const Q gc1 = avg4(qd::lds(G1p + me), g1c, qd::lds(G1p + dn), g1c_dn);
        const Q gc2 = avg4(g2p, g2c, qd::km1(g2p), qd::km1(g2c));
        cx_c = qadiff(g0c, gc1, gc2, qndx<T, IGA>(p_p, p_c), ny, nz);
      }
      // y-face j+1/2 (frame a = y, b = z, c = x)
      {
        const Q ny = qnd4<T, IGA>(qd::kp1(pc_up), qd::kp1(p_c), qd::km1(pc_up), qd::km1(p_c));
        const Q nz = qnd4<T, IGA>(pp_up, p_p, pm_up, p_m);
        const Q g2c_up = qd::lds(G2c + up);
        const Q gc1 = avg4(g2c_up, g2c, qd::km1(g2c_up), qd::km1(g2c));
        const Q gc2 = avg4(qd::lds(G0c + up), g0c, qd::lds(G0m + up), g0m);
        cy_c = qadiff(g1c, gc1, gc2, qndx<T, IGA>(pc_up, p_c), ny, nz);
        qd::sts(CYc + me, cy_c);
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

    // ---- C: betas at plane t (formulae_mpdata_fct_3d.hpp:48-143) ----
    Q bu_c = zero, bd_c = zero;
    if (FCT) {
      // C~ on the y-face j-1/2 below the own row: stored by row r-1 in stage B
      __syncthreads();
      const Q cy_dn = qd::lds(CYc + dn);
      // psi_min / psi_max of psi^n over the 7-point stencil at plane t (mpdata_fct_3d.hpp:31-55)
      Q mnq, mxq;
      {
        const Q s0c = qd::lds(S0c + me), s0p = qd::lds(S0p + me), s0m = qd::lds(S0m + me);
        const Q yp = qd::lds(S0c + up), ym = qd::lds(S0c + dn), zp = qd::kp1(s0c), zm = qd::km1(s0c);
        mnq = qd::qmin(qd::qmin(qd::qmin(qd::qmin(qd::qmin(qd::qmin(s0c, s0p), s0m), yp), ym), zp), zm);
        mxq = qd::qmax(qd::qmax(qd::qmax(qd::qmax(qd::qmax(qd::qmax(s0c, s0p), s0m), yp), ym), zp), zm);
      }
      const Q c = p_c;
      const Q xp = p_p, xm = p_m, yp = pc_up, ym = pc_dn, zp = qd::kp1(c), zm = qd::km1(c);
      Q fxm = cx_m, fxp = cx_c, fym = cy_dn, fyp = cy_c, fzm = qd::km1(cz_c), fzp = cz_c;
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

    // ---- D: limited fluxes at plane t-1 (formulae_mpdata_fct_3d.hpp:148-250) ----
    Q fxx, fyu, fyd, fzz;
    {
      Q Cx = cx_m, Cy = cy_m, Cyd = qd::lds(CYm + dn), Cz = cz_m;
      if (FCT) {
        const Q bu_dn = qd::lds(BUm + dn), bd_dn = qd::lds(BDm + dn);
        Cx = Cx * qd::qlim(Cx, bd_m, bu_c, bu_m, bd_c);
        Cy = Cy * qd::qlim(Cy, bd_m, qd::lds(BUm + up), bu_m, qd::lds(BDm + up));
        Cyd = Cyd * qd::qlim(Cyd, bd_dn, bu_m, bu_dn, bd_m);
        Cz = Cz * qd::qlim(Cz, bd_m, qd::kp1(bu_m), bu_m, qd::kp1(bd_m));
      }
      if (IGA) {
        fxx = Cx; fyu = Cy; fyd = Cyd; fzz = Cz;
      } else {
        fxx = qflux(p_m, p_c, Cx);
        fyu = qflux(p_m, qd::lds(S1m + up), Cy);
        fyd = qflux(qd::lds(S1m + dn), p_m, Cyd);
        fzz = qflux(p_m, qd::kp1(p_m), Cz);
      }
    }

    // ---- E: psi^{n+1} at plane t-1 ----
    {
      const int x = t - 1;
      const Q v = p_m + ((((-fxx) + fx_prev) + ((-fyu) + fyd)) + ((-fzz) + qd::km1(fzz)));
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
