// Fused 3D MPDATA step in FP32 with the infinite-gauge option (n_iters = 2,
// opts iga or iga|fct, all boundaries cyclic): the single-precision form of the
// kernel in fused3d.cuh, with the same 2.5D decomposition (a CTA owns a
// CR x 64 canvas of the (j, k) plane and marches along x; each thread owns one
// quad of 4 consecutive k of one canvas row) and the same stage schedule, but
// with the arithmetic regrouped for single precision:
//
//   * every face quantity is computed once: the upwind x-flux through face
//     x+1/2 computed for plane x+1 is the x-flux into plane x+2 one step later,
//     and the flux through face k-1/2 is the k+1/2 flux of the neighbouring
//     column (a shuffle), so each face is evaluated by one thread only;
//   * the four-point stencils of the antidiffusive velocity (the transverse
//     psi differences of formulae_mpdata_psi_3d.hpp and the Courant-number
//     averages of formulae_mpdata_gc_3d.hpp, all divided by 4) are written as
//     sums of two-point terms, e.g. for the x-face
//         ndy = ((psi(x+1,j+1) - psi(x+1,j-1)) + (psi(x,j+1) - psi(x,j-1))) / 4,
//     so the two-point terms are shared between the three faces of a point
//     and between consecutive planes (carried in registers along the march),
//     and the factors 1/4 * 1/4 * 1/2 are folded into one constant;
//   * arithmetic on aligned quads uses the paired FP32 instructions of sm_100
//     (two lanes per instruction: add/sub/mul/fma.rn.f32x2); expressions with a
//     k-shifted operand stay elementwise.
//
// The result equals the reference's formulae up to FP32 rounding (the order of
// additions differs from formulae_mpdata_3d.hpp:254-295); the properties that
// do not depend on rounding are kept exactly: every face flux enters the two
// cells it separates with the same value (mass conservation in FP64 sums) and
// the limiter uses the same antidiffusive velocities as the limited fluxes
// (FCT bounds).  The FP64 instantiation of fused3d.cuh keeps the reference's
// operation order for bitwise parity.
#pragma once

#include "fused3d.cuh"

namespace mpdx {
namespace f3s {

using Q = qd::q4<float>;
using f3::canvas;

// ---- paired (aligned) arithmetic: two FP32 lanes per instruction ----
__device__ __forceinline__ float2 m2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ Q padd(const Q &x, const Q &y) { return {__fadd2_rn(x.a, y.a), __fadd2_rn(x.b, y.b)}; }
// x - y = fma(y, -1, x): one rounding, as the subtraction
__device__ __forceinline__ Q psub(const Q &x, const Q &y) {
  const float2 m = m2(-1.f, -1.f);
  return {__ffma2_rn(y.a, m, x.a), __ffma2_rn(y.b, m, x.b)};
}
__device__ __forceinline__ Q pmul(const Q &x, const Q &y) { return {__fmul2_rn(x.a, y.a), __fmul2_rn(x.b, y.b)}; }
__device__ __forceinline__ Q pfma(const Q &x, const Q &y, const Q &z) {
  return {__ffma2_rn(x.a, y.a, z.a), __ffma2_rn(x.b, y.b, z.b)};
}
__device__ __forceinline__ Q pmuls(const Q &x, float s) {
  const float2 m = m2(s, s);
  return {__fmul2_rn(x.a, m), __fmul2_rn(x.b, m)};
}
// ---- elementwise (for k-shifted operands) ----
__device__ __forceinline__ Q sadd(const Q &x, const Q &y) {
  return qd::mk(x.a.x + y.a.x, x.a.y + y.a.y, x.b.x + y.b.x, x.b.y + y.b.y);
}
__device__ __forceinline__ Q ssub(const Q &x, const Q &y) {
  return qd::mk(x.a.x - y.a.x, x.a.y - y.a.y, x.b.x - y.b.x, x.b.y - y.b.y);
}

// upwind flux through a face with Courant number C between l and r:
// C * (C > 0 ? l : r)  (donorcell_formulae.hpp:25-34; one product is zero)
__device__ __forceinline__ Q flux(const Q &l, const Q &r, const Q &C) { return pmul(C, qd::sel_pos(C, l, r)); }

// antidiffusive velocity through one face from the two-point sums:
//   |C|/2 (1 - |C|) nx - C (S1 D1 + S2 D2) / 32
// (formulae_mpdata_3d.hpp:254-295 with G = 1 and iga: ndx = nx, the transverse
// derivatives D/4 and the Courant averages S/4)
__device__ __forceinline__ Q adiff(const Q &C, const Q &nx, const Q &S1, const Q &D1, const Q &S2, const Q &D2) {
  auto hc = [](float c) { return 0.5f * fabsf(c) * (1.f - fabsf(c)); };
  const Q h = qd::mk(hc(C.a.x), hc(C.a.y), hc(C.b.x), hc(C.b.y));
  const Q v = pfma(S2, D2, pmul(S1, D1));
  return pfma(pmuls(C, -1.f / 32.f), v, pmul(h, nx));
}

template <bool FCT, int CR>
__global__ void __launch_bounds__(CR * 16, 1) k_fused3d_s(const f3::args<float> A) {
  using C = canvas<CR>;
  constexpr int N = C::N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float *sm = reinterpret_cast<float *>(smem_raw);

  const int tid = threadIdx.x, lane = tid & 31;
  const int r = 2 * (tid >> 5) + (lane >> 4);   // canvas row
  const int q = lane & 15;                      // quad within the row
  const int me = r * C::CC + 4 * q;             // canvas offset of the own quad
  auto R = [&](int d) { const int rr = r + d; return rr >= 0 && rr < CR ? me + d * C::CC : me; };
  const int up = R(1), dn = R(-1);

  const int tile = blockIdx.x;
  const int j0 = (tile / A.tiles_z) * C::TY, k0 = (tile % A.tiles_z) * C::TZ;
  const int x0 = blockIdx.y * A.LX, x1 = min(x0 + A.LX, A.P0);

  const int jg = f3::pmod(j0 - 3 + r, A.P1);
  const int kb = k0 - 4 + 4 * q;
  const bool contig = kb >= 0 && kb + 3 < A.P2;
  int kc[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) kc[e] = f3::pmod(kb + e, A.P2);
  const long long ro_in = (long long)jg * A.in.s1, ro_g0 = (long long)jg * A.g0.s1;
  const long long ro_g1 = (long long)jg * A.g1.s1, ro_g2 = (long long)jg * A.g2.s1;

  auto plane = [&](int base, int nslots, int x) { return sm + (base + ((x % nslots) + nslots) % nslots) * N; };
  auto cp = [&](float *dst, const dfield<float> &f, long long ro, int x) {
    f3::gcopy(dst + me, f, f3::pmod(x, A.P0), ro, kb, contig, kc);
  };

  for (int p = tid; p < C::total * N; p += C::NT) sm[p] = 0.f;
  __syncthreads();

  const int ts = x0 - 3;
  for (int x = ts - 1; x <= ts + 2; ++x) cp(plane(C::S0, C::NS0, x), A.in, ro_in, x);
  for (int x = ts - 1; x <= ts + 1; ++x) cp(plane(C::G0, C::NG0, x), A.g0, ro_g0, x);
  for (int x = ts; x <= ts + 1; ++x) { cp(plane(C::G1, C::NG1, x), A.g1, ro_g1, x); cp(plane(C::G2, C::NG1, x), A.g2, ro_g2, x); }
  f3::cp_commit();

  const Q zero = qd::bc<float>(0.f);
  // carried along the march (own quad): psi1 at t-1, t; the upwind x-flux
  // through face t+1/2; the k-difference of psi1 at t and the k-sum of GC_z at
  // t; the antidiffusive / limited quantities of plane t-1
  Q p_m = zero, p_c = zero, fxa = zero, dzc = zero, szc = zero;
  Q cx_m = zero, cy_m = zero, cz_m = zero, bu_m = zero, bd_m = zero, fx_prev = zero;
  auto slot0 = [](int x, int n) { return ((x % n) + n) % n; };
  f3::ring<C::NS0> r_s0{slot0(ts - 1, C::NS0)};
  f3::ring<C::NG0> r_g0{slot0(ts - 1, C::NG0)};
  f3::ring<C::NG1> r_g1{slot0(ts, C::NG1)};
  f3::ring<3> r_s1{slot0(ts - 1, 3)};
  f3::ring<2> r_2{slot0(ts - 1, 2)};

  f3::plane_walker<float> w_in, w_g0, w_g1, w_g2;
  w_in.init(A.in, ts + 3, A.P0, ro_in);
  w_g0.init(A.g0, ts + 2, A.P0, ro_g0);
  w_g1.init(A.g1, ts + 2, A.P0, ro_g1);
  w_g2.init(A.g2, ts + 2, A.P0, ro_g2);
  for (int t = ts; t <= x1; ++t) {
    f3::cp_wait_all();
    __syncthreads();
    float *const s0b = sm + C::S0 * N, *const g0b = sm + C::G0 * N, *const g1b = sm + C::G1 * N, *const g2b = sm + C::G2 * N;
    f3::gcopy_row(s0b + r_s0.at(4) * N + me, w_in.p, kb, contig, kc);
    f3::gcopy_row(g0b + r_g0.at(3) * N + me, w_g0.p, kb, contig, kc);
    f3::gcopy_row(g1b + r_g1.at(2) * N + me, w_g1.p, kb, contig, kc);
    f3::gcopy_row(g2b + r_g1.at(2) * N + me, w_g2.p, kb, contig, kc);
    f3::cp_commit();
    w_in.next(); w_g0.next(); w_g1.next(); w_g2.next();
    const float *S0m = s0b + r_s0.at(0) * N, *S0c = s0b + r_s0.at(1) * N, *S0p = s0b + r_s0.at(2) * N;
    const float *S0pp = s0b + r_s0.at(3) * N;
    const float *G0m = g0b + r_g0.at(0) * N, *G0c = g0b + r_g0.at(1) * N, *G0p = g0b + r_g0.at(2) * N;
    const float *G1c = g1b + r_g1.at(0) * N, *G1p = g1b + r_g1.at(1) * N;
    const float *G2c = g2b + r_g1.at(0) * N, *G2p = g2b + r_g1.at(1) * N;
    float *const s1b = sm + C::S1 * N;
    const float *S1m = s1b + r_s1.at(0) * N, *S1c = s1b + r_s1.at(1) * N;
    float *S1p = s1b + r_s1.at(2) * N;
    const int sc = r_2.at(1) * N, sm1 = r_2.at(0) * N;
    float *CYc = sm + C::CY * N + sc, *BUc = sm + C::BU * N + sc, *BDc = sm + C::BD * N + sc;
    const float *CYm = sm + C::CY * N + sm1, *BUm = sm + C::BU * N + sm1, *BDm = sm + C::BD * N + sm1;
    r_s0.next(); r_g0.next(); r_g1.next(); r_s1.next(); r_2.next();

    // ---- A: psi1 at plane t+1 (mpdata_osc_3d.hpp:181-197) ----
    const Q c = qd::lds(S0p + me);
    const Q g1p = qd::lds(G1p + me), g1p_dn = qd::lds(G1p + dn), g2p = qd::lds(G2p + me);
    // the x-flux through face t+1/2 comes from the previous step, except on the first
    if (t == ts) fxa = flux(qd::lds(S0c + me), c, qd::lds(G0c + me));
    const Q fxb = flux(c, qd::lds(S0pp + me), qd::lds(G0p + me));   // face t+3/2
    const Q fyp = flux(c, qd::lds(S0p + up), g1p);
    const Q fym = flux(qd::lds(S0p + dn), c, g1p_dn);
    const Q fzp = flux(c, qd::kp1(c), g2p);
    const Q p_p = psub(c, padd(padd(psub(fxb, fxa), psub(fyp, fym)), ssub(fzp, qd::km1(fzp))));
    fxa = fxb;
    qd::sts(S1p + me, p_p);
    __syncthreads();
    const Q pp_up = qd::lds(S1p + up), pp_dn = qd::lds(S1p + dn);

    // ---- B: C~ on the own x-face t+1/2, y-face j+1/2 and z-face k+1/2 of plane t ----
    const Q pc_up = qd::lds(S1c + up), pc_dn = qd::lds(S1c + dn);
    const Q g0c = qd::lds(G0c + me), g0m = qd::lds(G0m + me);
    const Q g1c = qd::lds(G1c + me), g1c_dn = qd::lds(G1c + dn);
    const Q g2c = qd::lds(G2c + me);
    // two-point terms
    const Q dxo = psub(p_p, p_m);                                 // psi1 x+1 - x-1, own row
    const Q dyc = psub(pc_up, pc_dn);                             // psi1 j+1 - j-1 at t
    const Q dyp = psub(pp_up, pp_dn);                             // the same at t+1
    const Q kp_p = qd::kp1(p_p), km_p = qd::km1(p_p);
    const Q dzp = ssub(kp_p, km_p);                               // psi1 k+1 - k-1 at t+1
    const Q sxc = padd(g0c, g0m);                                 // GC_x faces t+-1/2
    const Q syc = padd(g1c, g1c_dn), syp = padd(g1p, g1p_dn);     // GC_y faces j+-1/2
    const Q szp = sadd(g2p, qd::km1(g2p));                        // GC_z faces k+-1/2 at t+1
    Q cx_c, cy_c, cz_c;
    // x-face t+1/2: transverse y (psi and GC_y), z (psi and GC_z)
    cx_c = adiff(g0c, psub(p_p, p_c), padd(syp, syc), padd(dyp, dyc), padd(szp, szc), padd(dzp, dzc));
    // y-face j+1/2 of plane t: transverse z, x
    {
      const Q g2c_up = qd::lds(G2c + up);
      const Q dz_up = ssub(qd::kp1(pc_up), qd::km1(pc_up));
      const Q sz_up = sadd(g2c_up, qd::km1(g2c_up));
      const Q dx_up = psub(pp_up, qd::lds(S1m + up));
      const Q sx_up = padd(qd::lds(G0c + up), qd::lds(G0m + up));
      cy_c = adiff(g1c, psub(pc_up, p_c), padd(sz_up, szc), padd(dz_up, dzc), padd(sx_up, sxc), padd(dx_up, dxo));
      qd::sts(CYc + me, cy_c);
    }
    // z-face k+1/2 of plane t: transverse x, y
    const Q kp_c = qd::kp1(p_c);
    cz_c = adiff(g2c, ssub(kp_c, p_c), sadd(qd::kp1(sxc), sxc), sadd(qd::kp1(dxo), dxo), sadd(qd::kp1(syc), syc),
                 sadd(qd::kp1(dyc), dyc));

    // ---- C: betas at plane t (formulae_mpdata_fct_3d.hpp:48-143) ----
    Q bu_c = zero, bd_c = zero;
    if (FCT) {
      __syncthreads();
      const Q cy_dn = qd::lds(CYc + dn);
      Q mnq, mxq;
      {
        const Q s0c = qd::lds(S0c + me), s0p = qd::lds(S0p + me), s0m = qd::lds(S0m + me);
        const Q yp = qd::lds(S0c + up), ym = qd::lds(S0c + dn), zp = qd::kp1(s0c), zm = qd::km1(s0c);
        mnq = qd::qmin(qd::qmin(qd::qmin(qd::qmin(qd::qmin(qd::qmin(s0c, s0p), s0m), yp), ym), zp), zm);
        mxq = qd::qmax(qd::qmax(qd::qmax(qd::qmax(qd::qmax(qd::qmax(s0c, s0p), s0m), yp), ym), zp), zm);
      }
      const Q xp = p_p, xm = p_m, yp = pc_up, ym = pc_dn, zp = kp_c, zm = qd::km1(p_c);
      const Q fxm = cx_m, fxp = cx_c, fym = cy_dn, fyp = cy_c, fzm = qd::km1(cz_c), fzp = cz_c;
      const Q hi = qd::qmax(mxq, qd::qmax(p_c, qd::qmax(xp, qd::qmax(xm, qd::qmax(yp, qd::qmax(ym, qd::qmax(zp, zm)))))));
      const Q lo = qd::qmin(mnq, qd::qmin(yp, qd::qmin(xm, qd::qmin(p_c, qd::qmin(xp, qd::qmin(zp, qd::qmin(zm, ym)))))));
      const Q du = padd(padd(psub(qd::pos(fxm), qd::neg(fxp)), psub(qd::pos(fym), qd::neg(fyp))),
                        psub(qd::pos(fzm), qd::neg(fzp)));
      const Q dd = padd(padd(psub(qd::pos(fxp), qd::neg(fxm)), psub(qd::pos(fyp), qd::neg(fym))),
                        psub(qd::pos(fzp), qd::neg(fzm)));
      const Q e = qd::bc<float>(FLT_EPSILON);
      bu_c = psub(hi, p_c) / padd(du, e);
      bd_c = psub(p_c, lo) / padd(dd, e);
      qd::sts(BUc + me, bu_c);
      qd::sts(BDc + me, bd_c);
    }

    // ---- D: limited fluxes at plane t-1 (formulae_mpdata_fct_3d.hpp:148-250) ----
    Q fxx = cx_m, fyu = cy_m, fyd = qd::lds(CYm + dn), fzz = cz_m;
    if (FCT) {
      const Q bu_dn = qd::lds(BUm + dn), bd_dn = qd::lds(BDm + dn);
      fxx = pmul(fxx, qd::qlim(fxx, bd_m, bu_c, bu_m, bd_c));
      fyu = pmul(fyu, qd::qlim(fyu, bd_m, qd::lds(BUm + up), bu_m, qd::lds(BDm + up)));
      fyd = pmul(fyd, qd::qlim(fyd, bd_dn, bu_m, bu_dn, bd_m));
      fzz = pmul(fzz, qd::qlim(fzz, bd_m, qd::kp1(bu_m), bu_m, qd::kp1(bd_m)));
    }

    // ---- E: psi^{n+1} at plane t-1 ----
    {
      const int x = t - 1;
      const Q v = psub(p_m, padd(padd(psub(fxx, fx_prev), psub(fyu, fyd)), ssub(fzz, qd::km1(fzz))));
      fx_prev = fxx;
      const int jrow = j0 - 3 + r;
      if (x >= x0 && x < x1 && r >= 3 && r < CR - 3 && jrow < A.P1 && q >= 1 && q < 15) {
        float *o = A.out.o + (long long)x * A.out.s0 + (long long)jrow * A.out.s1;
        if (contig) {
          qd::sts(o + kb, v);
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if (kb + e < A.P2) o[kb + e] = f3::elem(v, e);
        }
        if (x == 0 || jrow == 0 || kb == 0) {
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int k = kb + e;
            if (k >= A.P2) continue;
            const float val = f3::elem(v, e);
            const int xs[2] = {x, x == 0 ? A.n0 - 1 : -1};
            const int js[2] = {jrow, jrow == 0 ? A.n1 - 1 : -1};
            const int ks[2] = {k, k == 0 ? A.n2 - 1 : -1};
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
              for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int cc = 0; cc < 2; ++cc)
                  if ((a | b | cc) && xs[a] >= 0 && js[b] >= 0 && ks[cc] >= 0) A.out(xs[a], js[b], ks[cc]) = val;
          }
        }
      }
    }

    // shift the x-history
    p_m = p_c; p_c = p_p;
    dzc = dzp; szc = szp;
    cx_m = cx_c; cy_m = cy_c; cz_m = cz_c;
    bu_m = bu_c; bd_m = bd_c;
  }
  f3::cp_wait_all();
}

}  // namespace f3s
}  // namespace mpdx
