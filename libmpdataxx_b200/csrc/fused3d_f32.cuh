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
//     k-shifted operand stay elementwise;
//   * the march is unrolled by the period (4) of its rings of shared planes,
//     so every plane slot is a compile-time offset of one of three per-thread
//     shared addresses (own quad, row above, row below) and the carried
//     x-history is renamed rather than moved; C~ of the y-face and the betas
//     of the previous plane are read back from shared memory instead of being
//     carried, which keeps the kernel within the 128 registers that 512
//     threads per SM allow;
//   * the FCT quotients use the approximate-reciprocal division (qdiv).
//
// The result equals the reference's formulae up to FP32 rounding (the order of
// additions differs from formulae_mpdata_3d.hpp:254-295); the properties that
// do not depend on rounding are kept exactly: every face flux enters the two
// cells it separates with the same value (mass conservation in FP64 sums) and
// the limiter uses the same antidiffusive velocities as the limited fluxes
// (FCT bounds).  The FP64 instantiation of fused3d.cuh keeps the reference's
// operation order for bitwise parity.
//
// Plane prefetch: a CTA whose tile lies inside the periods along j and k (most
// of them) brings each plane of the march in with one bulk-tensor copy
// (cp.async.bulk.tensor, issued by one thread) whose completion is counted on an
// mbarrier in bytes, two barriers alternating by step; the other CTAs copy their
// quads with per-thread cp.async, wrapping around the seams.
#pragma once

#include <cuda.h>

#include "fused3d.cuh"

namespace mpdx {
namespace f3s {

using Q = qd::q4<float>;

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

// the FCT quotients (hi - psi) / (sum + eps): the approximate-reciprocal quotient
// of __fdividef (within 2 ulp for these denominators, which lie in
// [FLT_EPSILON, 2^126)); MPDX_F3S_IEEE_DIV=1 selects the correctly rounded one
#ifndef MPDX_F3S_IEEE_DIV
#define MPDX_F3S_IEEE_DIV 0
#endif
__device__ __forceinline__ Q qdiv(const Q &a, const Q &b) {
#if MPDX_F3S_IEEE_DIV
  return a / b;
#else
  return qd::mk(__fdividef(a.a.x, b.a.x), __fdividef(a.a.y, b.a.y), __fdividef(a.b.x, b.b.x), __fdividef(a.b.y, b.b.y));
#endif
}

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

// shared planes of the single-precision kernel, in units of N elements.  Every
// ring of planes along x has 4 slots (the 2-slot rings divide 4), so that with
// the march unrolled by 4 every slot is a compile-time constant: plane x lives
// in slot (x - ts) & 3 of its ring, ts being the first step of the CTA.
//   S0: psi^n planes t-1, t, t+1, t+2; with FCT the prefetch of plane t+3
//       into the slot of t-1 is issued once the limiter has read t-1 (with
//       per-thread copies each thread reads and refills only its own quad of
//       that slot; the bulk copy waits for the last warp);
//   G0: GC_x planes t-1, t, t+1, prefetch t+2;  G1, G2: t, t+1, prefetch t+2;
//   S1: psi1 planes t-1, t, t+1;  CY, BU, BD: planes t-1, t
template <int CR>
struct canvas_s {
  static constexpr int CC = 64, N = CR * CC, TY = CR - 6, TZ = 56, NT = CR * 16;
  static constexpr int S0 = 0, G0 = 4, G1 = 8, G2 = 12, S1 = 16, CY = 20, BU = 22, BD = 24, total = 26;
};

template <int V> struct phase { static constexpr int value = V; };

// shared-memory access at a 32-bit shared address plus a compile-time byte
// offset (the plane slot), so that each access is one instruction with an
// immediate offset and no per-slot address is kept in a register
template <int OFF>
__device__ __forceinline__ Q ldq(unsigned a) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4+%5];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a), "n"(OFF));
  return qd::mk(v.x, v.y, v.z, v.w);
}
template <int OFF>
__device__ __forceinline__ void stq(unsigned a, const Q &v) {
  asm volatile("st.shared.v4.f32 [%0+%1], {%2, %3, %4, %5};" ::"r"(a), "n"(OFF), "f"(v.a.x), "f"(v.a.y), "f"(v.b.x), "f"(v.b.y)
               : "memory");
}
// asynchronous copy of the own quad of one plane row: row points at column kb;
// where the quad crosses the period, column kb + e is read at kb + e + m_e P2,
// the four multiples packed as the bytes m_e + 1 of `wk`
template <int OFF>
__device__ __forceinline__ void cpq(unsigned a, const float *row, bool contig, unsigned wk, int P2) {
  if (contig) {
    asm volatile("cp.async.cg.shared.global [%0+%1], [%2], 16;\n" ::"r"(a), "n"(OFF), "l"(row) : "memory");
  } else {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int m = int((wk >> (8 * e)) & 0xffu) - 1;
      const float *g = row + e + m * P2;
      if (e == 0) asm volatile("cp.async.ca.shared.global [%0+%1], [%2], 4;\n" ::"r"(a), "n"(OFF), "l"(g) : "memory");
      if (e == 1) asm volatile("cp.async.ca.shared.global [%0+%1], [%2], 4;\n" ::"r"(a), "n"(OFF + 4), "l"(g) : "memory");
      if (e == 2) asm volatile("cp.async.ca.shared.global [%0+%1], [%2], 4;\n" ::"r"(a), "n"(OFF + 8), "l"(g) : "memory");
      if (e == 3) asm volatile("cp.async.ca.shared.global [%0+%1], [%2], 4;\n" ::"r"(a), "n"(OFF + 12), "l"(g) : "memory");
    }
  }
}

// ---- bulk-tensor (TMA) plane copies ----
// Tensor maps of the four input fields, each a 3D tiled map over (k, j, x) with
// extents (P2, P1, P0) and a box of 64 columns x CR rows x 1 plane: one box is one
// canvas plane of a CTA whose tile does not cross a periodic seam, at the canvas
// origin (k0 - 4, j0 - 3), k0 a multiple of 56 (16-byte aligned x coordinate).
struct tma_planes {
  CUtensorMap in, g0, g1, g2;
  unsigned *timeout;   // host-mapped word set when a completion wait gives up
  int on;              // 0: every CTA copies with per-thread cp.async
};

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
// one arrival that also adds `bytes` to the transaction count of the current phase
__device__ __forceinline__ void mbar_arrive_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// waits for the phase of parity `parity` to complete, for about two seconds at
// most; a wait that gives up sets *flag and clears `live`, after which this
// thread's further waits return at once (the results of the launch are invalid
// and the host reports the flag)
__device__ __forceinline__ void mbar_wait(unsigned bar, unsigned parity, bool &live, unsigned *flag) {
  if (!live || mbar_test(bar, parity)) return;
  const long long t0 = clock64();
  while (!mbar_test(bar, parity)) {
    if (clock64() - t0 > (1LL << 32)) {
      live = false;
      if (flag) { *reinterpret_cast<volatile unsigned *>(flag) = 1u; __threadfence_system(); }
      return;
    }
  }
}
// one box of a 3D map into shared memory; completion counted on `bar` in bytes
__device__ __forceinline__ void tma_plane(unsigned dst, const CUtensorMap *map, unsigned bar, int k, int j, int x) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
      ::"r"(dst), "l"(reinterpret_cast<unsigned long long>(map)), "r"(bar), "r"(k), "r"(j), "r"(x)
      : "memory");
}

template <bool FCT, int CR>
__global__ void __launch_bounds__(CR * 16, 1) k_fused3d_s(const f3::args<float> A, const __grid_constant__ tma_planes TM) {
  using C = canvas_s<CR>;
  constexpr int N = C::N;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float *const sm = reinterpret_cast<float *>(smem_raw);

  const int tid = threadIdx.x, lane = tid & 31;
  const int r = 2 * (tid >> 5) + (lane >> 4);   // canvas row
  const int q = lane & 15;                      // quad within the row
  const int me = r * C::CC + 4 * q;             // canvas offset of the own quad
  const int up = r + 1 < CR ? me + C::CC : me, dn = r > 0 ? me - C::CC : me;
  // shared addresses of the own quad and of the quads of the rows above / below
  const unsigned s_base = unsigned(__cvta_generic_to_shared(sm));
  const unsigned a_me = s_base + 4u * me, a_up = s_base + 4u * up, a_dn = s_base + 4u * dn;

  const int tile = blockIdx.x;
  const int j0 = (tile / A.tiles_z) * C::TY, k0 = (tile % A.tiles_z) * C::TZ;
  const int x0 = blockIdx.y * A.LX, x1 = min(x0 + A.LX, A.P0);
  // bulk-tensor plane copies for a tile inside the periods along j and k, into
  // 128-byte aligned planes; the two barriers and the warp counter of phase C
  // follow the planes
  const unsigned bar0 = s_base + unsigned(C::total * N * 4), bar1 = bar0 + 8u, cnt = bar0 + 16u;
  const bool tma = TM.on && k0 >= 4 && k0 + 60 <= A.P2 && j0 >= 3 && j0 + CR - 3 <= A.P1 && (s_base & 127u) == 0u;
  bool live = true;

  const int jg = f3::pmod(j0 - 3 + r, A.P1);
  const int kb = k0 - 4 + 4 * q;
  const bool contig = kb >= 0 && kb + 3 < A.P2;
  int kc[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) kc[e] = f3::pmod(kb + e, A.P2);
  // a quad crossing the period: column kb + e is kc[e] = kb + e + m_e P2 with
  // -1 <= m_e <= 64 / P2 (the canvas spans 64 columns from k0 - 4 >= -4),
  // packed as bytes m_e + 1
  unsigned wk = 0;
#pragma unroll
  for (int e = 0; e < 4; ++e) wk |= unsigned((kc[e] - (kb + e)) / A.P2 + 1) << (8 * e);
  // row offsets of the four inputs in elements (plane offsets are added per
  // step; a row offset is below 2^31 for any field that fits in HBM)
  const int o_in = jg * int(A.in.s1) + kb, o_g0 = jg * int(A.g0.s1) + kb;
  const int o_g1 = jg * int(A.g1.s1) + kb, o_g2 = jg * int(A.g2.s1) + kb;
  const int ts = x0 - 3;
  auto slot = [&](int base, int x) { return sm + (base + ((x - ts) & 3)) * N + me; };
  auto cp = [&](float *dst, const dfield<float> &f, int x) {
    f3::gcopy_row(dst, f.o + (long long)f3::pmod(x, A.P0) * f.s0 + (long long)jg * f.s1, kb, contig, kc);
  };

  for (int p = tid; p < C::total * N; p += C::NT) sm[p] = 0.f;
  if (tid == 0) {
    mbar_init(bar0, 1);
    mbar_init(bar1, 1);
    asm volatile("st.shared.u32 [%0], 0;" ::"r"(cnt) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  for (int x = ts - 1; x <= ts + 2; ++x) cp(slot(C::S0, x), A.in, x);
  for (int x = ts - 1; x <= ts + 1; ++x) cp(slot(C::G0, x), A.g0, x);
  for (int x = ts; x <= ts + 1; ++x) { cp(slot(C::G1, x), A.g1, x); cp(slot(C::G2, x), A.g2, x); }
  f3::cp_commit();
  f3::cp_wait_all();
  // the planes written so far (zeros, per-thread copies) before any bulk copy rewrites them
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();
  const Q zero = qd::bc<float>(0.f);
  // carried along the march (own quad): psi1 at t-1, t; the upwind x-flux
  // through face t+1/2; the k-difference of psi1 at t and the k-sum of GC_z
  // at t; C~ of the x- and z-faces of plane t-1 and the limited x-flux into it
  // (C~ of its y-face and its betas are read back from shared memory)
  Q p_m = zero, p_c = zero, fxa = flux(qd::lds(slot(C::S0, ts)), qd::lds(slot(C::S0, ts + 1)), qd::lds(slot(C::G0, ts)));
  Q dzc = zero, szc = zero;
  Q cx_m = zero, cz_m = zero, fx_prev = zero;
  // plane indices (modulo the period) of the next prefetches
  int xi = f3::pmod(ts + 3, A.P0), xg = f3::pmod(ts + 2, A.P0);
  const int jrow = j0 - 3 + r;
  const bool out_row = r >= 3 && r < CR - 3 && jrow < A.P1 && q >= 1 && q < 15;

  auto step = [&](int t, auto ph) {
    constexpr int PH = decltype(ph)::value;   // (t - ts) & 3
    constexpr int M = (PH + 3) & 3, T0 = PH, T1 = (PH + 1) & 3, T2 = (PH + 2) & 3, T3 = (PH + 3) & 3;
    constexpr int C2 = PH & 1, M2 = (PH + 1) & 1;
    // byte offsets of the plane slots
    constexpr int S0m = (C::S0 + M) * N * 4, S0c = (C::S0 + T0) * N * 4, S0p = (C::S0 + T1) * N * 4;
    constexpr int S0pp = (C::S0 + T2) * N * 4, S0n = (C::S0 + T3) * N * 4;
    constexpr int G0m = (C::G0 + M) * N * 4, G0c = (C::G0 + T0) * N * 4, G0p = (C::G0 + T1) * N * 4;
    constexpr int G0n = (C::G0 + T2) * N * 4;
    constexpr int G1c = (C::G1 + T0) * N * 4, G1p = (C::G1 + T1) * N * 4, G1n = (C::G1 + T2) * N * 4;
    constexpr int G2c = (C::G2 + T0) * N * 4, G2p = (C::G2 + T1) * N * 4, G2n = (C::G2 + T2) * N * 4;
    constexpr int S1m = (C::S1 + M) * N * 4, S1c = (C::S1 + T0) * N * 4, S1p = (C::S1 + T1) * N * 4;
    constexpr int CYc = (C::CY + C2) * N * 4, BUc = (C::BU + C2) * N * 4, BDc = (C::BD + C2) * N * 4;
    constexpr int CYm = (C::CY + M2) * N * 4, BUm = (C::BU + M2) * N * 4, BDm = (C::BD + M2) * N * 4;
    // the copies of the previous step (barrier (PH - 1) & 1, its use (PH - 1) >> 1
    // in the group of four steps); the first step's planes came in above
    constexpr int PB = (PH + 3) & 3;
    const unsigned bar = (PH & 1) ? bar1 : bar0;
    if (tma) {
      if (t != ts) mbar_wait((PB & 1) ? bar1 : bar0, unsigned(PB >> 1), live, TM.timeout);
    } else {
      f3::cp_wait_all();
    }
    __syncthreads();
    // prefetch: the advector planes t+2 and psi^n plane t+3 (with FCT issued below,
    // once the limiter has read the slot of t-1; its bytes are counted here)
    if (tma) {
      if (tid == 0) {
        mbar_arrive_tx(bar, 4u * N * 4u);
        if (!FCT) tma_plane(s_base + S0n, &TM.in, bar, k0 - 4, j0 - 3, xi);
        tma_plane(s_base + G0n, &TM.g0, bar, k0 - 4, j0 - 3, xg);
        tma_plane(s_base + G1n, &TM.g1, bar, k0 - 4, j0 - 3, xg);
        tma_plane(s_base + G2n, &TM.g2, bar, k0 - 4, j0 - 3, xg);
      }
    } else {
      if (!FCT) cpq<S0n>(a_me, A.in.o + ((long long)xi * A.in.s0 + o_in), contig, wk, A.P2);
      cpq<G0n>(a_me, A.g0.o + ((long long)xg * A.g0.s0 + o_g0), contig, wk, A.P2);
      cpq<G1n>(a_me, A.g1.o + ((long long)xg * A.g1.s0 + o_g1), contig, wk, A.P2);
      cpq<G2n>(a_me, A.g2.o + ((long long)xg * A.g2.s0 + o_g2), contig, wk, A.P2);
      f3::cp_commit();
    }
    xg = xg + 1 == A.P0 ? 0 : xg + 1;

    // ---- A: psi1 at plane t+1 (mpdata_osc_3d.hpp:181-197) ----
    const Q c = ldq<S0p>(a_me);
    const Q g1p = ldq<G1p>(a_me), g1p_dn = ldq<G1p>(a_dn), g2p = ldq<G2p>(a_me);
    const Q fxb = flux(c, ldq<S0pp>(a_me), ldq<G0p>(a_me));   // face t+3/2
    const Q fyp = flux(c, ldq<S0p>(a_up), g1p);
    const Q fym = flux(ldq<S0p>(a_dn), c, g1p_dn);
    const Q fzp = flux(c, qd::kp1(c), g2p);
    const Q p_p = psub(c, padd(padd(psub(fxb, fxa), psub(fyp, fym)), ssub(fzp, qd::km1(fzp))));
    fxa = fxb;
    stq<S1p>(a_me, p_p);
    __syncthreads();
    const Q pp_up = ldq<S1p>(a_up), pp_dn = ldq<S1p>(a_dn);

    // ---- B: C~ on the own x-face t+1/2, y-face j+1/2 and z-face k+1/2 of plane t ----
    // (computed on every canvas row, as are the limiter and the output below:
    // leaving the rows that do not need them to idle warps measured slower,
    // through the registers the extra control flow holds)
    Q kp_c, dzp, szp, cx_c, cy_c, cz_c;
    const Q pc_up = ldq<S1c>(a_up), pc_dn = ldq<S1c>(a_dn);
    {
      const Q g0c = ldq<G0c>(a_me), g0m = ldq<G0m>(a_me);
      const Q g1c = ldq<G1c>(a_me), g1c_dn = ldq<G1c>(a_dn);
      const Q g2c = ldq<G2c>(a_me);
      // two-point terms
      const Q dxo = psub(p_p, p_m);                                 // psi1 x+1 - x-1, own row
      const Q dyc = psub(pc_up, pc_dn);                             // psi1 j+1 - j-1 at t
      const Q dyp = psub(pp_up, pp_dn);                             // the same at t+1
      dzp = ssub(qd::kp1(p_p), qd::km1(p_p));                       // psi1 k+1 - k-1 at t+1
      const Q sxc = padd(g0c, g0m);                                 // GC_x faces t+-1/2
      const Q syc = padd(g1c, g1c_dn), syp = padd(g1p, g1p_dn);     // GC_y faces j+-1/2
      szp = sadd(g2p, qd::km1(g2p));                                // GC_z faces k+-1/2 at t+1
      // x-face t+1/2: transverse y (psi and GC_y), z (psi and GC_z)
      cx_c = adiff(g0c, psub(p_p, p_c), padd(syp, syc), padd(dyp, dyc), padd(szp, szc), padd(dzp, dzc));
      // y-face j+1/2 of plane t: transverse z, x
      {
        const Q g2c_up = ldq<G2c>(a_up);
        const Q dz_up = ssub(qd::kp1(pc_up), qd::km1(pc_up));
        const Q sz_up = sadd(g2c_up, qd::km1(g2c_up));
        const Q dx_up = psub(pp_up, ldq<S1m>(a_up));
        const Q sx_up = padd(ldq<G0c>(a_up), ldq<G0m>(a_up));
        cy_c = adiff(g1c, psub(pc_up, p_c), padd(sz_up, szc), padd(dz_up, dzc), padd(sx_up, sxc), padd(dx_up, dxo));
        stq<CYc>(a_me, cy_c);
      }
      // z-face k+1/2 of plane t: transverse x, y
      kp_c = qd::kp1(p_c);
      cz_c = adiff(g2c, ssub(kp_c, p_c), sadd(qd::kp1(sxc), sxc), sadd(qd::kp1(dxo), dxo), sadd(qd::kp1(syc), syc),
                   sadd(qd::kp1(dyc), dyc));
    }

    // ---- C: betas at plane t (formulae_mpdata_fct_3d.hpp:48-143) ----
    Q bu_c = zero, bd_c = zero;
    if (FCT) {
      __syncthreads();
      {
        const Q cy_dn = ldq<CYc>(a_dn);
        Q mnq, mxq;
        {
          const Q s0_c = ldq<S0c>(a_me), s0_m = ldq<S0m>(a_me);
          const Q yp = ldq<S0c>(a_up), ym = ldq<S0c>(a_dn), zp = qd::kp1(s0_c), zm = qd::km1(s0_c);
          mnq = qd::qmin(qd::qmin(qd::qmin(qd::qmin(qd::qmin(qd::qmin(s0_c, c), s0_m), yp), ym), zp), zm);
          mxq = qd::qmax(qd::qmax(qd::qmax(qd::qmax(qd::qmax(qd::qmax(s0_c, c), s0_m), yp), ym), zp), zm);
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
        bu_c = qdiv(psub(hi, p_c), padd(du, e));
        bd_c = qdiv(psub(p_c, lo), padd(dd, e));
        stq<BUc>(a_me, bu_c);
        stq<BDc>(a_me, bd_c);
      }
      // psi^n plane t+3 into the slot of t-1, now read: per thread its own quad;
      // in bulk by the last warp through here (the counter's acquire-release
      // orders every warp's reads of the slot before the copy)
      if (tma) {
        __syncwarp();
        if (lane == 0) {
          unsigned old;
          asm volatile("atom.acq_rel.cta.shared::cta.add.u32 %0, [%1], 1;" : "=r"(old) : "r"(cnt) : "memory");
          if (old % unsigned(C::NT / 32) == unsigned(C::NT / 32 - 1)) tma_plane(s_base + S0n, &TM.in, bar, k0 - 4, j0 - 3, xi);
        }
      } else {
        cpq<S0n>(a_me, A.in.o + ((long long)xi * A.in.s0 + o_in), contig, wk, A.P2);
        f3::cp_commit();
      }
    }
    xi = xi + 1 == A.P0 ? 0 : xi + 1;

    {
      // ---- D: limited fluxes at plane t-1 (formulae_mpdata_fct_3d.hpp:148-250) ----
      Q fxx = cx_m, fyu = ldq<CYm>(a_me), fyd = ldq<CYm>(a_dn), fzz = cz_m;
      if (FCT) {
        const Q bu_m = ldq<BUm>(a_me), bd_m = ldq<BDm>(a_me);
        const Q bu_dn = ldq<BUm>(a_dn), bd_dn = ldq<BDm>(a_dn);
        fxx = pmul(fxx, qd::qlim(fxx, bd_m, bu_c, bu_m, bd_c));
        fyu = pmul(fyu, qd::qlim(fyu, bd_m, ldq<BUm>(a_up), bu_m, ldq<BDm>(a_up)));
        fyd = pmul(fyd, qd::qlim(fyd, bd_dn, bu_m, bu_dn, bd_m));
        fzz = pmul(fzz, qd::qlim(fzz, bd_m, qd::kp1(bu_m), bu_m, qd::kp1(bd_m)));
      }

      // ---- E: psi^{n+1} at plane t-1 ----
      const int x = t - 1;
      const Q v = psub(p_m, padd(padd(psub(fxx, fx_prev), psub(fyu, fyd)), ssub(fzz, qd::km1(fzz))));
      fx_prev = fxx;
      if (out_row && x >= x0 && x < x1) {
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
    cx_m = cx_c; cz_m = cz_c;
  };

  // steps ts .. x1 (the last chunk rounds up to a whole unrolled group: the
  // extra steps read wrapped planes and store nothing)
  const int nsteps = (x1 - ts + 1 + 3) & ~3;
  for (int u = 0; u < nsteps; u += 4) {
    step(ts + u, phase<0>{});
    step(ts + u + 1, phase<1>{});
    step(ts + u + 2, phase<2>{});
    step(ts + u + 3, phase<3>{});
  }
  // no copy may land after the CTA has left: the last step (phase 3) counted its
  // copies on barrier 1, second use of the group (parity 1)
  if (tma) {
    bool fin = true;
    mbar_wait(bar1, 1u, fin, TM.timeout);
  } else {
    f3::cp_wait_all();
  }
}

}  // namespace f3s
}  // namespace mpdx
