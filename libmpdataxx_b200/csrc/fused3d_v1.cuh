// Fused 3D MPDATA step (n_iters = 2, options {0, fct, iga, iga|fct}, all
// boundaries cyclic): one kernel computes the upwind pass, the antidiffusive
// pseudo-velocities, the FCT limiter and the corrective pass, keeping every
// intermediate on chip.
//
// Decomposition (2.5D blocking): a CTA owns a TY x TZ column of the (j, k)
// plane and marches along x over LX planes.  Each plane stage keeps a ring of
// the planes it still needs in shared memory; x-neighbours come from the ring,
// (j, k)-neighbours from the halo of the plane.  Per step t the CTA
//   loads   psi^n(t+3), GC_x faces (t+2), GC_y / GC_z planes (t+2)   [cp.async, one step ahead]
//   psi1    = donor-cell(psi^n, GC)                 at plane t+1   (mpdata_osc_3d.hpp:181-197)
//   min/max of psi^n over the 7-point stencil       at plane t     (mpdata_fct_3d.hpp:31-55)
//   C~      = antidiff(psi1, GC)  x-faces (t+1/2), y/z faces of plane t   (formulae_mpdata_3d.hpp:254-295)
//   beta_up / beta_dn                               at plane t     (formulae_mpdata_fct_3d.hpp:48-143)
//   C_mono  = GC_mono(C~, betas)  x-faces (t-1/2), y/z faces of plane t-1 (formulae_mpdata_fct_3d.hpp:148-250)
//   psi^{n+1} = donor-cell(psi1, C_mono)            at plane t-1
// so the only DRAM traffic is psi^n and GC in, psi^{n+1} out (20 B per cell in
// FP32), plus halo re-reads that neighbouring CTAs mostly serve from L2.
//
// Periodicity follows libmpdata++'s cyclic convention (bcond/cyclic_3d.hpp):
// with n points per axis the period is n-1 and point n-1 duplicates point 0.
// The kernel computes the n-1 unique points and writes the duplicate copies.
// Expressions follow the reference's operand order; the FP64 instantiation is
// compiled without FMA contraction and reproduces the general path bitwise.
#pragma once

#include <cfloat>

#include "state.cuh"

namespace mpdx {
namespace f3 {

template <class T> struct lims;
template <> struct lims<float> {
  __device__ static float tiny() { return FLT_MIN; }
  __device__ static float eps() { return FLT_EPSILON; }
};
template <> struct lims<double> {
  __device__ static double tiny() { return DBL_MIN; }
  __device__ static double eps() { return DBL_EPSILON; }
};

template <class T> __device__ __forceinline__ T pos(T x) { return T(0) < x ? x : T(0); }   // std::max(0, x)
template <class T> __device__ __forceinline__ T neg(T x) { return x < T(0) ? x : T(0); }   // std::min(0, x)
template <class T> __device__ __forceinline__ T mx(T a, T b) { return a < b ? b : a; }
template <class T> __device__ __forceinline__ T mn(T a, T b) { return b < a ? b : a; }
template <class T> __device__ __forceinline__ T flux(T pl, T pr, T c) { return pos(c) * pl + neg(c) * pr; }
template <class T> __device__ __forceinline__ T frac(T nom, T den) { return nom / (den + lims<T>::tiny()); }

// region of the (j, k) plane relative to the tile origin: j in [J0, J0+NJ), k in [K0, K0+NK)
template <int J0, int NJ, int K0, int NK>
struct reg {
  static constexpr int j0 = J0, nj = NJ, k0 = K0, nk = NK, size = NJ * NK;
  __device__ __forceinline__ static int at(int j, int k) { return (j - J0) * NK + (k - K0); }
};

template <int TY, int TZ>
struct layout {
  using P0R = reg<-3, TY + 6, -3, TZ + 6>;  // psi^n
  using G0R = reg<-2, TY + 4, -2, TZ + 4>;  // GC_x faces
  using G1R = reg<-3, TY + 5, -2, TZ + 4>;  // GC_y faces (index j <-> face j+1/2)
  using G2R = reg<-2, TY + 4, -3, TZ + 5>;  // GC_z faces
  using P1R = reg<-2, TY + 4, -2, TZ + 4>;  // psi1
  using R1 = reg<-1, TY + 2, -1, TZ + 2>;   // psi_min/max, C~_x, betas
  using CYR = reg<-2, TY + 3, -1, TZ + 2>;  // C~_y faces j in [-2, TY]
  using CZR = reg<-1, TY + 2, -2, TZ + 3>;  // C~_z faces k in [-2, TZ]
  using MYR = reg<-1, TY + 1, 0, TZ>;       // C_mono_y faces j in [-1, TY)
  using MZR = reg<0, TY, -1, TZ + 1>;       // C_mono_z faces k in [-1, TZ)
  static constexpr int NP0 = 5, NG0 = 4, NG1 = 3, NP1 = 3, NC = 2, NB = 2;
  static constexpr int o_p0 = 0;
  static constexpr int o_g0 = o_p0 + NP0 * P0R::size;
  static constexpr int o_g1 = o_g0 + NG0 * G0R::size;
  static constexpr int o_g2 = o_g1 + NG1 * G1R::size;
  static constexpr int o_p1 = o_g2 + NG1 * G2R::size;
  static constexpr int o_mn = o_p1 + NP1 * P1R::size;
  static constexpr int o_mx = o_mn + R1::size;
  static constexpr int o_cx = o_mx + R1::size;
  static constexpr int o_cy = o_cx + NC * R1::size;
  static constexpr int o_cz = o_cy + NC * CYR::size;
  static constexpr int o_bu = o_cz + NC * CZR::size;
  static constexpr int o_bd = o_bu + NB * R1::size;
  static constexpr int o_my = o_bd + NB * R1::size;
  static constexpr int o_mz = o_my + MYR::size;
  static constexpr int total = o_mz + MZR::size;
  static constexpr int zero_from = o_p1;  // rings whose history starts undefined
};

template <class T>
struct args {
  dfield<T> in, out, g0, g1, g2;
  int P0, P1, P2;   // periods (n - 1)
  int n0, n1, n2;   // points per axis (duplicate at n - 1)
  int LX;           // planes per CTA
  int tiles_z;      // tiles along k
};

__device__ __forceinline__ int wrap(int x, int P) { return x < 0 ? x + P : (x >= P ? x - P : x); }

template <class T>
__device__ __forceinline__ void cp_async(T *smem, const T *gmem) {
  const unsigned s = unsigned(__cvta_generic_to_shared(smem));
  if (sizeof(T) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// load one plane region of field f (plane index x along axis 0, wrapped) into smem
// (cell and face indices wrap with the same period; the fused path requires
// P0 >= 5, P1 >= TY + 3 and P2 >= TZ + 3 so that one correction suffices)
template <class R, int NT, class T>
__device__ __forceinline__ void load_plane(T *dst, const dfield<T> &f, int x, int P0, int j0, int k0, int P1, int P2) {
  const int xi = wrap(x, P0);
  const T *base = f.o + (long long)xi * f.s0;
#pragma unroll 1
  for (int p = threadIdx.x; p < R::size; p += NT) {
    const int jr = R::j0 + p / R::nk, kr = R::k0 + p % R::nk;
    const int j = wrap(j0 + jr, P1), k = wrap(k0 + kr, P2);
    cp_async(dst + p, base + (long long)j * f.s1 + k);
  }
}

template <class T, bool IGA, bool FCT, int TY, int TZ, int NT>
__global__ void __launch_bounds__(NT) k_fused3d(const args<T> A) {
  using L = layout<TY, TZ>;
  using P0R = typename L::P0R; using G0R = typename L::G0R; using G1R = typename L::G1R;
  using G2R = typename L::G2R; using P1R = typename L::P1R; using R1 = typename L::R1;
  using CYR = typename L::CYR; using CZR = typename L::CZR; using MYR = typename L::MYR;
  using MZR = typename L::MZR;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);

  const int tile = blockIdx.x;
  const int j0 = (tile / A.tiles_z) * TY, k0 = (tile % A.tiles_z) * TZ;
  const int x0 = blockIdx.y * A.LX;
  const int x1 = min(x0 + A.LX, A.P0);  // exclusive end of the planes this CTA writes
  const int tid = threadIdx.x;

  // ring accessors (plane/face index -> slot, wrapped non-negative)
  auto slot = [](int x, int n) { return ((x % n) + n) % n; };
  auto P0 = [&](int x) { return sm + L::o_p0 + slot(x, L::NP0) * P0R::size; };
  auto G0 = [&](int x) { return sm + L::o_g0 + slot(x, L::NG0) * G0R::size; };
  auto G1 = [&](int x) { return sm + L::o_g1 + slot(x, L::NG1) * G1R::size; };
  auto G2 = [&](int x) { return sm + L::o_g2 + slot(x, L::NG1) * G2R::size; };
  auto P1 = [&](int x) { return sm + L::o_p1 + slot(x, L::NP1) * P1R::size; };
  auto CX = [&](int x) { return sm + L::o_cx + slot(x, L::NC) * R1::size; };
  auto CY = [&](int x) { return sm + L::o_cy + slot(x, L::NC) * CYR::size; };
  auto CZ = [&](int x) { return sm + L::o_cz + slot(x, L::NC) * CZR::size; };
  auto BU = [&](int x) { return sm + L::o_bu + slot(x, L::NB) * R1::size; };
  auto BD = [&](int x) { return sm + L::o_bd + slot(x, L::NB) * R1::size; };
  T *MN = sm + L::o_mn, *MX = sm + L::o_mx, *MY = sm + L::o_my, *MZ = sm + L::o_mz;

  // history rings start at zero (their first planes are never used for output)
  for (int p = L::zero_from + tid; p < L::total; p += NT) sm[p] = T(0);

  const int ts = x0 - 3;
  // prologue: psi^n planes ts-1..ts+2, GC_x faces ts-1..ts+1, GC_y/GC_z planes ts..ts+1
  for (int x = ts - 1; x <= ts + 2; ++x) load_plane<P0R, NT>(P0(x), A.in, x, A.P0, j0, k0, A.P1, A.P2);
  for (int x = ts - 1; x <= ts + 1; ++x) load_plane<G0R, NT>(G0(x), A.g0, x, A.P0, j0, k0, A.P1, A.P2);
  for (int x = ts; x <= ts + 1; ++x) {
    load_plane<G1R, NT>(G1(x), A.g1, x, A.P0, j0, k0, A.P1, A.P2);
    load_plane<G2R, NT>(G2(x), A.g2, x, A.P0, j0, k0, A.P1, A.P2);
  }
  cp_commit();

  constexpr int NOUT = (TY * TZ + NT - 1) / NT;
  T fx_prev[NOUT];  // donor-cell flux through the x-face behind each owned output point
#pragma unroll
  for (int q = 0; q < NOUT; ++q) fx_prev[q] = T(0);

  for (int t = ts; t <= x1; ++t) {
    cp_wait_all();
    __syncthreads();
    // prefetch the planes of step t+1
    load_plane<P0R, NT>(P0(t + 3), A.in, t + 3, A.P0, j0, k0, A.P1, A.P2);
    load_plane<G0R, NT>(G0(t + 2), A.g0, t + 2, A.P0, j0, k0, A.P1, A.P2);
    load_plane<G1R, NT>(G1(t + 2), A.g1, t + 2, A.P0, j0, k0, A.P1, A.P2);
    load_plane<G2R, NT>(G2(t + 2), A.g2, t + 2, A.P0, j0, k0, A.P1, A.P2);
    cp_commit();

    // ---- psi1 at plane t+1 (upwind pass) and psi_min/max at plane t ----
    {
      const T *pm = P0(t), *pc = P0(t + 1), *pp = P0(t + 2);
      const T *gxm = G0(t), *gxp = G0(t + 1), *gy = G1(t + 1), *gz = G2(t + 1);
      T *out = P1(t + 1);
#pragma unroll 2
      for (int p = tid; p < P1R::size; p += NT) {
        const int j = P1R::j0 + p / P1R::nk, k = P1R::k0 + p % P1R::nk;
        const T c = pc[P0R::at(j, k)];
        const T fxp = flux(c, pp[P0R::at(j, k)], gxp[G0R::at(j, k)]);
        const T fxm = flux(pm[P0R::at(j, k)], c, gxm[G0R::at(j, k)]);
        const T fyp = flux(c, pc[P0R::at(j + 1, k)], gy[G1R::at(j, k)]);
        const T fym = flux(pc[P0R::at(j - 1, k)], c, gy[G1R::at(j - 1, k)]);
        const T fzp = flux(c, pc[P0R::at(j, k + 1)], gz[G2R::at(j, k)]);
        const T fzm = flux(pc[P0R::at(j, k - 1)], c, gz[G2R::at(j, k - 1)]);
        out[p] = c + ((-fxp + fxm) + (-fyp + fym) + (-fzp + fzm)) / T(1);
      }
      if (FCT) {
        const T *qm = P0(t - 1), *qc = P0(t), *qp = P0(t + 1);
#pragma unroll 2
        for (int p = tid; p < R1::size; p += NT) {
          const int j = R1::j0 + p / R1::nk, k = R1::k0 + p % R1::nk;
          const T c = qc[P0R::at(j, k)], a = qp[P0R::at(j, k)], b = qm[P0R::at(j, k)];
          const T d = qc[P0R::at(j + 1, k)], e = qc[P0R::at(j - 1, k)];
          const T f = qc[P0R::at(j, k + 1)], g = qc[P0R::at(j, k - 1)];
          MN[p] = mn(mn(mn(mn(mn(mn(c, a), b), d), e), f), g);
          MX[p] = mx(mx(mx(mx(mx(mx(c, a), b), d), e), f), g);
        }
      }
    }
    __syncthreads();

    // ---- antidiffusive pseudo-velocities: x-faces t+1/2, y/z faces of plane t ----
    {
      const T *pm = P1(t - 1), *pc = P1(t), *pp = P1(t + 1);
      const T *g0m = G0(t - 1), *g0c = G0(t);
      const T *g1c = G1(t), *g1p = G1(t + 1), *g2c = G2(t), *g2p = G2(t + 1);
      T *cx = CX(t), *cy = CY(t), *cz = CZ(t);
      auto nd4 = [](T a, T b, T c, T d) -> T {
        if (IGA) return (a + b - c - d) / T(4);
        return frac(a + b - c - d, a + b + c + d);
      };
      auto ndx = [](T p1, T p0) -> T {
        if (IGA) return p1 - p0;  // 3D iga form (formulae_mpdata_psi_3d.hpp:304-318)
        return T(2) * frac(p1 - p0, p1 + p0);
      };
      // x-faces (dim 0; frame a = x, b = y, c = z)
#pragma unroll 1
      for (int p = tid; p < R1::size; p += NT) {
        const int j = R1::j0 + p / R1::nk, k = R1::k0 + p % R1::nk;
        const T C = g0c[G0R::at(j, k)];
        const T a0 = pc[P1R::at(j, k)], a1 = pp[P1R::at(j, k)];
        const T ny = nd4(pp[P1R::at(j + 1, k)], pc[P1R::at(j + 1, k)], pp[P1R::at(j - 1, k)], pc[P1R::at(j - 1, k)]);
        const T nz = nd4(pp[P1R::at(j, k + 1)], pc[P1R::at(j, k + 1)], pp[P1R::at(j, k - 1)], pc[P1R::at(j, k - 1)]);
        const T gc1 = (g1p[G1R::at(j, k)] + g1c[G1R::at(j, k)] + g1p[G1R::at(j - 1, k)] + g1c[G1R::at(j - 1, k)]) / T(4);
        const T gc2 = (g2p[G2R::at(j, k)] + g2c[G2R::at(j, k)] + g2p[G2R::at(j, k - 1)] + g2c[G2R::at(j, k - 1)]) / T(4);
        cx[p] = fabs(C) / T(2) * (T(1) - fabs(C) / T(1)) * ndx(a1, a0) - C / T(2) * (gc1 * ny + gc2 * nz) / T(1);
      }
      // y-faces j+1/2 of plane t (dim 1; frame a = y, b = z, c = x)
#pragma unroll 1
      for (int p = tid; p < CYR::size; p += NT) {
        const int j = CYR::j0 + p / CYR::nk, k = CYR::k0 + p % CYR::nk;
        const T C = g1c[G1R::at(j, k)];
        const T a0 = pc[P1R::at(j, k)], a1 = pc[P1R::at(j + 1, k)];
        const T ny = nd4(pc[P1R::at(j + 1, k + 1)], pc[P1R::at(j, k + 1)], pc[P1R::at(j + 1, k - 1)], pc[P1R::at(j, k - 1)]);
        const T nz = nd4(pp[P1R::at(j + 1, k)], pp[P1R::at(j, k)], pm[P1R::at(j + 1, k)], pm[P1R::at(j, k)]);
        const T gc1 = (g2c[G2R::at(j + 1, k)] + g2c[G2R::at(j, k)] + g2c[G2R::at(j + 1, k - 1)] + g2c[G2R::at(j, k - 1)]) / T(4);
        const T gc2 = (g0c[G0R::at(j + 1, k)] + g0c[G0R::at(j, k)] + g0m[G0R::at(j + 1, k)] + g0m[G0R::at(j, k)]) / T(4);
        cy[p] = fabs(C) / T(2) * (T(1) - fabs(C) / T(1)) * ndx(a1, a0) - C / T(2) * (gc1 * ny + gc2 * nz) / T(1);
      }
      // z-faces k+1/2 of plane t (dim 2; frame a = z, b = x, c = y)
#pragma unroll 1
      for (int p = tid; p < CZR::size; p += NT) {
        const int j = CZR::j0 + p / CZR::nk, k = CZR::k0 + p % CZR::nk;
        const T C = g2c[G2R::at(j, k)];
        const T a0 = pc[P1R::at(j, k)], a1 = pc[P1R::at(j, k + 1)];
        const T ny = nd4(pp[P1R::at(j, k + 1)], pp[P1R::at(j, k)], pm[P1R::at(j, k + 1)], pm[P1R::at(j, k)]);
        const T nz = nd4(pc[P1R::at(j + 1, k + 1)], pc[P1R::at(j + 1, k)], pc[P1R::at(j - 1, k + 1)], pc[P1R::at(j - 1, k)]);
        const T gc1 = (g0c[G0R::at(j, k + 1)] + g0c[G0R::at(j, k)] + g0m[G0R::at(j, k + 1)] + g0m[G0R::at(j, k)]) / T(4);
        const T gc2 = (g1c[G1R::at(j, k + 1)] + g1c[G1R::at(j, k)] + g1c[G1R::at(j - 1, k + 1)] + g1c[G1R::at(j - 1, k)]) / T(4);
        cz[p] = fabs(C) / T(2) * (T(1) - fabs(C) / T(1)) * ndx(a1, a0) - C / T(2) * (gc1 * ny + gc2 * nz) / T(1);
      }
    }
    __syncthreads();

    // ---- FCT betas at plane t ----
    if (FCT) {
      const T *pm = P1(t - 1), *pc = P1(t), *pp = P1(t + 1);
      const T *cxm = CX(t - 1), *cxc = CX(t), *cy = CY(t), *cz = CZ(t);
      T *bu = BU(t), *bd = BD(t);
#pragma unroll 1
      for (int p = tid; p < R1::size; p += NT) {
        const int j = R1::j0 + p / R1::nk, k = R1::k0 + p % R1::nk;
        const T c = pc[P1R::at(j, k)];
        const T xp = pp[P1R::at(j, k)], xm = pm[P1R::at(j, k)];
        const T yp = pc[P1R::at(j + 1, k)], ym = pc[P1R::at(j - 1, k)];
        const T zp = pc[P1R::at(j, k + 1)], zm = pc[P1R::at(j, k - 1)];
        // fluxes for the denominators (iga: the pseudo-velocity itself)
        T fxm = cxm[p], fxp = cxc[p], fym = cy[CYR::at(j - 1, k)], fyp = cy[CYR::at(j, k)];
        T fzm = cz[CZR::at(j, k - 1)], fzp = cz[CZR::at(j, k)];
        if (!IGA) {
          fxm = flux(xm, c, fxm); fxp = flux(c, xp, fxp);
          fym = flux(ym, c, fym); fyp = flux(c, yp, fyp);
          fzm = flux(zm, c, fzm); fzp = flux(c, zp, fzp);
        }
        const T hi = mx(MX[p], mx(c, mx(xp, mx(xm, mx(yp, mx(ym, mx(zp, zm)))))));
        const T lo = mn(MN[p], mn(yp, mn(xm, mn(c, mn(xp, mn(zp, mn(zm, ym)))))));
        const T du = (pos(fxm) - neg(fxp)) + (pos(fym) - neg(fyp)) + (pos(fzm) - neg(fzp));
        const T dd = (pos(fxp) - neg(fxm)) + (pos(fyp) - neg(fym)) + (pos(fzp) - neg(fzm));
        bu[p] = (hi - c) * T(1) / (du + lims<T>::eps());
        bd[p] = (c - lo) * T(1) / (dd + lims<T>::eps());
      }
      __syncthreads();
    }

    // ---- limited pseudo-velocities and corrective donor-cell pass at plane t-1 ----
    {
      const int x = t - 1;
      const T *pc = P1(x), *pp = P1(t);
      const T *cxc = CX(x), *cy = CY(x), *cz = CZ(x);
      const T *bu0 = BU(x), *bd0 = BD(x), *bu1 = BU(t), *bd1 = BD(t);
      auto lim = [](T C, T bd_l, T bu_r, T bu_l, T bd_r) -> T {
        return C > T(0) ? mn(T(1), mn(bd_l, bu_r)) : mn(T(1), mn(bu_l, bd_r));
      };
      // y / z faces into smem
#pragma unroll 1
      for (int p = tid; p < MYR::size; p += NT) {
        const int j = MYR::j0 + p / MYR::nk, k = MYR::k0 + p % MYR::nk;
        T C = cy[CYR::at(j, k)];
        if (FCT) C = C * lim(C, bd0[R1::at(j, k)], bu0[R1::at(j + 1, k)], bu0[R1::at(j, k)], bd0[R1::at(j + 1, k)]);
        MY[p] = IGA ? C : flux(pc[P1R::at(j, k)], pc[P1R::at(j + 1, k)], C);
      }
#pragma unroll 1
      for (int p = tid; p < MZR::size; p += NT) {
        const int j = MZR::j0 + p / MZR::nk, k = MZR::k0 + p % MZR::nk;
        T C = cz[CZR::at(j, k)];
        if (FCT) C = C * lim(C, bd0[R1::at(j, k)], bu0[R1::at(j, k + 1)], bu0[R1::at(j, k)], bd0[R1::at(j, k + 1)]);
        MZ[p] = IGA ? C : flux(pc[P1R::at(j, k)], pc[P1R::at(j, k + 1)], C);
      }
      __syncthreads();
      const bool write = x >= x0 && x < x1;
#pragma unroll
      for (int q = 0; q < NOUT; ++q) {
        const int p = tid + q * NT;
        if (p >= TY * TZ) break;
        const int j = p / TZ, k = p % TZ;
        // x-face x+1/2
        T C = cxc[R1::at(j, k)];
        if (FCT) C = C * lim(C, bd0[R1::at(j, k)], bu1[R1::at(j, k)], bu0[R1::at(j, k)], bd1[R1::at(j, k)]);
        const T fxp = IGA ? C : flux(pc[P1R::at(j, k)], pp[P1R::at(j, k)], C);
        const T fxm = fx_prev[q];
        fx_prev[q] = fxp;
        if (write) {
          const int jg = j0 + j, kg = k0 + k;
          if (jg < A.P1 && kg < A.P2) {
            const T v = pc[P1R::at(j, k)] + ((-fxp + fxm) + (-MY[MYR::at(j, k)] + MY[MYR::at(j - 1, k)]) +
                                              (-MZ[MZR::at(j, k)] + MZ[MZR::at(j, k - 1)])) / T(1);
            // the point and its cyclic duplicates at index n-1 (bcond/cyclic_3d.hpp convention)
            const int xs[2] = {x, x == 0 ? A.n0 - 1 : -1};
            const int js[2] = {jg, jg == 0 ? A.n1 - 1 : -1};
            const int ks[2] = {kg, kg == 0 ? A.n2 - 1 : -1};
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
              for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int c = 0; c < 2; ++c)
                  if (xs[a] >= 0 && js[b] >= 0 && ks[c] >= 0) A.out(xs[a], js[b], ks[c]) = v;
          }
        }
      }
    }
  }
  cp_wait_all();
}

}  // namespace f3
}  // namespace mpdx
